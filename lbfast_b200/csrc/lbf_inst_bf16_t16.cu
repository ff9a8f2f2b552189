// Fused step kernels with __nv_bfloat16 storage and float arithmetic, tiles of 32 x 16 nodes.
#include "lbf_inst.cuh"
namespace lbf {
LBF_INSTANTIATE(bf16, __nv_bfloat16, float, 16)
}  // namespace lbf
