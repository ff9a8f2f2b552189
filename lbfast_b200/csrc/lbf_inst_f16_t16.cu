// Fused step kernels with __half storage and float arithmetic, tiles of 32 x 16 nodes.
#include "lbf_inst.cuh"
namespace lbf {
LBF_INSTANTIATE(f16, __half, float, 16)
}  // namespace lbf
