// Fused step kernels with __half storage and float arithmetic, tiles of 32 x 8 nodes.
#include "lbf_inst.cuh"
namespace lbf {
LBF_INSTANTIATE(f16, __half, float, 8)
}  // namespace lbf
