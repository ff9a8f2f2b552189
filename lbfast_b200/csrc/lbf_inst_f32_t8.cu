// Fused step kernels with float storage and float arithmetic, tiles of 32 x 8 nodes.
#include "lbf_inst.cuh"
namespace lbf {
LBF_INSTANTIATE(f32, float, float, 8)
}  // namespace lbf
