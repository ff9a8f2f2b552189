// Fused step kernels with float storage and float arithmetic, tiles of 32 x 16 nodes.
#include "lbf_inst.cuh"
namespace lbf {
LBF_INSTANTIATE(f32, float, float, 16)
}  // namespace lbf
