// Fused step kernels with double storage and double arithmetic, tiles of 32 x 8 nodes.
#include "lbf_inst.cuh"
namespace lbf {
LBF_INSTANTIATE(f64, double, double, 8)
}  // namespace lbf
