// Fused step kernels with float storage and float arithmetic.
#include "lbf_inst.cuh"
namespace lbf {
StepLauncher step_launcher_f32(int lat, int ho, int tc) { return step_table<float, float>(lat, ho, tc); }
BatchOps batch_ops_f32(int lat, int ho, int tc) { return batch_table<float, float>(lat, ho, tc); }
}  // namespace lbf
