// Fused step kernels with __half storage and float arithmetic.
#include "lbf_inst.cuh"
namespace lbf {
StepLauncher step_launcher_f16(int lat, int ho, int tc) { return step_table<__half, float>(lat, ho, tc); }
BatchOps batch_ops_f16(int lat, int ho, int tc) { return batch_table<__half, float>(lat, ho, tc); }
}  // namespace lbf
