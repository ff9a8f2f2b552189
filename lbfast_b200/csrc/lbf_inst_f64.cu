// Fused step kernels with double storage and double arithmetic.
#include "lbf_inst.cuh"
namespace lbf {
StepLauncher step_launcher_f64(int lat, int ho, int tc) { return step_table<double, double>(lat, ho, tc); }
BatchOps batch_ops_f64(int lat, int ho, int tc) { return batch_table<double, double>(lat, ho, tc); }
}  // namespace lbf
