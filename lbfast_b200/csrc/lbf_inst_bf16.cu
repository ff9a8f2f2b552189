// Fused step kernels with __nv_bfloat16 storage and float arithmetic.
#include "lbf_inst.cuh"
namespace lbf {
StepLauncher step_launcher_bf16(int lat, int ho, int tc) { return step_table<__nv_bfloat16, float>(lat, ho, tc); }
BatchOps batch_ops_bf16(int lat, int ho, int tc) { return batch_table<__nv_bfloat16, float>(lat, ho, tc); }
}  // namespace lbf
