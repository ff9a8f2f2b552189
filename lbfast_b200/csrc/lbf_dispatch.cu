// lbf_dispatch.cu -- picks the instantiation unit of a storage type and tile height.
#include "../../include/lbfast_gpu.h"
#include "lbf_internal.h"

#include <algorithm>

namespace lbf {

StepLauncher step_launcher_f32_t8(int, int, int, int);
StepLauncher step_launcher_f32_t16(int, int, int, int);
StepLauncher step_launcher_f16_t8(int, int, int, int);
StepLauncher step_launcher_f16_t16(int, int, int, int);
StepLauncher step_launcher_bf16_t8(int, int, int, int);
StepLauncher step_launcher_bf16_t16(int, int, int, int);
StepLauncher step_launcher_f64_t8(int, int, int, int);
BatchOps batch_ops_f32_t8(int, int, int, int);
BatchOps batch_ops_f32_t16(int, int, int, int);
BatchOps batch_ops_f16_t8(int, int, int, int);
BatchOps batch_ops_f16_t16(int, int, int, int);
BatchOps batch_ops_bf16_t8(int, int, int, int);
BatchOps batch_ops_bf16_t16(int, int, int, int);
BatchOps batch_ops_f64_t8(int, int, int, int);

int resident_slots(int resident_per_sm) {
    static int nsm = 0;
    if (!nsm) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            nsm = 148;
    }
    return nsm * resident_per_sm;
}

// every resident CTA slot of the GPU, but no share shorter than 8 planes
int persistent_grid(long long W, int resident_per_sm) {
    constexpr long long MIN_SHARE = 8;
    const long long slots = resident_slots(resident_per_sm);
    return (int)std::max<long long>(1, std::min(slots, (W + MIN_SHARE - 1) / MIN_SHARE));
}

bool tile_available(int storage, int tile_y) {
    if (tile_y == 8) return true;
    return tile_y == 16 && storage != LBF_STORE_F64;  // FP64 rings of 16 rows exceed shared memory
}

StepLauncher step_launcher(int storage, int lat, int ho, int tc, int obs, int tile_y) {
    const bool t16 = tile_y == 16;
    switch (storage) {
        case LBF_STORE_F32: return t16 ? step_launcher_f32_t16(lat, ho, tc, obs) : step_launcher_f32_t8(lat, ho, tc, obs);
        case LBF_STORE_F16: return t16 ? step_launcher_f16_t16(lat, ho, tc, obs) : step_launcher_f16_t8(lat, ho, tc, obs);
        case LBF_STORE_BF16: return t16 ? step_launcher_bf16_t16(lat, ho, tc, obs) : step_launcher_bf16_t8(lat, ho, tc, obs);
        case LBF_STORE_F64: return t16 ? nullptr : step_launcher_f64_t8(lat, ho, tc, obs);
    }
    return nullptr;
}

BatchOps batch_ops(int storage, int lat, int ho, int tc, int obs, int tile_y) {
    const bool t16 = tile_y == 16;
    switch (storage) {
        case LBF_STORE_F32: return t16 ? batch_ops_f32_t16(lat, ho, tc, obs) : batch_ops_f32_t8(lat, ho, tc, obs);
        case LBF_STORE_F16: return t16 ? batch_ops_f16_t16(lat, ho, tc, obs) : batch_ops_f16_t8(lat, ho, tc, obs);
        case LBF_STORE_BF16: return t16 ? batch_ops_bf16_t16(lat, ho, tc, obs) : batch_ops_bf16_t8(lat, ho, tc, obs);
        case LBF_STORE_F64: if (!t16) return batch_ops_f64_t8(lat, ho, tc, obs);
    }
    BatchOps none{};
    return none;
}

}  // namespace lbf
