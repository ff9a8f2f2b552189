// lbf_noalloc.cu -- FP64 sums over caller-owned device fields without any
// device allocation.
//
// Some callers cannot let a library allocate device memory while they run:
// a Fortran integrator whose device arrays live inside OpenACC data regions
// owns every device buffer and hands the library only device pointers; a
// host application that hands out all device memory from its own pool does
// not want a second allocator beside it; a solver running inside a fixed
// device-memory budget cannot have a call grow its footprint (the allocation
// could fail mid-run or push it over).
// lbf_reduce_noalloc serves them: the caller passes the fields and receives
// the five sums, and the only scratch the computation needs -- one partial
// sum per z plane -- lives in a file-scope __device__ array that exists
// from module load to process exit.
//
// The scratch array holds LBF_NOALLOC_MAX_PLANES planes of five doubles plus
// the five totals (328 KB per GPU that loads the library).  Boxes with more z
// planes are rejected.  Every slot a call reads is written earlier in the same
// call, so nothing needs clearing between calls; calls that overlap on the
// GPU (other streams or host threads) share the array and race.
//
// The field pointers come straight from the caller, so before anything is
// launched each one is checked to be device (or managed) memory of the
// current device: a host address passed by mistake -- a Fortran call without
// `host_data use_device` -- is rejected with LBF_E_ARG instead of being read
// from the GPU.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>

#include "../../include/lbfast_gpu.h"
#include "lbf_internal.h"

namespace {

constexpr int NRED = 5;
constexpr int RED_THREADS = 256;

static __device__ __align__(256) double g_plane_sums[(LBF_NOALLOC_MAX_PLANES + 1) * NRED];

// failures are reported through lbf_last_error, like every other entry point
int fail(int code, const char* msg, cudaError_t e = cudaSuccess) {
    char buf[384];
    if (e != cudaSuccess)
        std::snprintf(buf, sizeof(buf), "lbf_reduce_noalloc: %s (%s)", msg, cudaGetErrorString(e));
    else
        std::snprintf(buf, sizeof(buf), "lbf_reduce_noalloc: %s", msg);
    lbf::record_error(buf);
    return code;
}

// LBF_OK when p is device or managed memory that the current device `dev` can
// read as a plain device pointer
int check_device_pointer(const void* p, int dev, const char* name) {
    cudaPointerAttributes a{};
    cudaError_t e = cudaPointerGetAttributes(&a, p);
    if (e != cudaSuccess) {
        cudaGetLastError();  // the failed query leaves a (non-sticky) error behind: clear it
        char msg[160];
        std::snprintf(msg, sizeof(msg), "%s is not a pointer the CUDA runtime knows", name);
        return fail(LBF_E_ARG, msg, e);
    }
    const bool dev_mem = a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
    if (!dev_mem || (a.type == cudaMemoryTypeDevice && a.device != dev)) {
        char msg[200];
        std::snprintf(msg, sizeof(msg),
                      "%s must be device memory of the current device %d (got %s); from Fortran pass it "
                      "inside `!$acc host_data use_device(...)`",
                      name, dev,
                      a.type == cudaMemoryTypeDevice ? "another device's memory"
                      : a.type == cudaMemoryTypeHost ? "pinned host memory"
                                                     : "host memory");
        return fail(LBF_E_ARG, msg);
    }
    return LBF_OK;
}

__device__ __forceinline__ void block_sum(double (&acc)[NRED], double (*red)[RED_THREADS]) {
#pragma unroll
    for (int k = 0; k < NRED; ++k) red[k][threadIdx.x] = acc[k];
    __syncthreads();
    for (int s = RED_THREADS / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s)
#pragma unroll
            for (int k = 0; k < NRED; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + s];
        __syncthreads();
    }
}

// one block per z plane: fixed-order sums of phi, P, u, v, w over fluid nodes
__global__ void __launch_bounds__(RED_THREADS) plane_sums_kernel(const float* mom, const float* phi,
                                                                 const int8_t* isf, long long plane, long long n,
                                                                 double* sums) {
    __shared__ double red[NRED][RED_THREADS];
    double acc[NRED] = {0, 0, 0, 0, 0};
    const long long base = (long long)blockIdx.x * plane;
    for (long long i = threadIdx.x; i < plane; i += RED_THREADS) {
        const long long c = base + i;
        if (isf) {
            const int f = isf[c];
            if (f != 1 && f != -1) continue;
        }
        if (phi) acc[0] += (double)phi[c];
        acc[1] += (double)mom[c];
        acc[2] += (double)mom[n + c];
        acc[3] += (double)mom[2 * n + c];
        acc[4] += (double)mom[3 * n + c];
    }
    block_sum(acc, red);
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < NRED; ++k) sums[blockIdx.x * NRED + k] = red[k][0];
}

// one block: fixed-order sum of the nz plane partials into the five totals
__global__ void __launch_bounds__(RED_THREADS) total_kernel(double* sums, int nz) {
    __shared__ double red[NRED][RED_THREADS];
    double acc[NRED] = {0, 0, 0, 0, 0};
    for (int z = threadIdx.x; z < nz; z += RED_THREADS)
#pragma unroll
        for (int k = 0; k < NRED; ++k) acc[k] += sums[z * NRED + k];
    block_sum(acc, red);
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < NRED; ++k) sums[LBF_NOALLOC_MAX_PLANES * NRED + k] = red[k][0];
}

}  // namespace

extern "C" int lbf_reduce_noalloc(const float* mom10, const float* phi, const int8_t* isfluid, int lx, int ly,
                                  int lz, double out[5]) {
    if (!mom10 || !out) return fail(LBF_E_ARG, "mom10 and out must not be NULL");
    if (lx < 1 || ly < 1 || lz < 1) return fail(LBF_E_ARG, "box dimensions must be positive");
    if (lz > LBF_NOALLOC_MAX_PLANES) {
        char msg[160];
        std::snprintf(msg, sizeof(msg), "lz = %d exceeds the %d z planes of the static scratch array", lz,
                      LBF_NOALLOC_MAX_PLANES);
        return fail(LBF_E_ARG, msg);
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(LBF_E_CUDA, "cudaGetDevice failed", e);
    int rc = check_device_pointer(mom10, dev, "mom10");
    if (rc == LBF_OK && phi) rc = check_device_pointer(phi, dev, "phi");
    if (rc == LBF_OK && isfluid) rc = check_device_pointer(isfluid, dev, "isfluid");
    if (rc != LBF_OK) return rc;
    // device address of the scratch array on the current device, looked up on
    // every call (a host-side query: host code cannot use the symbol itself as
    // a device address, and a looked-up address would go stale after a
    // cudaDeviceReset).  The first call on a device also loads this file's
    // kernels there, so make it before any stream capture.
    void* ptr = nullptr;
    e = cudaGetSymbolAddress(&ptr, g_plane_sums);
    if (e != cudaSuccess || !ptr) return fail(LBF_E_CUDA, "cudaGetSymbolAddress of the scratch array failed", e);
    double* sums = static_cast<double*>(ptr);
    const long long plane = (long long)lx * ly;
    const long long n = plane * lz;
    plane_sums_kernel<<<lz, RED_THREADS>>>(mom10, phi, isfluid, plane, n, sums);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(LBF_E_CUDA, "plane sum launch failed", e);
    total_kernel<<<1, RED_THREADS>>>(sums, lz);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(LBF_E_CUDA, "total launch failed", e);
    e = cudaMemcpy(out, sums + (long long)LBF_NOALLOC_MAX_PLANES * NRED, NRED * sizeof(double),
                   cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return fail(LBF_E_CUDA, "copy of the totals failed", e);
    // a diverged state is reported the way lbf_reduce reports it
    static const char* const names[NRED] = {"phi", "P", "u", "v", "w"};
    for (int k = 0; k < NRED; ++k)
        if (!std::isfinite(out[k])) {
            char msg[128];
            std::snprintf(msg, sizeof(msg), "the sum of %s over the fluid is not finite", names[k]);
            return fail(LBF_E_NUMERIC, msg);
        }
    return LBF_OK;
}
