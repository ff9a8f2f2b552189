// lbf_handle.h -- the device state behind an lbf_handle and the internal
// hooks the batched server (lbf_server.cu) shares with the single-box C ABI
// (lbf_capi.cu).  Not part of the C ABI.
#pragma once
#include <cuda_runtime.h>

#include "../../include/lbfast_gpu.h"
#include "lbf_internal.h"

struct lbf_handle {
    lbf_params p;
    int nx = 0, ny = 0, nz = 0;
    long long N = 0;
    int storage = 0;
    size_t esz = 4, psz = 4;
    bool tc = false, dr = false, obs = false;
    double omega = 0, beta = 0, kapp = 0, sharp_c = 0;
    double scale[lbf::NSCALE_H];
    void* mom[2] = {nullptr, nullptr};
    void* uold[2] = {nullptr, nullptr};
    void* phi[2] = {nullptr, nullptr};
    float* pres[2] = {nullptr, nullptr};  // P in FP32 when the other moments are 16-bit
    int8_t* isf = nullptr;
    bool isf_set = false;
    int cur = 0;
    long long step = 0;
    bool fields_set = false, primed = false;
    bool u_valid = false;  // uold[cur] holds the post-force velocity of the last step
    // wetting
    int nwet = 0;
    long long* wet_s = nullptr;
    int* wet_donor = nullptr;
    int* wet_flag = nullptr;
    double* wet_wn = nullptr;
    int* wet_shift = nullptr;
    void* wetW[2] = {nullptr, nullptr};
    int wet_pending = -1;         // W buffer holding ghost values not yet written
    int wet_pending_target = -1;  // phi buffer they belong to
    double cot_theta = 0;
    cudaStream_t stream = nullptr;
    int* d_err = nullptr;
    double* d_red = nullptr;
    void* staging = nullptr;
    size_t staging_bytes = 0;
    lbf::StepLauncher launcher = nullptr;
    int zseg = 0;
    int tile_y = 8;      // rows of the kernel tile
    double* d_mass = nullptr;  // phi correction: {sum, count, sum at the first step, face flux} (FP64)
    int obc_open = 0;  // open faces (openbc, non-periodic axes): bit 0 x, 1 y, 2 z
    long long* bb_nodes = nullptr;  // BOUNCE_BACK: the isfluid = -1 nodes
    long long nbb = 0;
    double* d_rnrm = nullptr;  // REPULSIVE_FLUX: normals (3 x N, FP64)
    void* d_rep = nullptr;     // REPULSIVE_FLUX: force of the step (3 x N, arithmetic type)
    bool tuned = true;   // false until the autotuner ran (tile_y = 0 requested)
    // z slab of a larger box (lbf_create_slab): the handle's box is the slab's
    // nzs planes plus SLAB_HALO halo planes on each side, filled from the
    // neighbouring slabs; zg0 is the slab's first plane in the global box of nzg
    bool slab = false;
    int zg0 = 0, nzs = 0, nzg = 0;
    // overlapped slab steps (lbf_slabs_step): the device, a stream for the
    // halo copies and events marking a step's end and the copies' end
    int device = 0;
    cudaStream_t xstream = nullptr;
    cudaEvent_t ev_done = nullptr, ev_copied = nullptr;
};

namespace lbf {
// halo planes of a z slab on each side: the step's phase-field stencils reach
// three planes (phi for the gradient of theta of the collision's neighbours)
constexpr int SLAB_HALO = 3;
}  // namespace lbf

namespace lbf {
// integrator pre-loop work (wetting) of a freshly filled handle
int handle_prime(lbf_handle* h);
// launch arguments of the next step of h (its current time level)
void handle_step_args(const lbf_handle* h, StepArgs& a, bool write_u);
// bookkeeping after one step of h was launched
void handle_advance(lbf_handle* h, bool wrote_u);
// device bytes lbf_create allocates for these parameters
size_t handle_bytes(const lbf_params* p);
// per-step work of h launched before its step kernel (wetting ghost update)
int handle_pre_step(lbf_handle* h);
// per-step work after the step kernel, on the new time level (phi mass correction)
int handle_post_step(lbf_handle* h);
// true when the per-step work of h repeats with period two (replayable)
bool handle_steady(const lbf_handle* h);
// frees the host<->device staging buffer (reallocated on the next transfer)
void handle_release_staging(lbf_handle* h);
}  // namespace lbf
