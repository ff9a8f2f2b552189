// lbf_capi.cu -- implementation of include/lbfast_gpu.h: device state,
// step orchestration and the host boundary.
//
// Step orchestration (integrator_module.f90:266-827 on one GPU): per time
// step one launch of the fused kernel, preceded -- with obstacles and two
// components -- by the wetting kernel.  The reference's per-launch
// cudaDeviceSynchronize (lb_cuda_driver_module.f90:944-983) is dropped:
// launches are stream-ordered and errors are checked at synchronising calls.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/lbfast_gpu.h"
#include "lbf_internal.h"
#include "lbf_handle.h"

namespace {

thread_local std::string g_last_error;

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

#define CUDA_TRY(expr)                                                                       \
    do {                                                                                     \
        cudaError_t e_ = (expr);                                                             \
        if (e_ != cudaSuccess)                                                               \
            return fail(LBF_E_CUDA, "%s: %s (%s:%d)", #expr, cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

// D3Q27 link table (vars_module.f90:319-338); D3Q19 = first 19 links
const int EXh[27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, 1, -1, -1, 1, 1, -1};
const int EYh[27] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, -1, 1, -1, 1};
const int EZh[27] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1};
// is D3Q27 link l a link of the lattice: D3Q19 = links 0-18, D3Q15 = links 0-6 and 19-26
bool link_in(int lat, int l) { return lat == 27 || (lat == 19 ? l < 19 : (l < 7 || l >= 19)); }

}  // namespace

namespace lbf {
void record_error(const char* msg) { g_last_error = msg; }
}  // namespace lbf



namespace {

int ensure_staging(lbf_handle* h, size_t bytes) {
    if (h->staging_bytes >= bytes) return LBF_OK;
    if (h->staging) cudaFree(h->staging);
    h->staging = nullptr;
    h->staging_bytes = 0;
    if (cudaMalloc(&h->staging, bytes) != cudaSuccess)
        return fail(LBF_E_NOMEM, "device staging allocation of %zu bytes failed", bytes);
    h->staging_bytes = bytes;
    return LBF_OK;
}

void free_all(lbf_handle* h) {
    for (int b = 0; b < 2; ++b) {
        cudaFree(h->mom[b]);
        cudaFree(h->uold[b]);
        cudaFree(h->phi[b]);
        cudaFree(h->pres[b]);
        cudaFree(h->wetW[b]);
    }
    cudaFree(h->isf);
    cudaFree(h->wet_s);
    cudaFree(h->wet_donor);
    cudaFree(h->wet_flag);
    cudaFree(h->wet_wn);
    cudaFree(h->wet_shift);
    cudaFree(h->d_err);
    cudaFree(h->d_red);
    cudaFree(h->d_mass);
    cudaFree(h->bb_nodes);
    cudaFree(h->d_rnrm);
    cudaFree(h->d_rep);
    cudaFree(h->staging);
    if (h->xstream) cudaStreamDestroy(h->xstream);
    if (h->ev_done) cudaEventDestroy(h->ev_done);
    if (h->ev_copied) cudaEventDestroy(h->ev_copied);
}

// automatic z segment: enough CTAs for about four waves on 148 SMs (two CTAs
// of 8 rows or one of 16 rows per SM), segments of at least 8 planes so the
// pipeline fill (5 planes) stays a small overhead
int auto_zseg(int nx, int ny, int nz, int tile_y) {
    long long cols = (long long)((nx + 31) / 32) * ((ny + tile_y - 1) / tile_y);
    long long target = 148LL * 4 * (tile_y == 8 ? 2 : 1);
    int nseg = (int)std::max<long long>(1, (target + cols - 1) / cols);
    int zseg = (nz + nseg - 1) / nseg;
    zseg = std::max(zseg, std::min(nz, 8));
    return zseg;
}

// Split planes for a box whose columns fill less than one wave of CTA slots:
// L such that the heads [0, L) on ncols slots and the tails [L, nzr) on the
// other slots (ceil(ncols / free) rounds of them) end together, for tails
// that run s times slower per plane (their halo re-reads miss the L2 that
// columns in step share) and a pipeline fill of 4 planes per segment; s from
// 1 to 1.5.  Measured at 256^3 (128 columns, 148 SMs): whole columns 1.027 ms,
// split at 229 0.924, at 233 0.940, at 220 1.039 -- the tails become the
// longer part below the optimum, so the autotuner times several planes.
std::vector<int> split_planes(int nx, int ny, int nzr, int tile_y, int storage) {
    std::vector<int> out;
    const long long cols = (long long)((nx + 31) / 32) * ((ny + tile_y - 1) / tile_y);
    const long long slots = lbf::resident_slots((tile_y == 8 && storage != LBF_STORE_F64) ? 2 : 1);
    if (cols >= slots || nzr < 16) return out;
    constexpr double FILL = 4.0;
    const double rounds = (double)((cols + (slots - cols) - 1) / (slots - cols));
    for (int i = 0; i <= 10; ++i) {
        const double s = 1.0 + 0.05 * i;
        const int L = (int)std::lround((rounds * (nzr + FILL) * s - FILL) / (1.0 + rounds * s));
        if (L >= 8 && L < nzr && std::find(out.begin(), out.end(), L) == out.end()) out.push_back(L);
    }
    return out;
}

// ---- autotuner of the schedule ----
// The tile height is fixed per storage (default_tile): kernels of different
// tile heights are different compilations whose floating-point contractions
// may differ in the last bit, while one kernel gives the same bits for every
// z segmentation and schedule -- so the tuned result is reproducible from run
// to run whatever the timings.  Every candidate launch steps the current time
// level into the other buffer set, which the next real step overwrites, so
// timing on the box's own fields leaves its state unchanged (wetting, which
// changes host-side state, is not part of a trial).  The winner is remembered
// per box shape and class.
struct TuneKey {
    int v[12];
    bool operator<(const TuneKey& o) const { return std::lexicographical_compare(v, v + 12, o.v, o.v + 12); }
};
std::mutex g_tune_mu;
std::map<TuneKey, std::pair<int, int>> g_tune_cache;

TuneKey tune_key(const lbf_handle* h) {
    const lbf_params& p = h->p;
    return TuneKey{{p.storage, p.lattice, p.highorder, p.twocomponent, p.densratio, p.obstacles, p.lx, p.ly, p.lz,
                    p.pbc_x * 4 + p.pbc_y * 2 + p.pbc_z, p.zseg, 0}};
}

int autotune(lbf_handle* h) {
    h->tuned = true;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CUDA_TRY(cudaStreamIsCapturing(h->stream, &cs));
    if (cs != cudaStreamCaptureStatusNone) return LBF_OK;  // keep the defaults inside a capture
    const TuneKey key = tune_key(h);
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) {
            h->tile_y = it->second.first;
            h->zseg = it->second.second;
            h->launcher = lbf::step_launcher(h->storage, h->p.lattice, h->p.highorder, lbf::kernel_tc(h->p), lbf::kernel_obs(h->p), h->tile_y);
            return LBF_OK;
        }
    }
    std::vector<std::pair<int, int>> cand;
    for (int ty : {h->tile_y}) {
        std::vector<int> zs;
        if (h->p.zseg != 0) {
            zs.push_back(h->zseg);
        } else {
            // the persistent schedule (0), and fixed segments: about four waves,
            // half and twice that, and whole columns.  Segments keep the CTAs
            // that run together on neighbouring columns at the same planes, so
            // halo re-reads hit in L2; the persistent schedule balances the SMs
            // exactly but staggers neighbours in z.
            const int za = auto_zseg(h->nx, h->ny, h->nz, ty), lo = std::min(h->nz, 8);
            std::vector<int> all = {0, za, std::max(lo, za / 2), std::min(h->nz, 2 * za), h->nz};
            // split columns (negative: the split plane)
            for (int L : split_planes(h->nx, h->ny, h->slab ? h->nzs : h->nz, ty, h->storage)) all.push_back(-L);
            for (int z : all)
                if (std::find(zs.begin(), zs.end(), z) == zs.end()) zs.push_back(z);
        }
        for (int z : zs) cand.emplace_back(ty, z);
    }
    cudaEvent_t e0, e1;
    CUDA_TRY(cudaEventCreate(&e0));
    CUDA_TRY(cudaEventCreate(&e1));
    float best = 1e30f;
    std::pair<int, int> pick(h->tile_y, h->zseg);
    int rc = LBF_OK;
    for (const auto& c : cand) {
        lbf::StepLauncher L = lbf::step_launcher(h->storage, h->p.lattice, h->p.highorder, lbf::kernel_tc(h->p), lbf::kernel_obs(h->p), c.first);
        if (!L) continue;
        lbf::StepArgs a;
        const int zs0 = h->zseg;
        h->zseg = c.second;
        lbf::handle_step_args(h, a, h->dr);
        h->zseg = zs0;
        cudaError_t e = L(a, h->stream);  // warm-up (first use sets the kernel's shared-memory limit)
        if (e == cudaSuccess) e = cudaEventRecord(e0, h->stream);
        for (int k = 0; k < 3 && e == cudaSuccess; ++k) e = L(a, h->stream);
        if (e == cudaSuccess) e = cudaEventRecord(e1, h->stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        float ms = 0;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        if (e != cudaSuccess) {
            rc = fail(LBF_E_CUDA, "autotune launch: %s", cudaGetErrorString(e));
            break;
        }
        if (ms < best) {
            best = ms;
            pick = c;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    h->tile_y = pick.first;
    h->zseg = pick.second;
    h->launcher = lbf::step_launcher(h->storage, h->p.lattice, h->p.highorder, lbf::kernel_tc(h->p), lbf::kernel_obs(h->p), h->tile_y);
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_cache[key] = pick;
    return LBF_OK;
}

// phi carried through the open faces by the state of buffer b into d_mass[3]
// (stays 0 without open faces)
cudaError_t launch_face_flux(lbf_handle* h, int b) {
    if (!h->obc_open || !h->tc) return cudaSuccess;
    double inv[4];
    for (int f = 0; f < 4; ++f) inv[f] = 1.0 / h->scale[f];
    return lbf::launch_phi_flux(h->storage, h->nx, h->ny, h->nz, h->obc_open, h->mom[b], h->pres[b], h->phi[b], h->isf, inv,
                                h->d_mass + 3, h->stream);
}

// Pre-loop wetting of integrator_module.f90:186-190 / one launch per step.
int launch_wet(lbf_handle* h, int in_buf, int out_buf, bool prime) {
    if (!(h->tc && h->obs) || h->nwet == 0) return LBF_OK;
    lbf::WetArgs a;
    a.n = h->nwet;
    a.nx = h->nx; a.ny = h->ny; a.nz = h->nz;
    a.pbx = h->p.pbc_x; a.pby = h->p.pbc_y; a.pbz = h->p.pbc_z;
    a.s_idx = h->wet_s;
    a.donor = h->wet_donor;
    a.flag = h->wet_flag;
    a.wn = h->wet_wn;
    a.shift = h->wet_shift;
    a.cot_theta = h->cot_theta;
    a.pin = h->phi[in_buf];
    a.prime = prime ? 1 : 0;
    if (prime) {
        // in place: the wetting only reads fluid donors and the node's own value
        a.wout = h->wetW[0];
        a.scatter_dst = nullptr;
        a.scatter_src = nullptr;
        CUDA_TRY(lbf::launch_wetting(h->storage, a, h->stream));
        CUDA_TRY(lbf::launch_wet_apply(h->storage, h->nwet, h->wet_s, h->wetW[0], h->phi[in_buf], h->stream));
        return LBF_OK;
    }
    int wbuf = h->wet_pending >= 0 ? 1 - h->wet_pending : 0;
    // ghost values of the previous step belong to that step's input buffer,
    // which is this step's output buffer and is not read during this step
    if (h->wet_pending >= 0 && h->wet_pending_target == out_buf) {
        a.scatter_dst = h->phi[out_buf];
        a.scatter_src = h->wetW[h->wet_pending];
    } else {
        a.scatter_dst = nullptr;
        a.scatter_src = nullptr;
    }
    a.wout = h->wetW[wbuf];
    CUDA_TRY(lbf::launch_wetting(h->storage, a, h->stream));
    h->wet_pending = wbuf;
    h->wet_pending_target = in_buf;
    return LBF_OK;
}

// write pending ghost values into their phi buffer (before phi is read out)
int flush_wet(lbf_handle* h) {
    if (h->wet_pending < 0) return LBF_OK;
    CUDA_TRY(lbf::launch_wet_apply(h->storage, h->nwet, h->wet_s, h->wetW[h->wet_pending],
                                   h->phi[h->wet_pending_target], h->stream));
    return LBF_OK;
}

int prime(lbf_handle* h) {
    if (h->d_mass)
        CUDA_TRY(lbf::launch_mass(h->storage, lbf::MASS_INITIAL, h->N, h->phi[h->cur], h->obs ? h->isf : nullptr, h->d_mass,
                                  h->stream));
    int rc = launch_wet(h, h->cur, 1 - h->cur, true);
    if (rc) return rc;
    // with open faces the pre-loop bcs_mesoscopic_phifields corrects once with
    // the flux of the initial state (integrator_module.f90:179-182)
    if (h->d_mass && h->obc_open) {
        CUDA_TRY(launch_face_flux(h, h->cur));
        CUDA_TRY(lbf::launch_mass(h->storage, lbf::MASS_APPLY, h->N, h->phi[h->cur], h->isf, h->d_mass, h->stream));
    }
    h->primed = true;
    return LBF_OK;
}

// power-of-two storage scale of a 16-bit field group: FP16 carries an 11-bit
// significand over 30 binades (6.1e-5 .. 65504), so the scale only has to keep
// values in range; the largest expected magnitude (the data's, never below a
// physical floor) is mapped to [2^8, 2^9): 128x headroom before overflow,
// full precision for values down to ~1e-7 of it
double pick_scale(int storage, double maxabs, double floor_mag) {
    if (storage != LBF_STORE_F16 && storage != LBF_STORE_BF16) return 1.0;
    double m = std::max(maxabs, floor_mag);
    int e = (int)std::floor(std::log2(256.0 / m));
    return std::ldexp(1.0, e);
}

bool is_half(int storage) { return storage == LBF_STORE_F16 || storage == LBF_STORE_BF16; }

}  // namespace

extern "C" {

const char* lbf_version(void) { return "lbfast-b200 1.0 (sm_100a)"; }

int lbf_last_error(char* buf, size_t n) {
    if (!buf || n == 0) return LBF_E_ARG;
    std::snprintf(buf, n, "%s", g_last_error.c_str());
    return LBF_OK;
}

int lbf_create(const lbf_params* p, lbf_handle** out) {
    if (!p || !out) return fail(LBF_E_ARG, "lbf_create: null argument");
    *out = nullptr;
    if (p->lx < 1 || p->ly < 1 || p->lz < 1) return fail(LBF_E_ARG, "box must be at least 1^3");
    if ((long long)p->lx * p->ly * p->lz > (1LL << 31) - 1)
        return fail(LBF_E_ARG, "box of %lld nodes exceeds 2^31-1", (long long)p->lx * p->ly * p->lz);
    if (p->lattice != 15 && p->lattice != 19 && p->lattice != 27)
        return fail(LBF_E_UNSUPPORTED, "LATTICE %d not supported (15, 19 or 27)", p->lattice);
    if (p->highorder && p->lattice != 27) return fail(LBF_E_ARG, "HIGHORDER requires LATTICE 27");
    if (p->densratio && !p->twocomponent) return fail(LBF_E_ARG, "DENSRATIO requires TWOCOMPONENT");
    if (p->storage < 0 || p->storage > 3) return fail(LBF_E_ARG, "unknown storage %d", p->storage);
    if (p->visc1 <= 0 || (p->twocomponent && p->visc2 <= 0)) return fail(LBF_E_ARG, "viscosities must be positive");
    if (p->twocomponent && (p->width <= 0)) return fail(LBF_E_ARG, "interface width must be positive");
    if (p->densratio && (p->rho_r <= 0 || p->rho_b <= 0)) return fail(LBF_E_ARG, "densities must be positive");
    if (p->phi_correction && !p->twocomponent) return fail(LBF_E_ARG, "phi_correction requires TWOCOMPONENT");
    // bcs_mesoscopic_hfields / _phifields run only with INTERNAL_OBSTACLES (integrator_module.f90:514-523)
    if (p->openbc && !p->obstacles) return fail(LBF_E_ARG, "openbc requires obstacles (INTERNAL_OBSTACLES)");
    if (p->bounce_back && !p->obstacles) return fail(LBF_E_ARG, "bounce_back requires obstacles (INTERNAL_OBSTACLES)");
    if (p->repulsive_flux && !p->twocomponent) return fail(LBF_E_ARG, "repulsive_flux requires TWOCOMPONENT");
    // an open axis holds a wall, the face plane and a wall at least
    if (p->openbc && ((!p->pbc_x && p->lx < 3) || (!p->pbc_y && p->ly < 3) || (!p->pbc_z && p->lz < 3)))
        return fail(LBF_E_ARG, "openbc: a non-periodic axis needs at least 3 nodes");
    lbf_handle* h = new (std::nothrow) lbf_handle();
    if (!h) return fail(LBF_E_NOMEM, "host allocation failed");
    h->p = *p;
    h->nx = p->lx; h->ny = p->ly; h->nz = p->lz;
    h->N = (long long)p->lx * p->ly * p->lz;
    h->storage = p->storage;
    h->esz = lbf::storage_bytes(p->storage);
    h->psz = lbf::phi_bytes(p->storage);
    h->tc = p->twocomponent != 0;
    h->dr = p->densratio != 0;
    h->obs = p->obstacles != 0;
    // LBFAST.f90:212-219
    double tau1 = p->visc1 * 3.0 + 0.5;
    h->omega = 1.0 / tau1;
    if (h->tc) {
        h->beta = 12.0 * p->sigma / p->width;
        h->kapp = 1.5 * p->sigma * p->width;
        h->sharp_c = 4.0 * p->tau_diff / p->width;
    }
    {
        const double pi = 3.1415926535897932384626433832795028841971;
        double th = (180.0 - p->wettab_r) * pi / 180.0;
        double s = std::sin(th), c = std::cos(th);
        h->cot_theta = std::fabs(s) < 1.0e-14 ? std::copysign(1.0e14, c) : c / s;
    }
    for (int i = 0; i < lbf::NSCALE_H; ++i) h->scale[i] = 1.0;
    if (p->tile_y != 0 && p->tile_y != 8 && p->tile_y != 16) {
        delete h;
        return fail(LBF_E_ARG, "tile_y must be 0 (autotuned), 8 or 16");
    }
    if (p->tile_y != 0 && !lbf::tile_available(p->storage, p->tile_y)) {
        delete h;
        return fail(LBF_E_UNSUPPORTED, "tile of %d rows not built for this storage", p->tile_y);
    }
    // rows of the tile: the one requested, else 16 (8 in FP64, whose rings of
    // 16 rows do not fit in shared memory); tile_y = 0 also tunes the schedule
    h->tile_y = p->tile_y ? p->tile_y : (lbf::tile_available(p->storage, 16) ? 16 : 8);
    h->tuned = p->tile_y != 0;
    h->launcher = lbf::step_launcher(p->storage, p->lattice, p->highorder, lbf::kernel_tc(*p), lbf::kernel_obs(*p), h->tile_y);
    if (!h->launcher) {
        delete h;
        return fail(LBF_E_UNSUPPORTED, "no kernel for this configuration");
    }
    // > 0: z segments; < 0: columns split at plane -zseg; 0: persistent schedule
    h->zseg = p->zseg > 0 ? std::min(p->zseg, p->lz) : (p->zseg < 0 ? std::max(p->zseg, -p->lz) : 0);
    bool ok = true;
    for (int b = 0; b < 2 && ok; ++b) {
        // 16-bit storage: Pi - u u (6 fields) in 16 bits, P, u, v, w in FP32 (pres)
        ok = ok && cudaMalloc(&h->mom[b], (is_half(h->storage) ? 6 : 10) * h->N * h->esz) == cudaSuccess;
        ok = ok && cudaMalloc(&h->uold[b], 3 * h->N * h->esz) == cudaSuccess;
        if (h->tc) ok = ok && cudaMalloc(&h->phi[b], h->N * h->psz) == cudaSuccess;
        if (is_half(h->storage)) ok = ok && cudaMalloc(&h->pres[b], 4 * h->N * sizeof(float)) == cudaSuccess;
    }
    if (ok && h->obs) ok = cudaMalloc(&h->isf, h->N) == cudaSuccess;
    if (ok) ok = cudaMalloc(&h->d_err, sizeof(int)) == cudaSuccess;
    if (ok) ok = cudaMalloc(&h->d_red, 5 * sizeof(double)) == cudaSuccess;
    if (ok && p->phi_correction) ok = cudaMalloc(&h->d_mass, 4 * sizeof(double)) == cudaSuccess;
    if (p->openbc) h->obc_open = (p->pbc_x ? 0 : 1) | (p->pbc_y ? 0 : 2) | (p->pbc_z ? 0 : 4);
    if (ok && p->repulsive_flux) {
        ok = cudaMalloc(&h->d_rnrm, 3 * h->N * sizeof(double)) == cudaSuccess;
        if (ok) ok = cudaMalloc(&h->d_rep, 3 * h->N * (p->storage == LBF_STORE_F64 ? 8 : 4)) == cudaSuccess;
    }
    if (!ok) {
        cudaGetLastError();
        free_all(h);
        size_t need = lbf::handle_bytes(p);
        delete h;
        return fail(LBF_E_NOMEM, "device allocation of %.3f GB failed", need / 1e9);
    }
    cudaMemset(h->d_err, 0, sizeof(int));
    if (h->obs) cudaMemset(h->isf, 1, h->N);
    if (h->d_mass) cudaMemset(h->d_mass, 0, 4 * sizeof(double));
    *out = h;
    return LBF_OK;
}

int lbf_destroy(lbf_handle* h) {
    if (!h) return fail(LBF_E_ARG, "lbf_destroy: null handle");
    cudaStreamSynchronize(h->stream);
    free_all(h);
    delete h;
    return LBF_OK;
}

int lbf_set_stream(lbf_handle* h, void* s) {
    if (!h) return fail(LBF_E_ARG, "null handle");
    h->stream = static_cast<cudaStream_t>(s);
    return LBF_OK;
}

int lbf_set_isfluid(lbf_handle* h, const int8_t* isf) {
    if (!h || !isf) return fail(LBF_E_ARG, "lbf_set_isfluid: null argument");
    const int nx = h->nx, ny = h->ny, nz = h->nz;
    for (long long i = 0; i < h->N; ++i)
        if (isf[i] != 0 && isf[i] != 1 && isf[i] != -1) return fail(LBF_E_ARG, "isfluid[%lld] = %d not in {1,-1,0}", i, isf[i]);
    if (!h->obs) {
        for (long long i = 0; i < h->N; ++i)
            if (isf[i] != 1) return fail(LBF_E_ARG, "isfluid has non-fluid nodes but obstacles = 0");
        return LBF_OK;
    }
    CUDA_TRY(cudaMemcpyAsync(h->isf, isf, h->N, cudaMemcpyHostToDevice, h->stream));
    h->isf_set = true;
    if (h->p.bounce_back) {
        // BOUNCE_BACK: the nodes whose wall links the half-way bounce-back rewrites
        std::vector<long long> nb;
        const long long plane = (long long)h->nx * h->ny;
        const long long i_lo = h->slab ? lbf::SLAB_HALO * plane : 0;
        const long long i_hi = h->slab ? (lbf::SLAB_HALO + h->nzs) * plane : h->N;
        for (long long i = i_lo; i < i_hi; ++i)
            if (isf[i] == -1) nb.push_back(i);
        cudaFree(h->bb_nodes);
        h->bb_nodes = nullptr;
        h->nbb = (long long)nb.size();
        if (h->nbb) {
            CUDA_TRY(cudaMalloc(&h->bb_nodes, nb.size() * sizeof(long long)));
            CUDA_TRY(cudaMemcpy(h->bb_nodes, nb.data(), nb.size() * sizeof(long long), cudaMemcpyHostToDevice));
        }
    }
    if (!h->tc) return LBF_OK;
    // wetting tables: PHI_int_boundary_kernel steps 1-2 (lb_cuda_boundary_module.f90:281-398),
    // in double; they depend on isfluid only.
    const int pb[3] = {h->p.pbc_x, h->p.pbc_y, h->p.pbc_z};
    const int dims[3] = {nx, ny, nz};
    const int lat = h->p.lattice;
    auto isf_at = [&](int x, int y, int z) -> int {
        int c[3] = {x, y, z};
        for (int d = 0; d < 3; ++d) {
            if (c[d] < 0 || c[d] >= dims[d]) {
                if (!pb[d]) return 1;  // never-written halo keeps isfluid = 1
                c[d] = (c[d] % dims[d] + dims[d]) % dims[d];
            }
        }
        return isf[((long long)c[2] * ny + c[1]) * nx + c[0]];
    };
    std::vector<long long> vs;
    std::vector<int> vd, vf, vsh;
    std::vector<double> vwn;
    // a slab wets the solid nodes of its own planes only (its halo planes are
    // the neighbours', copied with their ghost values), with the donor rules
    // of the whole box: a donor below its first plane is skipped, one beyond
    // its last plane is a wrapped donor
    const int k_lo = h->slab ? lbf::SLAB_HALO : 0, k_hi = h->slab ? lbf::SLAB_HALO + h->nzs : nz;
    for (int k = k_lo; k < k_hi; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                long long c = ((long long)k * ny + j) * nx + i;
                if (isf[c] != 0) continue;
                double wx = 0, wy = 0, wz = 0;
                for (int l = 1; l < 27; ++l) {
                    if (!link_in(lat, l)) continue;
                    int d2 = EXh[l] * EXh[l] + EYh[l] * EYh[l] + EZh[l] * EZh[l];
                    if (isf_at(i + EXh[l], j + EYh[l], k + EZh[l]) == 0) continue;
                    double sc = d2 == 1 ? 1.0 : d2 == 2 ? 0.5 : 1.0 / 3.0;
                    wx += sc * -EXh[l];
                    wy += sc * -EYh[l];
                    wz += sc * -EZh[l];
                }
                double wn = std::sqrt(wx * wx + wy * wy + wz * wz);
                if (wn < 1.0e-14) continue;
                wx /= wn; wy /= wn; wz /= wn;
                double best = -1.0e30;
                int bl = -1;
                for (int l = 1; l < 27; ++l) {
                    if (!link_in(lat, l)) continue;
                    int d2 = EXh[l] * EXh[l] + EYh[l] * EYh[l] + EZh[l] * EZh[l];
                    int f = isf_at(i + EXh[l], j + EYh[l], k + EZh[l]);
                    if (f != 1 && f != -1) continue;
                    double sc = d2 == 1 ? 1.0 : d2 == 2 ? 0.70710678118654752440 : 0.57735026918962576450;
                    double score = (-EXh[l] * wx + -EYh[l] * wy + -EZh[l] * wz) * sc;
                    if (score > best) { best = score; bl = l; }
                }
                if (bl < 0) continue;
                int dc[3] = {i + EXh[bl], j + EYh[bl], k + EZh[bl]};
                // the reference skips a donor on the low halo layer (local index 0)
                const int gz = h->slab ? h->zg0 + dc[2] - lbf::SLAB_HALO : dc[2];
                if (dc[0] == -1 || dc[1] == -1 || gz == -1) continue;
                int flag = lbf::WET_NORMAL;
                for (int d = 0; d < 3; ++d) {
                    if (h->slab && d == 2) {
                        // the donor plane is in the slab's box; the whole box wraps it
                        if (gz >= h->nzg && flag == lbf::WET_NORMAL) flag = lbf::WET_HIGHWRAP;
                        continue;
                    }
                    if (dc[d] >= dims[d]) {
                        if (!pb[d]) flag = lbf::WET_OUTSIDE;
                        else if (flag == lbf::WET_NORMAL) flag = lbf::WET_HIGHWRAP;
                        dc[d] -= dims[d];
                    }
                }
                if (flag == lbf::WET_OUTSIDE) dc[0] = dc[1] = dc[2] = 0;
                vs.push_back(c);
                vd.insert(vd.end(), {dc[0], dc[1], dc[2]});
                vf.push_back(flag);
                vwn.insert(vwn.end(), {wx, wy, wz});
                vsh.insert(vsh.end(), {-EXh[bl], -EYh[bl], -EZh[bl]});
            }
    // open faces: the wall nodes of each face (tangential indices 1 .. n-2)
    // take the phi of their neighbour on the plane next to them after the
    // wetting (boundary_cds_module.f90:1351-1663): entries of the same list
    if (h->obc_open) {
        std::unordered_map<long long, size_t> at;
        for (size_t e = 0; e < vs.size(); ++e) at[vs[e]] = e;
        for (int axis = 0; axis < 3; ++axis) {
            if (!(h->obc_open & (1 << axis))) continue;
            const int a1 = axis == 0 ? 1 : 0, a2 = axis == 2 ? 1 : 2;
            for (int side = 0; side < 2; ++side)
                for (int t2 = 1; t2 <= dims[a2] - 2; ++t2)
                    for (int t1 = 1; t1 <= dims[a1] - 2; ++t1) {
                        int w[3], d[3];
                        w[axis] = side ? dims[axis] - 1 : 0; w[a1] = t1; w[a2] = t2;
                        d[axis] = side ? dims[axis] - 2 : 1; d[a1] = t1; d[a2] = t2;
                        const long long c = ((long long)w[2] * ny + w[1]) * nx + w[0];
                        auto it = at.find(c);
                        size_t e;
                        if (it == at.end()) {
                            e = vs.size();
                            at[c] = e;
                            vs.push_back(c);
                            vd.insert(vd.end(), {0, 0, 0});
                            vf.push_back(0);
                            vwn.insert(vwn.end(), {0.0, 0.0, 0.0});
                            vsh.insert(vsh.end(), {0, 0, 0});
                        } else {
                            e = it->second;
                        }
                        vf[e] = lbf::WET_OPENCOPY;
                        vd[3 * e] = d[0]; vd[3 * e + 1] = d[1]; vd[3 * e + 2] = d[2];
                    }
        }
    }
    cudaFree(h->wet_s); cudaFree(h->wet_donor); cudaFree(h->wet_flag); cudaFree(h->wet_wn); cudaFree(h->wet_shift);
    cudaFree(h->wetW[0]); cudaFree(h->wetW[1]);
    h->wet_s = nullptr; h->wet_donor = nullptr; h->wet_flag = nullptr; h->wet_wn = nullptr; h->wet_shift = nullptr;
    h->wetW[0] = h->wetW[1] = nullptr;
    h->nwet = (int)vs.size();
    h->wet_pending = -1;
    if (h->nwet == 0) return LBF_OK;
    CUDA_TRY(cudaMalloc(&h->wet_s, vs.size() * sizeof(long long)));
    CUDA_TRY(cudaMalloc(&h->wet_donor, vd.size() * sizeof(int)));
    CUDA_TRY(cudaMalloc(&h->wet_flag, vf.size() * sizeof(int)));
    CUDA_TRY(cudaMalloc(&h->wet_wn, vwn.size() * sizeof(double)));
    CUDA_TRY(cudaMalloc(&h->wet_shift, vsh.size() * sizeof(int)));
    CUDA_TRY(cudaMalloc(&h->wetW[0], h->nwet * h->psz));
    CUDA_TRY(cudaMalloc(&h->wetW[1], h->nwet * h->psz));
    CUDA_TRY(cudaMemcpy(h->wet_s, vs.data(), vs.size() * sizeof(long long), cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(h->wet_donor, vd.data(), vd.size() * sizeof(int), cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(h->wet_flag, vf.data(), vf.size() * sizeof(int), cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(h->wet_wn, vwn.data(), vwn.size() * sizeof(double), cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(h->wet_shift, vsh.data(), vsh.size() * sizeof(int), cudaMemcpyHostToDevice));
    return LBF_OK;
}

int lbf_set_fields(lbf_handle* h, const void* mom10, const void* phi, int dtype) {
    if (!h || !mom10) return fail(LBF_E_ARG, "lbf_set_fields: null argument");
    if (dtype != LBF_F32 && dtype != LBF_F64) return fail(LBF_E_ARG, "dtype must be LBF_F32 or LBF_F64");
    if (h->tc && !phi) return fail(LBF_E_ARG, "two-component run needs phi");
    if (h->obs && !h->isf_set) return fail(LBF_E_STATE, "obstacles: call lbf_set_isfluid before lbf_set_fields");
    const size_t hb = dtype == LBF_F64 ? 8 : 4;
    const long long N = h->N;
    const bool half = h->storage == LBF_STORE_F16 || h->storage == LBF_STORE_BF16;
    int rc = LBF_OK;
    if (half) {
        // 16-bit storage keeps Pi - u u (the deviation from equilibrium) and
        // u_old with one power-of-two scale per group of fields; P, u, v, w
        // stay FP32: all ten fields are staged on the device, the group maxima
        // and Pi - u u are computed there
        rc = ensure_staging(h, 10 * N * hb);
        if (rc) return rc;
        CUDA_TRY(cudaMemcpyAsync(h->staging, mom10, 10 * N * hb, cudaMemcpyHostToDevice, h->stream));
        unsigned* d_max = reinterpret_cast<unsigned*>(h->d_red);
        CUDA_TRY(lbf::launch_upload_maxabs(dtype, N, h->staging, d_max, h->stream));
        unsigned bits[2];
        CUDA_TRY(cudaMemcpyAsync(bits, d_max, sizeof bits, cudaMemcpyDeviceToHost, h->stream));
        CUDA_TRY(cudaStreamSynchronize(h->stream));
        float mU, mPi;
        std::memcpy(&mU, &bits[0], sizeof mU);
        std::memcpy(&mPi, &bits[1], sizeof mPi);
        for (int f = 0; f < 4; ++f) h->scale[f] = 1.0;
        // u_old floor 1e-3: a flow that starts at rest keeps 11 significant
        // bits down to ~1e-6 and still represents |u| up to 0.5, beyond any
        // lattice Boltzmann velocity
        for (int f = 1; f <= 3; ++f) h->scale[lbf::NSCALE_H - 4 + f - 1] = pick_scale(h->storage, mU, 1e-3);
        for (int f = 4; f < 10; ++f) h->scale[f] = pick_scale(h->storage, mPi, 1e-4);
        for (int b = 0; b < 2; ++b) {
            for (int f = 0; f < 4; ++f) {
                const char* src = static_cast<const char*>(h->staging) + f * N * hb;
                // FP32 P, u, v, w (the phi conversion converts to FP32 here)
                CUDA_TRY(lbf::launch_convert_in(h->storage, true, src, dtype, h->pres[b] + f * N, N, 1.0, h->stream));
                if (f == 0) continue;
                char* udst = static_cast<char*>(h->uold[b]) + (f - 1) * N * h->esz;
                CUDA_TRY(lbf::launch_convert_in(h->storage, false, src, dtype, udst, N,
                                                h->scale[lbf::NSCALE_H - 4 + f - 1], h->stream));
            }
            for (int c = 0; c < 6; ++c)
                CUDA_TRY(lbf::launch_upload_pin(h->storage, dtype, N, h->staging, c,
                                                static_cast<char*>(h->mom[b]) + c * N * h->esz, h->scale[4 + c],
                                                h->stream));
        }
    } else {
        rc = ensure_staging(h, N * hb);
        if (rc) return rc;
        for (int f = 0; f < 10; ++f) {
            const char* src = static_cast<const char*>(mom10) + f * N * hb;
            CUDA_TRY(cudaMemcpyAsync(h->staging, src, N * hb, cudaMemcpyHostToDevice, h->stream));
            for (int b = 0; b < 2; ++b) {
                char* dst = static_cast<char*>(h->mom[b]) + f * N * h->esz;
                CUDA_TRY(lbf::launch_convert_in(h->storage, false, h->staging, dtype, dst, N, h->scale[f], h->stream));
                if (f >= 1 && f <= 3) {  // u_old of the first step = initial velocity (B := A)
                    char* udst = static_cast<char*>(h->uold[b]) + (f - 1) * N * h->esz;
                    CUDA_TRY(lbf::launch_convert_in(h->storage, false, h->staging, dtype, udst, N,
                                                    h->scale[lbf::NSCALE_H - 4 + f - 1], h->stream));
                }
            }
        }
    }
    if (h->tc) {
        CUDA_TRY(cudaMemcpyAsync(h->staging, phi, N * hb, cudaMemcpyHostToDevice, h->stream));
        for (int b = 0; b < 2; ++b)
            CUDA_TRY(lbf::launch_convert_in(h->storage, true, h->staging, dtype, h->phi[b], N, 1.0, h->stream));
    }
    h->cur = 0;
    h->step = 0;
    h->fields_set = true;
    h->primed = false;
    h->u_valid = false;
    h->wet_pending = -1;
    // the staging copies above are asynchronous with respect to the caller's
    // host buffers: complete them before returning
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return LBF_OK;
}

int lbf_step(lbf_handle* h, int nsteps) {
    if (!h) return fail(LBF_E_ARG, "lbf_step: null handle");
    if (nsteps < 0) return fail(LBF_E_ARG, "nsteps < 0");
    if (!h->fields_set) return fail(LBF_E_STATE, "lbf_step before lbf_set_fields");
    if (!h->primed) {
        int rc = prime(h);
        if (rc) return rc;
    }
    if (!h->tuned && nsteps > 0) {
        int rc = autotune(h);
        if (rc) return rc;
    }
    lbf::StepArgs a;
    for (int s = 0; s < nsteps; ++s) {
        int rc = lbf::handle_pre_step(h);
        if (rc) return rc;
        const bool write_u = h->dr || s == nsteps - 1;
        lbf::handle_step_args(h, a, write_u);
        cudaError_t e = h->launcher(a, h->stream);
        if (e != cudaSuccess) return fail(LBF_E_CUDA, "step kernel launch: %s", cudaGetErrorString(e));
        lbf::handle_advance(h, write_u);
        rc = lbf::handle_post_step(h);
        if (rc) return rc;
    }
    return LBF_OK;
}

int lbf_sync(lbf_handle* h) {
    if (!h) return fail(LBF_E_ARG, "lbf_sync: null handle");
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    CUDA_TRY(cudaGetLastError());
    return LBF_OK;
}

int lbf_get_step(lbf_handle* h, long long* step) {
    if (!h || !step) return fail(LBF_E_ARG, "lbf_get_step: null argument");
    *step = h->step;
    return LBF_OK;
}

int lbf_get_tuning(lbf_handle* h, int* tile_y, int* zseg) {
    if (!h || !tile_y || !zseg) return fail(LBF_E_ARG, "lbf_get_tuning: null argument");
    *tile_y = h->tile_y;
    *zseg = h->zseg;
    return LBF_OK;
}

int lbf_get_fields(lbf_handle* h, void* mom10, void* phi, void* uold, int dtype) {
    if (!h) return fail(LBF_E_ARG, "lbf_get_fields: null handle");
    if (dtype != LBF_F32 && dtype != LBF_F64) return fail(LBF_E_ARG, "dtype must be LBF_F32 or LBF_F64");
    if (!h->fields_set) return fail(LBF_E_STATE, "lbf_get_fields before lbf_set_fields");
    if (!h->primed) {
        int rc = prime(h);
        if (rc) return rc;
    }
    const size_t hb = dtype == LBF_F64 ? 8 : 4;
    const long long N = h->N;
    int rc = ensure_staging(h, N * hb);
    if (rc) return rc;
    auto out_field = [&](const void* src, bool is_phi, double inv, void* dst) -> int {
        CUDA_TRY(lbf::launch_convert_out(h->storage, is_phi, src, h->staging, dtype, N, inv, h->stream));
        CUDA_TRY(cudaMemcpyAsync(dst, h->staging, N * hb, cudaMemcpyDeviceToHost, h->stream));
        CUDA_TRY(cudaStreamSynchronize(h->stream));
        return LBF_OK;
    };
    if (mom10) {
        const bool half = is_half(h->storage);
        double inv[lbf::NSCALE_H];
        for (int f = 0; f < lbf::NSCALE_H; ++f) inv[f] = 1.0 / h->scale[f];
        for (int f = 0; f < 10; ++f) {
            char* dst = static_cast<char*>(mom10) + f * N * hb;
            if (f < 4 && half) {
                rc = out_field(h->pres[h->cur] + f * N, true, 1.0, dst);
            } else if (f >= 4 && half) {
                // stored Pi - u u: the equilibrium part is added back on the device
                CUDA_TRY(lbf::launch_download_pi(h->storage, dtype, N, h->mom[h->cur], h->pres[h->cur] + N, inv,
                                                  f - 4, h->staging, h->stream));
                CUDA_TRY(cudaMemcpyAsync(dst, h->staging, N * hb, cudaMemcpyDeviceToHost, h->stream));
                CUDA_TRY(cudaStreamSynchronize(h->stream));
            } else {
                rc = out_field(static_cast<const char*>(h->mom[h->cur]) + f * N * h->esz, false, inv[f], dst);
            }
            if (rc) return rc;
        }
    }
    if (phi && h->tc) {
        rc = out_field(h->phi[h->cur], true, 1.0, phi);
        if (rc) return rc;
    }
    if (uold) {
        for (int f = 0; f < 3; ++f) {
            char* dst = static_cast<char*>(uold) + f * N * hb;
            if (h->u_valid || h->step == 0) {
                rc = out_field(static_cast<const char*>(h->uold[h->cur]) + f * N * h->esz, false,
                               1.0 / h->scale[lbf::NSCALE_H - 4 + f], dst);
            } else if (is_half(h->storage)) {
                rc = out_field(h->pres[h->cur] + (1 + f) * N, true, 1.0, dst);
            } else {
                rc = out_field(static_cast<const char*>(h->mom[h->cur]) + (1 + f) * N * h->esz, false,
                               1.0 / h->scale[1 + f], dst);
            }
            if (rc) return rc;
        }
    }
    return LBF_OK;
}

int lbf_get_print_fields(lbf_handle* h, float* rho, float* vel, float* press) {
    if (!h) return fail(LBF_E_ARG, "lbf_get_print_fields: null handle");
    if (!h->fields_set) return fail(LBF_E_STATE, "lbf_get_print_fields before lbf_set_fields");
    if (!h->primed) {
        int rc = prime(h);
        if (rc) return rc;
    }
    int rc = flush_wet(h);
    if (rc) return rc;
    const long long N = h->N;
    rc = ensure_staging(h, 5 * N * sizeof(float));
    if (rc) return rc;
    // the copy_print of step n reads the input buffer of step n after the force
    // half-step: P of that buffer, the post-force velocity, phi after wetting
    const int src = h->step == 0 ? h->cur : 1 - h->cur;
    lbf::PrintArgs a;
    a.N = N;
    a.mode = !h->tc ? 0 : ((h->p.printphi || !h->dr) ? 1 : 2);
    a.rho_r = h->p.rho_r;
    a.rho_b = h->p.rho_b;
    a.P = is_half(h->storage) ? static_cast<const void*>(h->pres[src]) : h->mom[src];
    a.sP = 1.0 / h->scale[0];
    a.vel32 = nullptr;
    if (h->step == 0) {
        a.vel = static_cast<const char*>(h->mom[h->cur]) + 1 * N * h->esz;
        if (is_half(h->storage)) a.vel32 = h->pres[h->cur] + N;
        for (int f = 0; f < 3; ++f) a.su[f] = 1.0 / h->scale[1 + f];
    } else {
        if (!h->u_valid) return fail(LBF_E_STATE, "velocity of the last step was not kept");
        a.vel = h->uold[h->cur];
        for (int f = 0; f < 3; ++f) a.su[f] = 1.0 / h->scale[lbf::NSCALE_H - 4 + f];
    }
    a.phi = h->tc ? h->phi[src] : nullptr;
    // after a step, its sums of the input phi are still in d_mass
    a.mass = h->step == 0 ? nullptr : h->d_mass;
    a.isf = h->obs ? h->isf : nullptr;
    float* d = static_cast<float*>(h->staging);
    a.rho = rho ? d : nullptr;
    a.vel_out = vel ? d + N : nullptr;
    a.press = press ? d + 4 * N : nullptr;
    CUDA_TRY(lbf::launch_print(h->storage, a, h->stream));
    if (rho) CUDA_TRY(cudaMemcpyAsync(rho, d, N * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    if (vel) CUDA_TRY(cudaMemcpyAsync(vel, d + N, 3 * N * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    if (press) CUDA_TRY(cudaMemcpyAsync(press, d + 4 * N, N * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return LBF_OK;
}

int lbf_reduce(lbf_handle* h, double out[5]) {
    if (!h || !out) return fail(LBF_E_ARG, "lbf_reduce: null argument");
    if (!h->fields_set) return fail(LBF_E_STATE, "lbf_reduce before lbf_set_fields");
    if (h->slab) return fail(LBF_E_UNSUPPORTED, "lbf_reduce of a slab: sum the slabs' fields (lbf_get_fields)");
    double inv[4];
    for (int f = 0; f < 4; ++f) inv[f] = 1.0 / h->scale[f];
    CUDA_TRY(lbf::launch_reduce(h->storage, h->N, h->mom[h->cur], h->pres[h->cur], h->tc ? h->phi[h->cur] : nullptr,
                                h->obs ? h->isf : nullptr, inv, h->d_red, h->stream));
    CUDA_TRY(cudaMemcpyAsync(out, h->d_red, 5 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    for (int k = 0; k < 5; ++k)
        if (!std::isfinite(out[k]))
            return fail(LBF_E_NUMERIC, "lbf_reduce: the sum of %s over the fluid is not finite at step %lld",
                        k == 0 ? "phi" : k == 1 ? "P" : k == 2 ? "u" : k == 3 ? "v" : "w", h->step);
    return LBF_OK;
}

}  // extern "C"

// ---- z slabs of a larger box ----
// A slab is a handle on planes [z0, z1) of a box periodic in z, with
// SLAB_HALO planes on each side that hold copies of the neighbouring slabs'
// planes.  Its step advances its own planes only; between steps the halos of
// the current time level are refilled from the neighbours -- in one process
// by lbf_slabs_exchange, across processes or GPUs by copying the regions
// lbf_slab_region names (NCCL send/recv, peer copies).  Every node's
// arithmetic is the single box's, so the slabs together give the single
// box's bits.
namespace {
// field f of the current time level (f < nmom: the storage-type moments;
// then the FP32 P, u, v, w of 16-bit storage; then u_old; then phi) and the
// bytes of one of its planes
bool slab_field(lbf_handle* h, int f, char** base, size_t* plane_bytes) {
    const long long plane = (long long)h->nx * h->ny;
    const int nmom = is_half(h->storage) ? 6 : 10, n32 = is_half(h->storage) ? 4 : 0;
    const int c = h->cur;
    if (f < nmom) {
        *base = static_cast<char*>(h->mom[c]) + (size_t)f * h->N * h->esz;
        *plane_bytes = plane * h->esz;
    } else if (f < nmom + n32) {
        *base = reinterpret_cast<char*>(h->pres[c] + (size_t)(f - nmom) * h->N);
        *plane_bytes = plane * sizeof(float);
    } else if (f < nmom + n32 + 3) {
        *base = static_cast<char*>(h->uold[c]) + (size_t)(f - nmom - n32) * h->N * h->esz;
        *plane_bytes = plane * h->esz;
    } else if (f == nmom + n32 + 3 && h->tc) {
        *base = static_cast<char*>(h->phi[c]);
        *plane_bytes = plane * h->psz;
    } else {
        return false;
    }
    return true;
}
int slab_nfields(const lbf_handle* h) { return 13 + (h->tc ? 1 : 0); }
}  // namespace

extern "C" int lbf_slab_region(lbf_handle* h, int side, int recv, int field, void** ptr, size_t* bytes);

namespace {
// check that the slabs form one box's ring and can be exchanged
int check_slabs(lbf_handle* const* slabs, int n, const char* who) {
    if (!slabs || n < 1) return fail(LBF_E_ARG, "%s: no slabs", who);
    for (int i = 0; i < n; ++i) {
        if (!slabs[i] || !slabs[i]->slab) return fail(LBF_E_ARG, "%s: handle %d is not a slab", who, i);
        if (slab_nfields(slabs[i]) != slab_nfields(slabs[0]) || slabs[i]->storage != slabs[0]->storage ||
            slabs[i]->nx != slabs[0]->nx || slabs[i]->ny != slabs[0]->ny)
            return fail(LBF_E_ARG, "%s: slab %d does not match slab 0", who, i);
        if (!slabs[i]->fields_set) return fail(LBF_E_STATE, "%s: slab %d has no fields", who, i);
    }
    return LBF_OK;
}

// copy the halo regions of slab i's current time level from its neighbours, on stream st
int slab_recv(lbf_handle* const* slabs, int n, int i, cudaStream_t st) {
    lbf_handle* lo = slabs[(i + n - 1) % n];
    lbf_handle* hi = slabs[(i + 1) % n];
    for (int f = 0; f < slab_nfields(slabs[i]); ++f) {
        void *dst, *src;
        size_t b, b2;
        lbf_slab_region(slabs[i], 0, 1, f, &dst, &b);
        lbf_slab_region(lo, 1, 0, f, &src, &b2);
        CUDA_TRY(cudaMemcpyAsync(dst, src, b, cudaMemcpyDefault, st));
        lbf_slab_region(slabs[i], 1, 1, f, &dst, &b);
        lbf_slab_region(hi, 0, 0, f, &src, &b2);
        CUDA_TRY(cudaMemcpyAsync(dst, src, b, cudaMemcpyDefault, st));
    }
    return LBF_OK;
}

}  // namespace

extern "C" {

int lbf_create_slab(const lbf_params* global, int z0, int z1, lbf_handle** out) {
    if (!global || !out) return fail(LBF_E_ARG, "lbf_create_slab: null argument");
    *out = nullptr;
    if (!global->pbc_z) return fail(LBF_E_UNSUPPORTED, "lbf_create_slab: the box must be periodic in z");
    if (z0 < 0 || z1 > global->lz || z1 - z0 < lbf::SLAB_HALO)
        return fail(LBF_E_ARG, "lbf_create_slab: planes [%d, %d) of %d: a slab needs %d planes at least", z0, z1,
                    global->lz, lbf::SLAB_HALO);
    if (global->phi_correction || global->repulsive_flux || global->openbc)
        return fail(LBF_E_UNSUPPORTED,
                    "lbf_create_slab: phi_correction, repulsive_flux and openbc need box-wide data (not for slabs)");
    lbf_params p = *global;
    p.lz = (z1 - z0) + 2 * lbf::SLAB_HALO;
    p.pbc_z = 0;  // the halo planes are real planes of the slab's box
    int rc = lbf_create(&p, out);
    if (rc) return rc;
    lbf_handle* h = *out;
    h->slab = true;
    h->zg0 = z0;
    h->nzs = z1 - z0;
    h->nzg = global->lz;
    cudaGetDevice(&h->device);
    return LBF_OK;
}

int lbf_slab_nregions(lbf_handle* h, int* n) {
    if (!h || !n) return fail(LBF_E_ARG, "lbf_slab_nregions: null argument");
    if (!h->slab) return fail(LBF_E_ARG, "lbf_slab_nregions: not a slab");
    *n = slab_nfields(h);
    return LBF_OK;
}

int lbf_slab_region(lbf_handle* h, int side, int recv, int field, void** ptr, size_t* bytes) {
    if (!h || !ptr || !bytes) return fail(LBF_E_ARG, "lbf_slab_region: null argument");
    if (!h->slab) return fail(LBF_E_ARG, "lbf_slab_region: not a slab");
    if (side < 0 || side > 1 || field < 0 || field >= slab_nfields(h))
        return fail(LBF_E_ARG, "lbf_slab_region: side %d / field %d out of range", side, field);
    char* base;
    size_t pb;
    slab_field(h, field, &base, &pb);
    const int H = lbf::SLAB_HALO;
    // low side: send the first H own planes, receive into planes 0 .. H-1;
    // high side: send the last H own planes, receive into the H planes after them
    const int first = side == 0 ? (recv ? 0 : H) : (recv ? H + h->nzs : h->nzs);
    *ptr = base + (size_t)first * pb;
    *bytes = (size_t)H * pb;
    return LBF_OK;
}

int lbf_slabs_exchange(lbf_handle* const* slabs, int n) {
    if (!slabs || n < 1) return fail(LBF_E_ARG, "lbf_slabs_exchange: no slabs");
    for (int i = 0; i < n; ++i) {
        if (!slabs[i] || !slabs[i]->slab) return fail(LBF_E_ARG, "lbf_slabs_exchange: handle %d is not a slab", i);
        if (slab_nfields(slabs[i]) != slab_nfields(slabs[0]) || slabs[i]->storage != slabs[0]->storage ||
            slabs[i]->nx != slabs[0]->nx || slabs[i]->ny != slabs[0]->ny)
            return fail(LBF_E_ARG, "lbf_slabs_exchange: slab %d does not match slab 0", i);
    }
    // every slab's step must be complete before its planes are copied
    for (int i = 0; i < n; ++i) CUDA_TRY(cudaStreamSynchronize(slabs[i]->stream));
    for (int i = 0; i < n; ++i) {
        int rc = slab_recv(slabs, n, i, slabs[i]->stream);
        if (rc) return rc;
    }
    for (int i = 0; i < n; ++i) CUDA_TRY(cudaStreamSynchronize(slabs[i]->stream));
    return LBF_OK;
}

int lbf_slabs_step(lbf_handle* const* slabs, int n, int nsteps) {
    int rc = check_slabs(slabs, n, "lbf_slabs_step");
    if (rc) return rc;
    if (nsteps < 0) return fail(LBF_E_ARG, "lbf_slabs_step: nsteps < 0");
    int dev0 = 0;
    CUDA_TRY(cudaGetDevice(&dev0));
    // the pre-loop wetting of every slab, then the halos of the first input
    bool fresh = false;
    for (int i = 0; i < n && !rc; ++i) {
        lbf_handle* h = slabs[i];
        CUDA_TRY(cudaSetDevice(h->device));
        if (!h->primed) {
            rc = prime(h);
            fresh = true;
        }
        if (!rc && !h->tuned && nsteps > 0) rc = autotune(h);
        if (!rc && !h->xstream) {
            cudaError_t e = cudaStreamCreateWithFlags(&h->xstream, cudaStreamNonBlocking);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->ev_done, cudaEventDisableTiming);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->ev_copied, cudaEventDisableTiming);
            if (e != cudaSuccess) rc = fail(LBF_E_CUDA, "lbf_slabs_step: %s", cudaGetErrorString(e));
        }
    }
    if (!rc && fresh) rc = lbf_slabs_exchange(slabs, n);
    const int H = lbf::SLAB_HALO;
    for (int s = 0; s < nsteps && !rc; ++s) {
        // every slab's previous step is done before its planes are sent
        for (int i = 0; i < n && !rc; ++i) {
            cudaSetDevice(slabs[i]->device);
            if (cudaEventRecord(slabs[i]->ev_done, slabs[i]->stream) != cudaSuccess)
                rc = fail(LBF_E_CUDA, "lbf_slabs_step: event record failed");
        }
        for (int i = 0; i < n && !rc; ++i) {
            lbf_handle* h = slabs[i];
            cudaSetDevice(h->device);
            const bool write_u = h->dr || s == nsteps - 1;
            lbf::StepArgs a;
            lbf::handle_step_args(h, a, write_u);
            // the planes whose stencils stay clear of the halos (4 planes
            // from each face: phi of the collision's theta neighbours) run
            // while the halos of this step's input arrive
            const int in_lo = H + 4, in_hi = H + h->nzs - 4;
            if (in_hi > in_lo) {
                a.zlo = in_lo;
                a.zhi = in_hi;
                cudaError_t e = h->launcher(a, h->stream);
                if (e != cudaSuccess) { rc = fail(LBF_E_CUDA, "slab step: %s", cudaGetErrorString(e)); break; }
            }
            for (int j : {(i + n - 1) % n, (i + 1) % n, i})
                if (cudaStreamWaitEvent(h->xstream, slabs[j]->ev_done, 0) != cudaSuccess)
                    rc = fail(LBF_E_CUDA, "lbf_slabs_step: stream wait failed");
            if (!rc) rc = slab_recv(slabs, n, i, h->xstream);
            if (!rc && cudaEventRecord(h->ev_copied, h->xstream) != cudaSuccess)
                rc = fail(LBF_E_CUDA, "lbf_slabs_step: event record failed");
            if (!rc && cudaStreamWaitEvent(h->stream, h->ev_copied, 0) != cudaSuccess)
                rc = fail(LBF_E_CUDA, "lbf_slabs_step: stream wait failed");
            // the per-step work that reads the halos (wetting), then the planes next to them
            if (!rc) rc = lbf::handle_pre_step(h);
            if (rc) break;
            const int ranges[2][2] = {{H, in_hi > in_lo ? in_lo : H + h->nzs}, {in_hi > in_lo ? in_hi : H + h->nzs, H + h->nzs}};
            for (const auto& r : ranges) {
                if (r[1] <= r[0]) continue;
                a.zlo = r[0];
                a.zhi = r[1];
                cudaError_t e = h->launcher(a, h->stream);
                if (e != cudaSuccess) { rc = fail(LBF_E_CUDA, "slab step: %s", cudaGetErrorString(e)); break; }
            }
        }
        // all slabs advance together: a slab's next send reads the planes this step wrote
        for (int i = 0; i < n && !rc; ++i) {
            lbf_handle* h = slabs[i];
            cudaSetDevice(h->device);
            lbf::handle_advance(h, h->dr || s == nsteps - 1);
            rc = lbf::handle_post_step(h);
        }
    }
    // the halos of the new time level, for lbf_get_fields and the next call
    if (!rc) rc = lbf_slabs_exchange(slabs, n);
    cudaSetDevice(dev0);
    return rc;
}

}  // extern "C"

// ---- full-state checkpoint ----
// Every stored field of both time levels in the storage precision (moments,
// the FP32 P, u, v, w of 16-bit storage, u_old, phi), the wetting ghost
// values still waiting to be written, the mass-correction sums, the
// per-field scales, the step count and the time-level index: a run resumed
// from it continues bit for bit.  The file starts with a header that the
// reader checks against the handle (box, storage, lattice and switches).
namespace {
constexpr char kCkptMagic[8] = {'L', 'B', 'F', 'C', 'K', 'P', 'T', '1'};
struct CkptHeader {
    char magic[8];
    int32_t version, lx, ly, lz, storage, lattice, highorder, twocomponent, densratio, obstacles;
    int32_t phi_correction, repulsive_flux, nwet, cur, primed, u_valid, wet_pending, wet_pending_target;
    int64_t step;
    double scale[lbf::NSCALE_H];
};

// the device regions of a handle that hold state, with their byte counts
std::vector<std::pair<void*, size_t>> state_regions(lbf_handle* h) {
    std::vector<std::pair<void*, size_t>> r;
    const size_t N = (size_t)h->N;
    const bool half = is_half(h->storage);
    for (int b = 0; b < 2; ++b) {
        r.emplace_back(h->mom[b], (half ? 6 : 10) * N * h->esz);
        r.emplace_back(h->uold[b], 3 * N * h->esz);
        if (h->tc) r.emplace_back(h->phi[b], N * h->psz);
        if (half) r.emplace_back(h->pres[b], 4 * N * sizeof(float));
        if (h->nwet > 0) r.emplace_back(h->wetW[b], (size_t)h->nwet * h->psz);
    }
    if (h->d_mass) r.emplace_back(h->d_mass, 4 * sizeof(double));
    return r;
}

constexpr size_t kCkptChunk = size_t(64) << 20;
}  // namespace

extern "C" {

int lbf_write_checkpoint(lbf_handle* h, const char* path) {
    if (!h || !path) return fail(LBF_E_ARG, "lbf_write_checkpoint: null argument");
    if (!h->fields_set) return fail(LBF_E_STATE, "lbf_write_checkpoint before lbf_set_fields");
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    CkptHeader hd;
    std::memset(&hd, 0, sizeof hd);
    std::memcpy(hd.magic, kCkptMagic, 8);
    hd.version = 1;
    hd.lx = h->nx; hd.ly = h->ny; hd.lz = h->nz;
    hd.storage = h->storage; hd.lattice = h->p.lattice; hd.highorder = h->p.highorder;
    hd.twocomponent = h->p.twocomponent; hd.densratio = h->p.densratio; hd.obstacles = h->p.obstacles;
    hd.phi_correction = h->p.phi_correction; hd.repulsive_flux = h->p.repulsive_flux; hd.nwet = h->nwet;
    hd.cur = h->cur; hd.primed = h->primed; hd.u_valid = h->u_valid;
    hd.wet_pending = h->wet_pending; hd.wet_pending_target = h->wet_pending_target;
    hd.step = h->step;
    for (int i = 0; i < lbf::NSCALE_H; ++i) hd.scale[i] = h->scale[i];
    std::FILE* f = std::fopen(path, "wb");
    if (!f) return fail(LBF_E_IO, "lbf_write_checkpoint: cannot open %s", path);
    bool ok = std::fwrite(&hd, sizeof hd, 1, f) == 1;
    std::vector<char> buf;
    cudaError_t e = cudaSuccess;
    for (const auto& reg : state_regions(h)) {
        for (size_t off = 0; ok && off < reg.second; off += kCkptChunk) {
            const size_t n = std::min(kCkptChunk, reg.second - off);
            buf.resize(n);
            e = cudaMemcpy(buf.data(), static_cast<const char*>(reg.first) + off, n, cudaMemcpyDeviceToHost);
            ok = e == cudaSuccess && std::fwrite(buf.data(), 1, n, f) == n;
        }
    }
    if (std::fclose(f) != 0) ok = false;
    if (e != cudaSuccess) return fail(LBF_E_CUDA, "lbf_write_checkpoint: %s", cudaGetErrorString(e));
    return ok ? LBF_OK : fail(LBF_E_IO, "lbf_write_checkpoint: write to %s failed", path);
}

int lbf_read_checkpoint(lbf_handle* h, const char* path) {
    if (!h || !path) return fail(LBF_E_ARG, "lbf_read_checkpoint: null argument");
    if (h->obs && !h->isf_set) return fail(LBF_E_STATE, "obstacles: call lbf_set_isfluid before lbf_read_checkpoint");
    std::FILE* f = std::fopen(path, "rb");
    if (!f) return fail(LBF_E_IO, "lbf_read_checkpoint: cannot open %s", path);
    CkptHeader hd;
    bool ok = std::fread(&hd, sizeof hd, 1, f) == 1 && std::memcmp(hd.magic, kCkptMagic, 8) == 0 && hd.version == 1;
    if (!ok) {
        std::fclose(f);
        return fail(LBF_E_IO, "lbf_read_checkpoint: %s is not a checkpoint of this library", path);
    }
    if (hd.lx != h->nx || hd.ly != h->ny || hd.lz != h->nz || hd.storage != h->storage ||
        hd.lattice != h->p.lattice || hd.highorder != h->p.highorder || hd.twocomponent != h->p.twocomponent ||
        hd.densratio != h->p.densratio || hd.obstacles != h->p.obstacles ||
        hd.phi_correction != h->p.phi_correction || hd.repulsive_flux != h->p.repulsive_flux || hd.nwet != h->nwet) {
        std::fclose(f);
        return fail(LBF_E_ARG, "lbf_read_checkpoint: %s was written for another box, storage or configuration", path);
    }
    std::vector<char> buf;
    cudaError_t e = cudaSuccess;
    for (const auto& reg : state_regions(h)) {
        for (size_t off = 0; ok && off < reg.second; off += kCkptChunk) {
            const size_t n = std::min(kCkptChunk, reg.second - off);
            buf.resize(n);
            ok = std::fread(buf.data(), 1, n, f) == n;
            if (ok) e = cudaMemcpy(static_cast<char*>(reg.first) + off, buf.data(), n, cudaMemcpyHostToDevice);
            ok = ok && e == cudaSuccess;
        }
    }
    if (ok) ok = std::fgetc(f) == EOF;  // nothing after the state
    std::fclose(f);
    if (e != cudaSuccess) return fail(LBF_E_CUDA, "lbf_read_checkpoint: %s", cudaGetErrorString(e));
    if (!ok) return fail(LBF_E_IO, "lbf_read_checkpoint: %s is truncated or too long", path);
    h->cur = hd.cur;
    h->primed = hd.primed != 0;
    h->u_valid = hd.u_valid != 0;
    h->wet_pending = hd.wet_pending;
    h->wet_pending_target = hd.wet_pending_target;
    h->step = hd.step;
    for (int i = 0; i < lbf::NSCALE_H; ++i) h->scale[i] = hd.scale[i];
    h->fields_set = true;
    return LBF_OK;
}

}  // extern "C"

namespace lbf {

int handle_prime(lbf_handle* h) { return h->primed ? LBF_OK : prime(h); }

void handle_step_args(const lbf_handle* h, StepArgs& a, bool write_u) {
    const int in = h->cur, out = 1 - h->cur;
    a.nx = h->nx; a.ny = h->ny; a.nz = h->nz;
    a.pbx = h->p.pbc_x; a.pby = h->p.pbc_y; a.pbz = h->p.pbc_z;
    a.densratio = h->dr; a.obstacles = h->obs; a.zseg = h->zseg; a.smag = h->p.smagorinsky;
    a.zlo = h->slab ? lbf::SLAB_HALO : 0;
    a.zhi = h->slab ? lbf::SLAB_HALO + h->nzs : h->nz;
    a.omega = h->omega; a.visc1 = h->p.visc1; a.visc2 = h->p.visc2;
    a.rho_r = h->tc ? h->p.rho_r : 1.0; a.rho_b = h->tc ? h->p.rho_b : 1.0;
    a.beta = h->beta; a.kapp = h->kapp; a.sharp_c = h->sharp_c; a.tau_diff = h->p.tau_diff;
    a.fx = h->p.fx; a.fy = h->p.fy; a.fz = h->p.fz;
    for (int i = 0; i < NSCALE_H; ++i) a.scale[i] = h->scale[i];
    a.isf = h->obs ? h->isf : nullptr;
    a.err = h->d_err;
    a.rep = h->d_rep;
    a.mass = h->d_mass;
    a.min = h->mom[in];
    a.mout = h->mom[out];
    a.uin = h->uold[in];
    a.uout = h->uold[out];
    a.pin = h->phi[in];
    a.pout = h->phi[out];
    a.pres_in = h->pres[in];
    a.pres_out = h->pres[out];
    a.write_u = write_u ? 1 : 0;
}

void handle_advance(lbf_handle* h, bool wrote_u) {
    h->cur = 1 - h->cur;
    h->step++;
    h->u_valid = wrote_u;
}

size_t handle_bytes(const lbf_params* p) {
    const long long N = (long long)p->lx * p->ly * p->lz;
    const size_t esz = storage_bytes(p->storage), psz = phi_bytes(p->storage);
    const bool half = p->storage == LBF_STORE_F16 || p->storage == LBF_STORE_BF16;
    // per time level: the moments (16-bit storage: Pi - u u in 16 bits, P, u,
    // v, w in FP32) and u_old
    size_t b = half ? 2 * (9 * N * esz + 4 * N * sizeof(float)) : 2 * (13 * N * esz);
    if (p->twocomponent) b += 2 * N * psz;
    if (p->obstacles) b += N;
    if (p->phi_correction) b += 4 * sizeof(double);
    if (p->repulsive_flux) b += 3 * N * (sizeof(double) + (p->storage == LBF_STORE_F64 ? 8 : 4));
    return b;
}

int handle_pre_step(lbf_handle* h) {
    int rc = launch_wet(h, h->cur, 1 - h->cur, false);
    if (rc) return rc;
    if (h->d_mass) {
        // phi mass correction of this step's input phi (bcs_mesoscopic_phifields,
        // integrator_module.f90:297): its sum and interface count, and the phi
        // the input state carries through open faces; the step's kernels apply
        // the correction where they read a node's phi
        CUDA_TRY(launch_face_flux(h, h->cur));
        CUDA_TRY(lbf::launch_mass(h->storage, lbf::MASS_SUM, h->N, h->phi[h->cur], h->obs ? h->isf : nullptr,
                                  h->d_mass, h->stream));
    }
    if (!h->d_rep) return LBF_OK;
    // REPULSIVE_FLUX force of this step from its input phi (integrator_module.f90:325-328)
    lbf::RepulsiveArgs a;
    a.nx = h->nx; a.ny = h->ny; a.nz = h->nz;
    a.pbx = h->p.pbc_x; a.pby = h->p.pbc_y; a.pbz = h->p.pbc_z;
    a.width = h->p.width; a.a_rep = h->p.a_rep; a.cos_opp_t = h->p.cos_opp_t; a.q_th = h->p.q_th;
    a.isf = h->obs ? h->isf : nullptr;
    a.phi = h->phi[h->cur];
    a.nrm = h->d_rnrm;
    a.force = h->d_rep;
    a.mass = h->d_mass;
    CUDA_TRY(lbf::launch_repulsive(h->storage, a, h->stream));
    return LBF_OK;
}

int handle_post_step(lbf_handle* h) {
    // wall passes on the step's output moments (buffer cur after the advance),
    // from the step's input buffers (1 - cur), which the step left intact:
    // BOUNCE_BACK, then the open faces (bcs_mesoscopic_hfields after the fused kernel)
    if (h->obc_open || h->nbb) {
        const int in = 1 - h->cur;
        lbf::BoundaryArgs a;
        a.smag = h->p.smagorinsky;
        a.rep = h->d_rep;
        a.nodes = h->bb_nodes;
        a.nnodes = h->nbb;
        a.axis = a.side = a.type = 0;
        a.press = 0.0;
        a.vel[0] = a.vel[1] = a.vel[2] = 0.0;
        a.nx = h->nx; a.ny = h->ny; a.nz = h->nz;
        a.pbx = h->p.pbc_x; a.pby = h->p.pbc_y; a.pbz = h->p.pbc_z;
        a.lattice = h->p.lattice; a.highorder = h->p.highorder; a.tc = h->tc; a.dr = h->dr;
        a.omega = h->omega; a.visc1 = h->p.visc1; a.visc2 = h->p.visc2;
        a.rho_r = h->tc ? h->p.rho_r : 1.0; a.rho_b = h->tc ? h->p.rho_b : 1.0;
        a.beta = h->beta; a.kapp = h->kapp; a.sharp_c = h->sharp_c; a.tau_diff = h->p.tau_diff;
        a.fx = h->p.fx; a.fy = h->p.fy; a.fz = h->p.fz;
        a.isf = h->isf;
        a.min = h->mom[in]; a.pres_in = h->pres[in]; a.uin = h->uold[in];
        a.phi = h->tc ? h->phi[in] : nullptr;
        a.mom = h->mom[h->cur]; a.pres = h->pres[h->cur];
        for (int f = 0; f < lbf::NSCALE_H; ++f) a.scale[f] = h->scale[f];
        a.mass = h->d_mass;
        if (h->nbb) CUDA_TRY(lbf::launch_bounce_back(h->storage, a, h->stream));
        for (int axis = 0; axis < 3; ++axis) {
            if (!(h->obc_open & (1 << axis))) continue;
            for (int side = 0; side < 2; ++side) {
                a.axis = axis; a.side = side;
                a.type = h->p.openbc_type[axis][side];
                a.press = h->p.openbc_press[axis][side];
                for (int d = 0; d < 3; ++d) a.vel[d] = h->p.openbc_vel[axis][side][d];
                CUDA_TRY(lbf::launch_open_face(h->storage, a, h->stream));
            }
        }
    }
    return LBF_OK;
}

bool handle_steady(const lbf_handle* h) { return !(h->tc && h->obs && h->nwet > 0) || h->wet_pending >= 0; }

void handle_release_staging(lbf_handle* h) {
    if (!h->staging) return;
    cudaFree(h->staging);
    h->staging = nullptr;
    h->staging_bytes = 0;
}

}  // namespace lbf
