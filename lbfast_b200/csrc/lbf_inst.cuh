// lbf_inst.cuh -- launch wrappers of the fused step kernel; included once per
// storage type by lbf_inst_<storage>.cu so the instantiations compile in
// parallel.
#pragma once
#include "lbf_internal.h"
#include "lbf_stream_kernel.cuh"

#include <algorithm>

namespace lbf {

static_assert(TX == STEP_TILE_X, "host tile width must match the kernel's");

template <typename S, typename R> void make_params(const StepArgs& a, StepParams<S, R>& p) {
    using SP = typename PhiStore<S>::type;
    p.nx = a.nx; p.ny = a.ny; p.nz = a.nz;
    p.pbx = a.pbx; p.pby = a.pby; p.pbz = a.pbz;
    p.plane = (long long)a.nx * a.ny;
    p.N = p.plane * a.nz;
    p.densratio = a.densratio; p.obstacles = a.obstacles; p.write_u = a.write_u; p.smag = a.smag;
    p.zseg = a.zseg;
    p.zlo = a.zlo;
    p.zhi = a.zhi;
    p.omega = (R)a.omega; p.visc1 = (R)a.visc1; p.visc2 = (R)a.visc2;
    p.rho_r = (R)a.rho_r; p.rho_b = (R)a.rho_b; p.beta = (R)a.beta; p.kapp = (R)a.kapp;
    p.sharp_c = (R)a.sharp_c; p.tau_diff = (R)a.tau_diff;
    p.fx = (R)a.fx; p.fy = (R)a.fy; p.fz = (R)a.fz;
    for (int i = 0; i < NSCALE; ++i) {
        p.scale[i] = (R)a.scale[i];
        p.inv_scale[i] = (R)(1.0 / a.scale[i]);
    }
    p.min = static_cast<const S*>(a.min);
    p.mout = static_cast<S*>(a.mout);
    p.uin = static_cast<const S*>(a.uin);
    p.uout = static_cast<S*>(a.uout);
    p.pin = static_cast<const SP*>(a.pin);
    p.pout = static_cast<SP*>(a.pout);
    p.pres_in = a.pres_in;
    p.pres_out = a.pres_out;
    p.isf = a.isf;
    p.err = a.err;
    p.rep = static_cast<const R*>(a.rep);
    p.mass = a.mass;
}

template <int LAT, bool HO, bool TC, typename S, typename R, int TYV, bool REP = false, bool OBS = true>
cudaError_t launch_stream(const StepArgs& a, cudaStream_t st) {
    static bool attr_set = false;
    const size_t smem = stream_smem_bytes<LAT, TC, S, R, TYV>();
    if (!attr_set) {
        cudaError_t e = cudaFuncSetAttribute(stream_kernel<LAT, HO, TC, S, R, TYV, REP, OBS>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        attr_set = true;
    }
    StepParams<S, R> p;
    make_params(a, p);
    const int nzr = a.zhi - a.zlo;
    if (nzr <= 0) return cudaSuccess;
    if (a.zseg < 0) {
        // split columns: a head and a tail segment per column
        const long long ncols = (long long)((a.nx + TX - 1) / TX) * ((a.ny + TYV - 1) / TYV);
        stream_kernel<LAT, HO, TC, S, R, TYV, REP, OBS><<<(unsigned)(2 * ncols), TX * TYV, smem, st>>>(p);
        return cudaGetLastError();
    }
    if (a.zseg > 0) {
        dim3 grid((a.nx + TX - 1) / TX, (a.ny + TYV - 1) / TYV, (nzr + a.zseg - 1) / a.zseg);
        stream_kernel<LAT, HO, TC, S, R, TYV, REP, OBS><<<grid, TX * TYV, smem, st>>>(p);
        return cudaGetLastError();
    }
    static int resident = 0;  // CTAs per SM at this shared-memory size
    if (!resident) {
        cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, stream_kernel<LAT, HO, TC, S, R, TYV, REP, OBS>,
                                                                      TX * TYV, smem);
        if (e != cudaSuccess) return e;
        if (resident < 1) return cudaErrorInvalidConfiguration;
    }
    const long long W = (long long)((a.nx + TX - 1) / TX) * ((a.ny + TYV - 1) / TYV) * nzr;
    const int grid = persistent_grid(W, resident);
    stream_kernel<LAT, HO, TC, S, R, TYV, REP, OBS><<<grid, TX * TYV, smem, st>>>(p);
    return cudaGetLastError();
}

// One launch advancing many boxes of one kernel class: d_boxes holds one
// StepParams per box, d_work one (box, first column-plane, end column-plane)
// per CTA.
template <int LAT, bool HO, bool TC, typename S, typename R, int TYV, bool REP = false, bool OBS = true>
cudaError_t launch_stream_batched(const void* d_boxes, const int4* d_work, int nwork, cudaStream_t st) {
    static bool attr_set = false;
    const size_t smem = stream_smem_bytes<LAT, TC, S, R, TYV>();
    if (!attr_set) {
        cudaError_t e = cudaFuncSetAttribute(stream_kernel_batched<LAT, HO, TC, S, R, TYV, REP, OBS>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        attr_set = true;
    }
    if (nwork <= 0) return cudaSuccess;
    stream_kernel_batched<LAT, HO, TC, S, R, TYV, REP, OBS>
        <<<nwork, TX * TYV, smem, st>>>(static_cast<const StepParams<S, R>*>(d_boxes), d_work);
    return cudaGetLastError();
}

template <int LAT, bool HO, bool TC, typename S, typename R, int TYV, bool REP = false, bool OBS = true> int batched_resident() {
    static int resident = 0;
    if (!resident) {
        const size_t smem = stream_smem_bytes<LAT, TC, S, R, TYV>();
        if (cudaFuncSetAttribute(stream_kernel_batched<LAT, HO, TC, S, R, TYV, REP, OBS>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, stream_kernel_batched<LAT, HO, TC, S, R, TYV, REP, OBS>,
                                                          TX * TYV, smem) != cudaSuccess)
            resident = 1;
        resident = std::max(resident, 1);
    }
    return resident;
}

template <typename S, typename R> void fill_params(const StepArgs& a, void* dst) {
    make_params(a, *static_cast<StepParams<S, R>*>(dst));
}

// the kernel classes of one storage type and tile height; tc: 0 one
// component, 1 two components, 2 two components with REPULSIVE_FLUX; obs:
// obstacles
template <int LAT, bool HO, typename S, typename R, int TYV, bool OBS> StepLauncher step_class(int tc) {
    return tc == 2 ? &launch_stream<LAT, HO, true, S, R, TYV, true, OBS>
                   : tc ? &launch_stream<LAT, HO, true, S, R, TYV, false, OBS>
                        : &launch_stream<LAT, HO, false, S, R, TYV, false, OBS>;
}
template <int LAT, bool HO, typename S, typename R, int TYV> StepLauncher step_class(int tc, int obs) {
    return obs ? step_class<LAT, HO, S, R, TYV, true>(tc) : step_class<LAT, HO, S, R, TYV, false>(tc);
}
template <typename S, typename R, int TYV> StepLauncher step_table(int lat, int ho, int tc, int obs) {
    if (lat == 15 && !ho) return step_class<15, false, S, R, TYV>(tc, obs);
    if (lat == 19 && !ho) return step_class<19, false, S, R, TYV>(tc, obs);
    if (lat == 27 && ho) return step_class<27, true, S, R, TYV>(tc, obs);
    if (lat == 27 && !ho) return step_class<27, false, S, R, TYV>(tc, obs);
    return nullptr;
}

template <int LAT, bool HO, typename S, typename R, int TYV, bool OBS> void batch_class(int tc, BatchOps& o) {
    if (tc == 2) {
        o.launch = &launch_stream_batched<LAT, HO, true, S, R, TYV, true, OBS>;
        o.resident = &batched_resident<LAT, HO, true, S, R, TYV, true, OBS>;
    } else if (tc) {
        o.launch = &launch_stream_batched<LAT, HO, true, S, R, TYV, false, OBS>;
        o.resident = &batched_resident<LAT, HO, true, S, R, TYV, false, OBS>;
    } else {
        o.launch = &launch_stream_batched<LAT, HO, false, S, R, TYV, false, OBS>;
        o.resident = &batched_resident<LAT, HO, false, S, R, TYV, false, OBS>;
    }
}
// The batched kernels keep obstacles a run-time flag (OBS = true for every
// box): the obstacle-free compilation of the batched kernel, unlike the
// single-box one, ran the droplet-ensemble server slower and erratically
// (3.2-5.2 against a steady 5.5 solves/s, interleaved runs on one box).
template <int LAT, bool HO, typename S, typename R, int TYV> void batch_class(int tc, int, BatchOps& o) {
    batch_class<LAT, HO, S, R, TYV, true>(tc, o);
}
template <typename S, typename R, int TYV> BatchOps batch_table(int lat, int ho, int tc, int obs) {
    BatchOps o;
    o.params_bytes = sizeof(StepParams<S, R>);
    o.fill = &fill_params<S, R>;
    o.tile_y = TYV;
    o.launch = nullptr;
    o.resident = nullptr;
    if (lat == 15 && !ho) batch_class<15, false, S, R, TYV>(tc, obs, o);
    if (lat == 19 && !ho) batch_class<19, false, S, R, TYV>(tc, obs, o);
    if (lat == 27 && ho) batch_class<27, true, S, R, TYV>(tc, obs, o);
    if (lat == 27 && !ho) batch_class<27, false, S, R, TYV>(tc, obs, o);
    return o;
}

// instantiation unit of one storage type and tile height (lbf_inst_<storage>_t<rows>.cu)
#define LBF_INSTANTIATE(NAME, S, R, TYV)                                                                  \
    StepLauncher step_launcher_##NAME##_t##TYV(int lat, int ho, int tc, int obs) {                        \
        return step_table<S, R, TYV>(lat, ho, tc, obs);                                                   \
    }                                                                                                     \
    BatchOps batch_ops_##NAME##_t##TYV(int lat, int ho, int tc, int obs) { return batch_table<S, R, TYV>(lat, ho, tc, obs); }

}  // namespace lbf
