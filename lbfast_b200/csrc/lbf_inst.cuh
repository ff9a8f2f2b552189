// lbf_inst.cuh -- launch wrappers of the fused step kernel; included once per
// storage type by lbf_inst_<storage>.cu so the instantiations compile in
// parallel.
#pragma once
#include "lbf_internal.h"
#include "lbf_stream_kernel.cuh"

namespace lbf {

template <int LAT, bool HO, bool TC, typename S, typename R>
cudaError_t launch_stream(const StepArgs& a, cudaStream_t st) {
    using SP = typename PhiStore<S>::type;
    static bool attr_set = false;
    const size_t smem = stream_smem_bytes_v2<LAT, TC, S, R>();
    if (!attr_set) {
        cudaError_t e = cudaFuncSetAttribute(stream_kernel<LAT, HO, TC, S, R>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        attr_set = true;
    }
    StepParams<S, R> p;
    p.nx = a.nx; p.ny = a.ny; p.nz = a.nz;
    p.pbx = a.pbx; p.pby = a.pby; p.pbz = a.pbz;
    p.plane = (long long)a.nx * a.ny;
    p.N = p.plane * a.nz;
    p.densratio = a.densratio; p.obstacles = a.obstacles; p.write_u = a.write_u;
    p.zseg = a.zseg;
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
    dim3 grid((a.nx + TX - 1) / TX, (a.ny + TY - 1) / TY, (a.nz + a.zseg - 1) / a.zseg);
    stream_kernel<LAT, HO, TC, S, R><<<grid, NT, smem, st>>>(p);
    return cudaGetLastError();
}

template <typename S, typename R> StepLauncher step_table(int lat, int ho, int tc) {
    if (lat == 19) return tc ? &launch_stream<19, false, true, S, R> : &launch_stream<19, false, false, S, R>;
    if (lat != 27) return nullptr;
    if (ho) return tc ? &launch_stream<27, true, true, S, R> : &launch_stream<27, true, false, S, R>;
    return tc ? &launch_stream<27, false, true, S, R> : &launch_stream<27, false, false, S, R>;
}

}  // namespace lbf
