// lbf_lattice.cuh -- lattice constants and per-node arithmetic of the LBFAST
// time step, written for the fused sm_100a kernel.
//
// Link order, weights and opposites follow the reference's tables
// (vars_module.f90:319-338 for D3Q27, :666-684 for D3Q19), so that
// populations, isfluid neighbour tests and bounce-back pairings line up with
// the reference's.
//
// The post-collision population of the reference's fused kernel
// (lb_cuda_fused_module.f90:637-713) is a Hermite expansion:
//     f*_l = sum_r Minv_mrt(r,l) m*_r,   Minv_mrt(r,l) = w_l H_r(c_l) / <H_r,H_r>
// with coefficients
//     m*_0  = P
//     m*_a  = u_a + F_a/2
//     m*_ab = u_a u_b + (1-omega) Pn_ab + (u_a F_b + u_b F_a)/2
//     m*_r  = eq_r(u) + (1-omega) neq_r(u,Pn)          r >= 10 (HIGHORDER)
// where eq_r / neq_r are the monomials and recursive-regularisation terms the
// reference writes out for rows 10..26 (lb_cuda_fused_module.f90:667-703).
// On D3Q27 the expansion factorises over the three axes (D3Q27 = D1Q3^3),
// so populations come from 27 coefficients by three passes of a 3-point
// transform instead of a 27x27 product; D3Q19 uses the direct per-link form.
#pragma once
#include <cstdint>
#include <cuda_fp16.h>
#include <cuda_bf16.h>

namespace lbf {

// D3Q27 link table.  D3Q19 is its first 19 entries (vars_module.f90:666-684),
// D3Q15 the entries 0-6 and 19-26 (vars_module.f90:685-703): both in the
// reference's own link order, so loops over the D3Q27 indices of a lattice's
// links visit them in the reference's order.
__host__ __device__ constexpr int EX(int l) {
    constexpr int t[27] = {0, 1,-1, 0, 0, 0, 0, 1,-1, 1,-1, 0, 0, 0, 0, 1,-1,-1, 1, 1,-1, 1,-1,-1, 1, 1,-1};
    return t[l];
}
__host__ __device__ constexpr int EY(int l) {
    constexpr int t[27] = {0, 0, 0, 1,-1, 0, 0, 1,-1,-1, 1, 1,-1, 1,-1, 0, 0, 0, 0, 1,-1,-1, 1,-1, 1,-1, 1};
    return t[l];
}
__host__ __device__ constexpr int EZ(int l) {
    constexpr int t[27] = {0, 0, 0, 0, 0, 1,-1, 0, 0, 0, 0, 1,-1,-1, 1, 1,-1, 1,-1, 1,-1, 1,-1, 1,-1,-1, 1};
    return t[l];
}
__host__ __device__ constexpr int OPP(int l) {
    constexpr int t[27] = {0, 2, 1, 4, 3, 6, 5, 8, 7,10, 9,12,11,14,13,16,15,18,17,20,19,22,21,24,23,26,25};
    return t[l];
}
// is D3Q27 link l a link of lattice LAT (27, 19 or 15)
template <int LAT> __host__ __device__ constexpr bool IN(int l) {
    return LAT == 27 ? true : LAT == 19 ? l < 19 : (l < 7 || l >= 19);
}
__host__ __device__ constexpr bool in_lattice(int lat, int l) {
    return lat == 27 ? true : lat == 19 ? l < 19 : (l < 7 || l >= 19);
}
// weight of link l; D3Q27: 8/27, 2/27, 1/54, 1/216; D3Q19: 1/3, 1/18, 1/36;
// D3Q15: 2/9, 1/9, 1/72
template <int LAT> __host__ __device__ constexpr double WL(int l) {
    return LAT == 27 ? ((EX(l) * EX(l) + EY(l) * EY(l) + EZ(l) * EZ(l)) == 0 ? 8.0 / 27.0 :
                        (EX(l) * EX(l) + EY(l) * EY(l) + EZ(l) * EZ(l)) == 1 ? 2.0 / 27.0 :
                        (EX(l) * EX(l) + EY(l) * EY(l) + EZ(l) * EZ(l)) == 2 ? 1.0 / 54.0 : 1.0 / 216.0)
         : LAT == 19 ? ((EX(l) * EX(l) + EY(l) * EY(l) + EZ(l) * EZ(l)) == 0 ? 1.0 / 3.0 :
                        (EX(l) * EX(l) + EY(l) * EY(l) + EZ(l) * EZ(l)) == 1 ? 1.0 / 18.0 : 1.0 / 36.0)
                     : ((EX(l) * EX(l) + EY(l) * EY(l) + EZ(l) * EZ(l)) == 0 ? 2.0 / 9.0 :
                        (EX(l) * EX(l) + EY(l) * EY(l) + EZ(l) * EZ(l)) == 1 ? 1.0 / 9.0 : 1.0 / 72.0);
}
// link index of velocity (cx,cy,cz) in the D3Q27 ordering
__host__ __device__ constexpr int LINK(int cx, int cy, int cz) {
    int r = -1;
    for (int l = 0; l < 27; ++l)
        if (EX(l) == cx && EY(l) == cy && EZ(l) == cz) r = l;
    return r;
}

template <typename R> __device__ __forceinline__ R fmaf_t(R a, R b, R c) { return fma(a, b, c); }

// ---------------------------------------------------------------------------
// storage codecs: fields live in HBM as S; arithmetic is in R.  Scaled 16-bit
// storage keeps value*scale (scale per field, chosen on the host).
// ---------------------------------------------------------------------------
// ld = raw + dec: raw issues the load of a stored value, dec turns it into
// the arithmetic type, so a load can be issued well before its value is used
template <typename S> struct Codec;
template <> struct Codec<float> {
    static constexpr bool scaled = false;
    template <typename R> __device__ static R ld(const float* p, long long i, R) { return (R)__ldg(p + i); }
    __device__ static float raw(const float* p, long long i) { return __ldg(p + i); }
    template <typename R> __device__ static R dec(float s, R) { return (R)s; }
    template <typename R> __device__ static void st(float* p, long long i, R v, R) { p[i] = (float)v; }
};
template <> struct Codec<double> {
    static constexpr bool scaled = false;
    template <typename R> __device__ static R ld(const double* p, long long i, R) { return (R)__ldg(p + i); }
    __device__ static double raw(const double* p, long long i) { return __ldg(p + i); }
    template <typename R> __device__ static R dec(double s, R) { return (R)s; }
    template <typename R> __device__ static void st(double* p, long long i, R v, R) { p[i] = (double)v; }
};
template <> struct Codec<__half> {
    static constexpr bool scaled = true;
    template <typename R> __device__ static R ld(const __half* p, long long i, R inv) {
        return (R)__half2float(__ldg(p + i)) * inv;
    }
    __device__ static __half raw(const __half* p, long long i) { return __ldg(p + i); }
    template <typename R> __device__ static R dec(__half s, R inv) { return (R)__half2float(s) * inv; }
    template <typename R> __device__ static void st(__half* p, long long i, R v, R sc) {
        p[i] = __float2half_rn((float)(v * sc));
    }
};
template <> struct Codec<__nv_bfloat16> {
    static constexpr bool scaled = true;
    template <typename R> __device__ static R ld(const __nv_bfloat16* p, long long i, R inv) {
        return (R)__bfloat162float(__ldg(p + i)) * inv;
    }
    __device__ static __nv_bfloat16 raw(const __nv_bfloat16* p, long long i) { return __ldg(p + i); }
    template <typename R> __device__ static R dec(__nv_bfloat16 s, R inv) { return (R)__bfloat162float(s) * inv; }
    template <typename R> __device__ static void st(__nv_bfloat16* p, long long i, R v, R sc) {
        p[i] = __float2bfloat16_rn((float)(v * sc));
    }
};

// phi, P and the velocity keep 32-bit storage when the other moments are
// stored in 16 bits: phi lives in [0,1] and a 16-bit mantissa cannot resolve
// its interface profile; P and u are carried from step to step (P is
// conserved, u changes by the body force, ~1e-6 a step on ~1e-4 in a driven
// channel), so a 16-bit rounding of them every step would add up instead of
// relaxing away as the rounding of Pi - u u and of u_old (rewritten from the
// 32-bit u every step) does.
template <typename S> struct PhiStore { using type = S; };
template <> struct PhiStore<__half> { using type = float; };
template <> struct PhiStore<__nv_bfloat16> { using type = float; };

// Where the ten moment fields live.  FP32 / FP64 storage: one array of
// 10 x N in the storage type.  16-bit storage: P, u, v, w in an FP32 array of
// 4 x N (`pres`), Pi - u u in the 16-bit array (6 x N, field f >= 4 at
// (f - 4) x N).
template <typename S> struct Layout {
    static constexpr bool split = Codec<S>::scaled;
    static constexpr int nmom = split ? 6 : 10;  // fields of the storage-type array
    static constexpr int n32 = split ? 4 : 0;    // fields of the FP32 array
    // offset of field f in the storage-type array (f >= 4 when split)
    __host__ __device__ static constexpr long long off(int f, long long N) {
        return split ? (long long)(f - 4) * N : (long long)f * N;
    }
};

// field slots of the per-field scale table
enum : int { F_P = 0, F_U = 1, F_PXX = 4, F_UOLD = 10, F_PHI = 13, NSCALE = 14 };

// ---------------------------------------------------------------------------
// phi mass correction of a step's input phi (bcs_mesoscopic_phifields,
// boundary_cds_module.f90:1864-1885, with apply_lagrangian_phi_kernel,
// lb_cuda_boundary_module.f90:549-560).  m = {sum of the input phi over
// fluid nodes, count of those with 0.5 < phi < 0.9, the initial sum, the phi
// carried through open faces}, all FP64 in device memory.  The reference
// corrects the input phi in place after compute_norm has read it, so the
// gradient, normal and Laplacian of the step see the uncorrected values and
// the moments, collision and phi update the corrected ones; the kernels here
// leave phi in memory untouched and correct a node's value where those read it.
// ---------------------------------------------------------------------------
// correction per interface node, or false when there is none to apply
__device__ __forceinline__ bool mass_corr(const double* m, double& corr) {
    if (!m) return false;
    const double cnt = m[1];
    if (!(cnt > 0.0)) return false;
    corr = (m[2] + m[3] - m[0]) / cnt;
    return true;
}
// the corrected value of a fluid node, rounded to the storage type SP of phi
template <typename SP> __device__ __forceinline__ double mass_corrected(double v, double corr) {
    return (v > 0.5 && v < 0.9) ? (double)(SP)(v + corr) : v;
}

// ---------------------------------------------------------------------------
// kernel parameters (by value)
// ---------------------------------------------------------------------------
template <typename S, typename R> struct StepParams {
    int nx, ny, nz;
    int pbx, pby, pbz;
    long long plane;  // nx*ny
    long long N;      // nx*ny*nz
    int densratio, obstacles, write_u, smag;
    int zseg;         // planes per z segment
    int zlo, zhi;     // the planes advanced: zlo <= z < zhi (0 and nz but for a slab)
    R omega, visc1, visc2, rho_r, rho_b, beta, kapp, sharp_c, tau_diff, fx, fy, fz;
    R scale[NSCALE], inv_scale[NSCALE];
    const S* min;     // moments, input (10 x N; 16-bit storage: Pi - u u, 6 x N, see Layout)
    S* mout;          // moments, output
    const float* pres_in;  // 4 x N: P, u, v, w, input (16-bit storage only)
    float* pres_out;       // 4 x N: P, u, v, w, output (16-bit storage only)
    const S* uin;     // 3 x N velocity of the previous step (DENSRATIO)
    S* uout;          // 3 x N velocity after the force half-step
    const typename PhiStore<S>::type* pin;  // N phase field, input
    typename PhiStore<S>::type* pout;       // N phase field, output (fluid nodes)
    const int8_t* isf;  // N isfluid (obstacles), else nullptr
    int* err;         // device error word
    const R* rep;     // REPULSIVE_FLUX force (3 x N), else nullptr
    const double* mass;  // phi mass correction of the input phi (see mass_corr), else nullptr
};

}  // namespace lbf
