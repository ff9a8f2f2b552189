// lbf_walls.cu -- wall passes after the fused step: the open faces of the
// reference's bcs_mesoscopic_hfields (boundary_cds_module.f90:57-1311), the
// phi they carry (BCPHIFLUX, :1667-1861), and the half-way bounce-back of
// BOUNCE_BACK (lb_cuda_fused_module.f90:20-424).  They touch only the
// isfluid = -1 nodes next to walls, so they run as small kernels after the
// step, as the reference runs its wall code after its fused kernel.  A wall
// node needs its moments after the force half-step and its total force, which
// the fused step holds only in registers; these kernels recompute them from
// the step's input buffers (left intact by the step), so the fused step
// carries no code for them.
#include <type_traits>

#include "lbf_internal.h"
#include "lbf_stream_kernel.cuh"

namespace lbf {
namespace {

template <typename Fn> cudaError_t by_storage(int storage, Fn&& fn) {
    switch (storage) {
        case 0: return fn(float{});
        case 1: return fn(__half{});
        case 2: return fn(__nv_bfloat16{});
        case 3: return fn(double{});
    }
    return cudaErrorInvalidValue;
}

int grid_for(long long n, int bs) {
    long long b = (n + bs - 1) / bs;
    if (b > 148LL * 32) b = 148LL * 32;
    return (int)(b < 1 ? 1 : b);
}

// factor of axis multiplicity m of the D3Q27 Hermite row r in Minv_mrt(r, l)
// = w_l prod_axes F(m, c): 1, c / cs^2, (c^2 - cs^2) / (2 cs^4)
__device__ __forceinline__ double hfac(int m, int c) {
    return m == 0 ? 1.0 : m == 1 ? 3.0 * c : 4.5 * ((double)(c * c) - 1.0 / 3.0);
}

// axis multiplicities of the rows 10..26 of Minv_mrt (vars_module.f90:360-521)
__device__ __constant__ int c_hmul[17][3] = {
    {2, 1, 0}, {2, 0, 1}, {1, 2, 0}, {1, 0, 2}, {0, 1, 2}, {0, 2, 1}, {1, 1, 1}, {2, 2, 0}, {2, 0, 2},
    {0, 2, 2}, {1, 1, 2}, {1, 2, 1}, {2, 1, 1}, {2, 1, 2}, {2, 2, 1}, {1, 2, 2}, {2, 2, 2}};

// HIGHORDER coefficients of rows 10..26 of a population built from velocity
// (U, V, W) and non-equilibrium stress p (xx, yy, zz, xy, xz, yz): the
// equilibrium monomial + (1 - omega) x the non-equilibrium projection, as
// lb_cuda_fused_module.f90:667-703 writes them
__device__ void ho_coeffs(double U, double V, double W, const double (&p)[6], double om1, double (&hm)[17]) {
    const double pxx = p[0], pyy = p[1], pzz = p[2], pxy = p[3], pxz = p[4], pyz = p[5];
    const double eq[17] = {U * U * V, U * U * W, U * V * V, U * W * W, V * W * W, V * V * W, U * V * W,
                           U * U * V * V, U * U * W * W, V * V * W * W, U * V * W * W, U * V * V * W,
                           U * U * V * W, U * U * V * W * W, U * U * V * V * W, U * V * V * W * W,
                           U * U * V * V * W * W};
    const double nq[17] = {
        2 * pxy * U + pxx * V,
        2 * pxz * U + pxx * W,
        pyy * U + 2 * pxy * V,
        pzz * U + 2 * pxz * W,
        pzz * V + 2 * pyz * W,
        2 * pyz * V + pyy * W,
        pyz * U + pxz * V + pxy * W,
        pyy * U * U + 2 * V * (3 * pxy * U + pxx * V),
        pzz * U * U + 2 * W * (3 * pxz * U + pxx * W),
        pzz * V * V + 2 * W * (3 * pyz * V + pyy * W),
        pzz * U * V + W * (3 * pyz * U + 3 * pxz * V + 2 * pxy * W),
        2 * pyz * U * V + pxz * V * V + 2 * pyy * U * W + 4 * pxy * V * W,
        pyz * U * U + 2 * pxz * U * V + 4 * pxy * U * W + 2 * pxx * V * W,
        pzz * U * U * V + 3 * W * (pyz * U * U + 2 * pxz * U * V + 2 * pxy * U * W + pxx * V * W),
        2 * U * V * (pyz * U + pxz * V) + 2 * pyy * U * U * W + V * (10 * pxy * U + 3 * pxx * V) * W,
        pzz * U * V * V + 3 * W * (2 * pyz * U * V + pxz * V * V + pyy * U * W + 2 * pxy * V * W),
        pzz * U * U * V * V +
            W * (6 * U * V * (pyz * U + pxz * V) + 3 * pyy * U * U * W + 2 * V * (7 * pxy * U + 2 * pxx * V) * W)};
#pragma unroll
    for (int r = 0; r < 17; ++r) hm[r] = eq[r] + om1 * nq[r];
}

// sum_r Minv_mrt(r, l) hm[r] / w_l over rows 10..26 for link (cx, cy, cz)
__device__ double ho_sum(int cx, int cy, int cz, const double (&hm)[17]) {
    double hs = 0.0;
#pragma unroll
    for (int r = 0; r < 17; ++r)
        hs += hfac(c_hmul[r][0], cx) * hfac(c_hmul[r][1], cy) * hfac(c_hmul[r][2], cz) * hm[r];
    return hs;
}

// 4.5 (c c - cs^2 delta) : p  (with the off-diagonal terms counted twice)
__device__ __forceinline__ double qform(double dx, double dy, double dz, const double (&p)[6]) {
    const double cssq = 1.0 / 3.0;
    return 4.5 * ((dx * dx - cssq) * p[0] + (dy * dy - cssq) * p[1] + (dz * dz - cssq) * p[2] +
                  2.0 * (dx * dy) * p[3] + 2.0 * (dx * dz) * p[4] + 2.0 * (dy * dz) * p[5]);
}

// State of a wall node after the force half-step, recomputed in FP64 from the
// step's input buffers: moments (P, u, v, w, Pi) as the moments kernel leaves
// them (lb_cuda_moments_module.f90:104-339), the total force the collision
// uses, and phi -- with the phase-field inputs of compute_norm
// (lb_cuda_auxfields_module.f90:72-135) and div theta (:1136-1157) at the
// node, the 27-point stencils in full.
struct NodeState {
    double m[10];
    double tf[3];
    double phi, rhophi;
};

template <typename S>
__device__ void node_state(const BoundaryArgs& a, int x, int y, int z, long long g, NodeState& ns) {
    using SP = typename PhiStore<S>::type;
    using CD = Codec<S>;
    const long long plane = (long long)a.nx * a.ny, N = plane * a.nz;
    const S* min = static_cast<const S*>(a.min);
    const double cssq = 1.0 / 3.0;
    using LY = Layout<S>;
    double P, u, v, w;
    if constexpr (LY::split) {
        P = a.pres_in[g]; u = a.pres_in[N + g]; v = a.pres_in[2 * N + g]; w = a.pres_in[3 * N + g];
    } else {
        P = (double)CD::ld(min, g, 1.0);
        u = (double)CD::ld(min + N, g, 1.0 / a.scale[1]);
        v = (double)CD::ld(min + 2 * N, g, 1.0 / a.scale[2]);
        w = (double)CD::ld(min + 3 * N, g, 1.0 / a.scale[3]);
    }
    double pi[6];
#pragma unroll
    for (int f = 0; f < 6; ++f) pi[f] = (double)CD::ld(min + LY::off(4 + f, N), g, 1.0 / a.scale[4 + f]);
    if constexpr (CD::scaled) {  // 16-bit storage keeps Pi - u u
        pi[0] += u * u; pi[1] += v * v; pi[2] += w * w;
        pi[3] += u * v; pi[4] += u * w; pi[5] += v * w;
    }
    double phi = 0, lap = 0, divt = 0, gfx = 0, gfy = 0, gfz = 0;
    if (a.tc) {
        const SP* ph = static_cast<const SP*>(a.phi);
        // phi beyond a non-periodic face is 0 (never-written halo)
        auto PHI = [&](int i, int j, int k) -> double {
            bool ok = true;
            const int xx = wrap_coord(i, a.nx, a.pbx, ok), yy = wrap_coord(j, a.ny, a.pby, ok);
            const int zz = wrap_coord(k, a.nz, a.pbz, ok);
            return ok ? (double)ph[(long long)zz * plane + (long long)yy * a.nx + xx] : 0.0;
        };
        // theta = phi (1 - phi) n on fluid nodes, 0 elsewhere and beyond non-periodic faces
        double th[3][3][3][3];
#pragma unroll 1
        for (int dz = -1; dz <= 1; ++dz)
#pragma unroll 1
            for (int dy = -1; dy <= 1; ++dy)
#pragma unroll 1
                for (int dx = -1; dx <= 1; ++dx) {
                    const int i = x + dx, j = y + dy, k = z + dz;
                    bool ok = true;
                    const int xx = wrap_coord(i, a.nx, a.pbx, ok), yy = wrap_coord(j, a.ny, a.pby, ok);
                    const int zz = wrap_coord(k, a.nz, a.pbz, ok);
                    double t0 = 0, t1 = 0, t2 = 0;
                    if (ok) {
                        const int f = a.isf[(long long)zz * plane + (long long)yy * a.nx + xx];
                        if (f == 1 || f == -1) {
                            double gx, gy, gz;
                            iso_grad<double>([&](int p, int q, int r) { return PHI(i + p, j + q, k + r); }, gx, gy, gz);
                            const double mg = sqrt(gx * gx + gy * gy + gz * gz);
                            const double den = mg + 1.0e-9;
                            const double c0 = PHI(i, j, k);
                            t0 = c0 * (1.0 - c0) * (gx / den);
                            t1 = c0 * (1.0 - c0) * (gy / den);
                            t2 = c0 * (1.0 - c0) * (gz / den);
                            if (dx == 0 && dy == 0 && dz == 0) {
                                gfx = (gx / den) * mg; gfy = (gy / den) * mg; gfz = (gz / den) * mg;
                            }
                        }
                    }
                    th[0][dz + 1][dy + 1][dx + 1] = t0;
                    th[1][dz + 1][dy + 1][dx + 1] = t1;
                    th[2][dz + 1][dy + 1][dx + 1] = t2;
                }
        double d0, d1, d2, e0, e1, e2, f0, f1, f2;
        iso_grad<double>([&](int p, int q, int r) { return th[0][r + 1][q + 1][p + 1]; }, d0, d1, d2);
        iso_grad<double>([&](int p, int q, int r) { return th[1][r + 1][q + 1][p + 1]; }, e0, e1, e2);
        iso_grad<double>([&](int p, int q, int r) { return th[2][r + 1][q + 1][p + 1]; }, f0, f1, f2);
        divt = d0 + e1 + f2;
        phi = PHI(x, y, z);
        // 6 (sum_l w_l phi(x + c_l) - phi), D3Q27 weights
        double sw = 0;
#pragma unroll 1
        for (int l = 0; l < 27; ++l) sw += WL<27>(l) * PHI(x + EX(l), y + EY(l), z + EZ(l));
        lap = 6.0 * (sw - phi);
        // the moments, collision and phi update see the input phi after the
        // mass correction; compute_norm above read it before (see mass_corr)
        double corr;
        if (mass_corr(a.mass, corr)) phi = mass_corrected<SP>(phi, corr);
    }
    // moments prologue (lb_cuda_moments_module.f90:104-339)
    double rhophi = 1.0, fxv = a.fx, fyv = a.fy, fzv = a.fz, grx = 0, gry = 0, grz = 0, mask = 0, cv = 0;
    if (a.tc) mask = 4.0 * phi * (1.0 - phi);
    if (a.dr) {
        rhophi = a.rho_r * phi + (1.0 - phi) * a.rho_b;
        fxv = rhophi * a.fx; fyv = rhophi * a.fy; fzv = rhophi * a.fz;
    }
    if (a.tc) {
        const double chem = 4.0 * a.beta * phi * (phi - 1.0) * (phi - 0.5) - a.kapp * lap;
        fxv += chem * gfx; fyv += chem * gfy; fzv += chem * gfz;
        if (a.rep) {  // REPULSIVE_FLUX (lb_cuda_moments_module.f90:148-160)
            using R = typename std::conditional<sizeof(S) == 8, double, float>::type;
            const R* rp = static_cast<const R*>(a.rep);
            double t[3];
            for (int d = 0; d < 3; ++d) {
                t[d] = (double)rp[d * N + g] * rhophi;
                if (fabs(t[d]) > 1.0e-3) t[d] = t[d] > 0 ? 1.0e-3 : -1.0e-3;
            }
            fxv += t[0] * rhophi; fyv += t[1] * rhophi; fzv += t[2] * rhophi;
        }
    }
    if (a.dr) {
        grx = (a.rho_r - a.rho_b) * gfx; gry = (a.rho_r - a.rho_b) * gfy; grz = (a.rho_r - a.rho_b) * gfz;
        fxv -= mask * P * cssq * grx; fyv -= mask * P * cssq * gry; fzv -= mask * P * cssq * grz;
    }
    double tfx = fxv, tfy = fyv, tfz = fzv;
    if (a.dr) {
        const S* uin = static_cast<const S*>(a.uin);
        const double uo = (double)CD::ld(uin, g, 1.0 / a.scale[F_UOLD]);
        const double vo = (double)CD::ld(uin + N, g, 1.0 / a.scale[F_UOLD + 1]);
        const double wo = (double)CD::ld(uin + 2 * N, g, 1.0 / a.scale[F_UOLD + 2]);
        const double qxx = pi[0] - uo * uo, qyy = pi[1] - vo * vo, qzz = pi[2] - wo * wo;
        const double qxy = pi[3] - uo * vo, qxz = pi[4] - uo * wo, qyz = pi[5] - vo * wo;
        const double visc = (a.rho_r * a.visc1 * phi + (1.0 - phi) * a.visc2 * a.rho_b) / rhophi;
        cv = visc / ((visc * 3.0 + 0.5) * cssq);
        fxv -= mask * cv * (qxx * grx + qxy * gry + qxz * grz);
        fyv -= mask * cv * (qyy * gry + qxy * grx + qyz * grz);
        fzv -= mask * cv * (qzz * grz + qxz * grx + qyz * gry);
        u += 0.5 * fxv / rhophi; v += 0.5 * fyv / rhophi; w += 0.5 * fzv / rhophi;
        const double dd = (a.rho_r - a.rho_b) * (a.tau_diff * lap - a.sharp_c * divt);
        const double den = 1.0 - 0.5 * dd / rhophi;
        u /= den; v /= den; w /= den;
        tfx -= dd * u; tfy -= dd * v; tfz -= dd * w;
        fxv -= dd * u; fyv -= dd * v; fzv -= dd * w;
    } else {
        u += 0.5 * fxv / rhophi; v += 0.5 * fyv / rhophi; w += 0.5 * fzv / rhophi;
    }
    double* m = ns.m;
    m[0] = P; m[1] = u; m[2] = v; m[3] = w;
    m[4] = pi[0] + fxv * u / rhophi;
    m[5] = pi[1] + fyv * v / rhophi;
    m[6] = pi[2] + fzv * w / rhophi;
    m[7] = pi[3] + 0.5 * (fyv * u + fxv * v) / rhophi;
    m[8] = pi[4] + 0.5 * (fzv * u + fxv * w) / rhophi;
    m[9] = pi[5] + 0.5 * (fzv * v + fyv * w) / rhophi;
    if (a.dr) {
        const double qxx = m[4] - u * u, qyy = m[5] - v * v, qzz = m[6] - w * w;
        const double qxy = m[7] - u * v, qxz = m[8] - u * w, qyz = m[9] - v * w;
        tfx -= mask * cv * (qxx * grx + qxy * gry + qxz * grz);
        tfy -= mask * cv * (qyy * gry + qxy * grx + qyz * grz);
        tfz -= mask * cv * (qzz * grz + qxz * grx + qyz * gry);
    }
    ns.tf[0] = tfx; ns.tf[1] = tfy; ns.tf[2] = tfz;
    ns.phi = phi;
    ns.rhophi = rhophi;
}

// the step's output moments at node g, in the reference's convention
// (Pi = sum f (c c - cs^2 delta)), and back
template <typename S> __device__ void load_out(const BoundaryArgs& a, long long g, long long N, double (&o)[10]) {
    using CD = Codec<S>;
    using LY = Layout<S>;
    const S* mom = static_cast<const S*>(a.mom);
    if constexpr (LY::split) {
#pragma unroll
        for (int f = 0; f < 4; ++f) o[f] = a.pres[f * N + g];
    } else {
#pragma unroll
        for (int f = 0; f < 4; ++f) o[f] = (double)CD::ld(mom + f * N, g, 1.0 / a.scale[f]);
    }
#pragma unroll
    for (int f = 4; f < 10; ++f) o[f] = (double)CD::ld(mom + LY::off(f, N), g, 1.0 / a.scale[f]);
    if constexpr (CD::scaled) {  // 16-bit storage keeps Pi - u u
        o[4] += o[1] * o[1]; o[5] += o[2] * o[2]; o[6] += o[3] * o[3];
        o[7] += o[1] * o[2]; o[8] += o[1] * o[3]; o[9] += o[2] * o[3];
    }
}
template <typename S> __device__ void store_out(const BoundaryArgs& a, long long g, long long N, double (&o)[10]) {
    using R = typename std::conditional<sizeof(S) == 8, double, float>::type;
    using CD = Codec<S>;
    using LY = Layout<S>;
    S* mom = static_cast<S*>(a.mom);
    if constexpr (LY::split) {
#pragma unroll
        for (int f = 0; f < 4; ++f) a.pres[f * N + g] = (float)o[f];
        o[4] -= o[1] * o[1]; o[5] -= o[2] * o[2]; o[6] -= o[3] * o[3];
        o[7] -= o[1] * o[2]; o[8] -= o[1] * o[3]; o[9] -= o[2] * o[3];
    } else {
#pragma unroll
        for (int f = 0; f < 4; ++f) CD::st(mom + f * N, g, (R)o[f], (R)a.scale[f]);
    }
#pragma unroll
    for (int f = 4; f < 10; ++f) CD::st(mom + LY::off(f, N), g, (R)o[f], (R)a.scale[f]);
}

// add fp times the moment weights of link (dx, dy, dz) (reference convention)
__device__ __forceinline__ void add_link(double (&o)[10], double fp, double dx, double dy, double dz) {
    const double cssq = 1.0 / 3.0;
    o[0] += fp;
    o[1] += fp * dx; o[2] += fp * dy; o[3] += fp * dz;
    o[4] += fp * (dx * dx - cssq); o[5] += fp * (dy * dy - cssq); o[6] += fp * (dz * dz - cssq);
    o[7] += fp * (dx * dy); o[8] += fp * (dx * dz); o[9] += fp * (dy * dz);
}

// relaxation rate of the collision at a node: molecular from phi, or
// SMAGORINSKI from the non-equilibrium stress (lb_cuda_fused_module.f90:590-616)
__device__ double collision_omega(const BoundaryArgs& a, const NodeState& ns, const double (&pn)[6]) {
    const double inv = a.dr ? 1.0 / ns.rhophi : 1.0;
    double visc = a.visc1, om = a.omega;
    if (a.tc) {
        visc = (a.rho_r * a.visc1 * ns.phi + (1.0 - ns.phi) * a.visc2 * a.rho_b) * inv;
        om = 1.0 / (visc * 3.0 + 0.5);
    }
    if (a.smag) {
        const double QQ = pn[0] * pn[0] + pn[1] * pn[1] + pn[2] * pn[2] +
                          2.0 * (pn[3] * pn[3] + pn[4] * pn[4] + pn[5] * pn[5]);
        const double v3 = 3.0 * visc;
        om = 1.0 / (0.5 + (1.0 / 6.0) * (v3 + sqrt(v3 * v3 + SMAG_C * sqrt(2.0 * QQ) * inv)));
    }
    return om;
}

// Open face, one thread per face node; FP64 arithmetic, as the reference's
// boundary code (real(kind=db)), on every storage type.
template <typename S, int LAT, bool HO>
__global__ void open_face_kernel(const BoundaryArgs a) {
    const int n[3] = {a.nx, a.ny, a.nz};
    const int a1 = a.axis == 0 ? 1 : 0, a2 = a.axis == 2 ? 1 : 2;
    const int m1 = n[a1] - 2, m2 = n[a2] - 2;
    if (m1 <= 0 || m2 <= 0) return;
    const long long tot = (long long)m1 * m2;
    const long long plane = (long long)a.nx * a.ny, N = plane * a.nz;
    const double cssq = 1.0 / 3.0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
         t += (long long)gridDim.x * blockDim.x) {
        int x[3];
        x[a.axis] = a.side ? n[a.axis] - 2 : 1;
        x[a1] = 1 + (int)(t % m1);
        x[a2] = 1 + (int)(t / m1);
        const long long g = x[2] * plane + (long long)x[1] * a.nx + x[0];
        if (a.isf[g] != -1) continue;
        NodeState ns;
        node_state<S>(a, x[0], x[1], x[2], g, ns);
        // Pi' = Pi - cs^2 P - u u of the node's moments after the force half-step
        const double press = ns.m[0], u = ns.m[1], v = ns.m[2], w = ns.m[3];
        const double pq[6] = {ns.m[4] - cssq * press - u * u, ns.m[5] - cssq * press - v * v,
                              ns.m[6] - cssq * press - w * w, ns.m[7] - u * v, ns.m[8] - u * w, ns.m[9] - v * w};
        // the molecular relaxation rate (boundary_cds_module.f90:151-162)
        double om = a.omega;
        if (a.tc) {
            const double visc = (a.rho_r * a.visc1 * ns.phi + (1.0 - ns.phi) * a.visc2 * a.rho_b) / ns.rhophi;
            om = 1.0 / (visc * 3.0 + 0.5);
        }
        const double om1 = 1.0 - om;
        double pb = press, ub = u, vb = v, wb = w;
        if (a.type == 1) {
            pb = a.press;
        } else if (a.type != 2) {
            ub = a.vel[0]; vb = a.vel[1]; wb = a.vel[2];
        }
        const double uu = 0.5 * (ub * ub + vb * vb + wb * wb) * 3.0;
        double hm[17];
        if constexpr (HO) ho_coeffs(ub, vb, wb, pq, om1, hm);
        double o[10];
        load_out<S>(a, g, N, o);
#pragma unroll
        for (int l = 1; l < 27; ++l) {
            if (!IN<LAT>(l)) continue;
            const int cx = EX(l), cy = EY(l), cz = EZ(l);
            // upstream node x - c_l: inside the box (the face nodes keep one
            // node away from every box face)
            const long long gu = g - ((long long)cz * plane + (long long)cy * a.nx + cx);
            if (a.isf[gu] != 0) continue;
            const double wl = WL<LAT>(l);
            const double dx = cx, dy = cy, dz = cz;
            const double qn = qform(dx, dy, dz, pq);
            // the bounce-back population, taken out with the weights c_a c_b
            const double fo = wl * press + om1 * (wl * qn);
            o[0] -= fo;
            o[1] -= fo * dx; o[2] -= fo * dy; o[3] -= fo * dz;
            o[4] -= fo * (dx * dx); o[5] -= fo * (dy * dy); o[6] -= fo * (dz * dz);
            o[7] -= fo * (dx * dy); o[8] -= fo * (dx * dz); o[9] -= fo * (dy * dz);
            // the face's population
            const double udotc = (ub * dx + vb * dy + wb * dz) * 3.0;
            double fn = wl * (pb + udotc + 0.5 * udotc * udotc - uu) + om1 * (wl * qn);
            if constexpr (HO) fn += wl * ho_sum(cx, cy, cz, hm);
            add_link(o, fn, dx, dy, dz);
        }
        store_out<S>(a, g, N, o);
    }
}

// BOUNCE_BACK, one thread per isfluid = -1 node.  The step added for each
// wall link l (upstream x - c_l solid) the moment-space population
// w_l P + (1 - omega) fneq (LB_int_boundary, lb_cuda_boundary_module.f90:162-199)
// and the solid node's push, which is zero; fused_LB_kernel_bb
// (lb_cuda_fused_module.f90:364-380) brings instead the node's own
// post-collision population of the opposite link.  FP64.
template <typename S, int LAT, bool HO>
__global__ void bounce_back_kernel(const BoundaryArgs a) {
    const long long plane = (long long)a.nx * a.ny, N = plane * a.nz;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < a.nnodes;
         t += (long long)gridDim.x * blockDim.x) {
        const long long g = a.nodes[t];
        const int z = (int)(g / plane), y = (int)((g - z * plane) / a.nx), x = (int)(g - z * plane - (long long)y * a.nx);
        NodeState ns;
        node_state<S>(a, x, y, z, g, ns);
        const double P = ns.m[0], u = ns.m[1], v = ns.m[2], w = ns.m[3];
        const double pn[6] = {ns.m[4] - u * u, ns.m[5] - v * v, ns.m[6] - w * w,
                              ns.m[7] - u * v, ns.m[8] - u * w, ns.m[9] - v * w};
        const double om = collision_omega(a, ns, pn);
        const double om1 = 1.0 - om;
        const double inv = a.dr ? 1.0 / ns.rhophi : 1.0;
        const double Fx = ns.tf[0] * inv, Fy = ns.tf[1] * inv, Fz = ns.tf[2] * inv;
        const double uu = 0.5 * (u * u + v * v + w * w) * 3.0;
        double hm[17];
        if constexpr (HO) ho_coeffs(u, v, w, pn, om1, hm);
        double o[10];
        load_out<S>(a, g, N, o);
#pragma unroll
        for (int l = 1; l < 27; ++l) {
            if (!IN<LAT>(l)) continue;
            const int cx = EX(l), cy = EY(l), cz = EZ(l);
            bool ok = true;
            const int ux = wrap_coord(x - cx, a.nx, a.pbx, ok), uy = wrap_coord(y - cy, a.ny, a.pby, ok);
            const int uz = wrap_coord(z - cz, a.nz, a.pbz, ok);
            if (!ok || a.isf[(long long)uz * plane + (long long)uy * a.nx + ux] != 0) continue;
            const double dx = cx, dy = cy, dz = cz;
            // out: the moment-space population of link l the step added
            const double wl = WL<LAT>(l);
            add_link(o, -(wl * P + om1 * (wl * qform(dx, dy, dz, pn))), dx, dy, dz);
            // in: the node's post-collision population of the opposite link,
            // arriving as link l (lb_cuda_fused_module.f90:637-713)
            const double ex = -dx, ey = -dy, ez = -dz;
            const double ud = (u * ex + v * ey + w * ez) * 3.0;
            double feq = wl * (P + ud + 0.5 * ud * ud - uu);
            double fne = om1 * (wl * qform(ex, ey, ez, pn));
            if constexpr (HO) feq += wl * ho_sum(-cx, -cy, -cz, hm);
            const double fd = wl * (((ex - u) + ud * ex) * Fx + ((ey - v) + ud * ey) * Fy + ((ez - w) + ud * ez) * Fz) * 3.0;
            add_link(o, feq + fne + 0.5 * fd, dx, dy, dz);
        }
        store_out<S>(a, g, N, o);
    }
}

template <typename S>
__global__ void phi_flux_kernel(int nx, int ny, int nz, int axis, int side, const S* mom, const float* pres,
                                const void* phi_, const int8_t* isf, double inv_scale, double* out) {
    using SP = typename PhiStore<S>::type;
    using CD = Codec<S>;
    const SP* phi = static_cast<const SP*>(phi_);
    const int n[3] = {nx, ny, nz};
    const int a1 = axis == 0 ? 1 : 0, a2 = axis == 2 ? 1 : 2;
    const long long tot = (long long)n[a1] * n[a2];
    const long long plane = (long long)nx * ny, N = plane * nz;
    // the velocity component normal to the face (FP32 with 16-bit storage)
    const S* un = mom + (1 + axis) * N;
    const float* un32 = Layout<S>::split ? pres + (1 + axis) * N : nullptr;
    double acc = 0.0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
         t += (long long)gridDim.x * blockDim.x) {
        int x[3];
        x[axis] = side ? n[axis] - 2 : 1;
        x[a1] = (int)(t % n[a1]);
        x[a2] = (int)(t / n[a1]);
        const long long g = x[2] * plane + (long long)x[1] * nx + x[0];
        if (isf[g] != -1) continue;
        const double q = (un32 ? (double)un32[g] : (double)CD::ld(un, g, inv_scale)) * (double)phi[g];
        acc += side ? -q : q;
    }
    __shared__ double red[256];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicAdd(out, red[0]);
}

}  // namespace

cudaError_t launch_open_face(int storage, const BoundaryArgs& a, cudaStream_t st) {
    const int n[3] = {a.nx, a.ny, a.nz};
    const long long tot = (long long)(n[a.axis == 0 ? 1 : 0] - 2) * (n[a.axis == 2 ? 1 : 2] - 2);
    if (tot <= 0 || n[a.axis] < 3) return cudaSuccess;
    const int grid = grid_for(tot, 128);
    return by_storage(storage, [&](auto tag) {
        using S = decltype(tag);
        if (a.lattice == 27 && a.highorder) open_face_kernel<S, 27, true><<<grid, 128, 0, st>>>(a);
        else if (a.lattice == 27) open_face_kernel<S, 27, false><<<grid, 128, 0, st>>>(a);
        else if (a.lattice == 19) open_face_kernel<S, 19, false><<<grid, 128, 0, st>>>(a);
        else open_face_kernel<S, 15, false><<<grid, 128, 0, st>>>(a);
        return cudaGetLastError();
    });
}

cudaError_t launch_bounce_back(int storage, const BoundaryArgs& a, cudaStream_t st) {
    if (a.nnodes <= 0) return cudaSuccess;
    const int grid = grid_for(a.nnodes, 128);
    return by_storage(storage, [&](auto tag) {
        using S = decltype(tag);
        if (a.lattice == 27 && a.highorder) bounce_back_kernel<S, 27, true><<<grid, 128, 0, st>>>(a);
        else if (a.lattice == 27) bounce_back_kernel<S, 27, false><<<grid, 128, 0, st>>>(a);
        else if (a.lattice == 19) bounce_back_kernel<S, 19, false><<<grid, 128, 0, st>>>(a);
        else bounce_back_kernel<S, 15, false><<<grid, 128, 0, st>>>(a);
        return cudaGetLastError();
    });
}

cudaError_t launch_phi_flux(int storage, int nx, int ny, int nz, int open, const void* mom, const float* pres,
                            const void* phi, const int8_t* isf, const double* inv_scale, double* d_flux,
                            cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(d_flux, 0, sizeof(double), st);
    if (e != cudaSuccess) return e;
    const int n[3] = {nx, ny, nz};
    return by_storage(storage, [&](auto tag) {
        using S = decltype(tag);
        for (int axis = 0; axis < 3; ++axis) {
            if (!(open & (1 << axis)) || n[axis] < 3) continue;
            const long long tot = (long long)n[axis == 0 ? 1 : 0] * n[axis == 2 ? 1 : 2];
            for (int side = 0; side < 2; ++side)
                phi_flux_kernel<S><<<grid_for(tot, 256), 256, 0, st>>>(nx, ny, nz, axis, side,
                                                                       static_cast<const S*>(mom), pres, phi, isf,
                                                                       inv_scale[1 + axis], d_flux);
        }
        return cudaGetLastError();
    });
}

}  // namespace lbf
