// lbf_stream.cuh -- the fused LBFAST time step for sm_100a.
//
// One launch performs what the reference does in five kernels plus four
// halo copies per half-step (integrator_module.f90:270-544):
//   compute_norm_interface (lb_cuda_auxfields_module.f90:19-139)
//   compute_div_theta_n    (lb_cuda_auxfields_module.f90:1085-1164)
//   moments_LB             (lb_cuda_moments_module.f90:19-341)
//   fused_LB collide+stream(lb_cuda_fused_module.f90:426-750)
//   update_phifields       (lb_cuda_update_phi_module.f90:19-104)
//   LB_int_boundary        (lb_cuda_boundary_module.f90:19-216)
//   exchange_*_intpbc      (mpi_module.f90:2203-3286) -> periodic index wrap
//
// Work decomposition.  A CTA owns a 32 x TY column of the box and sweeps a
// segment of z planes.  For collision plane q it keeps in shared memory
//   phi   planes q-1..q+3 on the tile + 3-node ring   (5-slot ring)
//   in-plane partials of the separable phase-field stencils of phi (tile +
//           2-node ring) and of theta (tile + 1-node ring)
//   theta = phi(1-phi) n on the tile + 2-node ring and g~ = n|grad phi| on
//           the tile + 1-node ring
//   post-collision populations of plane q on the tile + 1-node ring (the
//           centre group of a node, read only by its own output, stays in
//           the registers of the thread that collided it).
// Each output node then pulls f*_l(x - c_l) from shared memory: the nine
// (cx,cy) populations of each cz slice of plane q go to output plane q+cz,
// accumulated in registers; plane q-1 is complete after plane q and is
// written out.  Halo nodes are recomputed instead of exchanged, so one step
// reads the moments, the previous velocity and phi once and writes them once
// (plus halo rereads that hit L2).
//
// Non-periodic directions: nodes outside the box carry isfluid = 1 and zero
// fields, as the reference's never-written halo layers do.
#pragma once
#include "lbf_lattice.cuh"

namespace lbf {

constexpr int TX = 32;                                   // tile width: one warp per tile row
constexpr int R1X = TX + 2, R2X = TX + 4, R3X = TX + 6;  // region widths
constexpr int PHI_SLOTS = 5;

// A tile of TY_ rows (8 or 16) and its regions: collision R1 = tile + 1-node
// ring, theta R2 = tile + 2, phi R3 = tile + 3.
template <int TY_> struct Tile {
    static constexpr int TY = TY_, NT = TX * TY_;
    static constexpr int R1Y = TY_ + 2, R1N = R1X * R1Y;
    static constexpr int R2Y = TY_ + 4, R2N = R2X * R2Y;
    static constexpr int R3Y = TY_ + 6, R3N = R3X * R3Y;
    static constexpr int NRING1 = R1N - NT;  // ring nodes of R1 (84 for 8 rows, 100 for 16)
    // The ring collisions go to the last RW warps (a warp pays for its slowest
    // lane, so those warps carry two collisions); the theta work goes to the
    // other NTH threads only, KTH nodes each, which balances the first phase.
    static constexpr int RW = (NRING1 + 31) / 32;
    static constexpr int NTH = NT - 32 * RW;
    static constexpr int KTH = (R2N + NTH - 1) / NTH;
    static_assert(R3N <= 3 * NT, "phi loads assume at most 3 nodes per thread");
    static_assert(KTH <= 3, "theta nodes per thread");
};

__device__ __forceinline__ int wrap_coord(int g, int n, int periodic, bool& ok) {
    if (g < 0) {
        if (periodic) { g = g % n; if (g < 0) g += n; } else ok = false;
    } else if (g >= n) {
        if (periodic) g = g % n; else ok = false;
    }
    return g;
}

// D3Q27 isotropic gradient of the reference (lb_cuda_auxfields_module.f90:72-100),
// always with D3Q27 weights (used by the wetting kernel; the step kernel
// evaluates the same stencil in separable form).  a(i,j,k) reads phi at offset (i,j,k).
template <typename R, typename A> __device__ __forceinline__ void iso_grad(const A& a, R& gx, R& gy, R& gz) {
    const R p1 = R(2.0 / 27.0), p2 = R(1.0 / 54.0), p3 = R(1.0 / 216.0);
    gx = R(3) * (p1 * (a(1, 0, 0) - a(-1, 0, 0)) +
                 p2 * ((a(1, 1, 0) - a(-1, -1, 0)) + (a(1, -1, 0) - a(-1, 1, 0)) +
                       (a(1, 0, 1) - a(-1, 0, -1)) + (a(1, 0, -1) - a(-1, 0, 1))) +
                 p3 * ((a(1, 1, 1) - a(-1, -1, -1)) + (a(1, -1, -1) - a(-1, 1, 1)) +
                       (a(1, -1, 1) - a(-1, 1, -1)) + (a(1, 1, -1) - a(-1, -1, 1))));
    gy = R(3) * (p1 * (a(0, 1, 0) - a(0, -1, 0)) +
                 p2 * ((a(1, 1, 0) - a(-1, -1, 0)) + (a(-1, 1, 0) - a(1, -1, 0)) +
                       (a(0, 1, 1) - a(0, -1, -1)) + (a(0, 1, -1) - a(0, -1, 1))) +
                 p3 * ((a(1, 1, 1) - a(-1, -1, -1)) + (a(-1, 1, -1) - a(1, -1, 1)) +
                       (a(1, 1, -1) - a(-1, -1, 1)) + (a(-1, 1, 1) - a(1, -1, -1))));
    gz = R(3) * (p1 * (a(0, 0, 1) - a(0, 0, -1)) +
                 p2 * ((a(1, 0, 1) - a(-1, 0, -1)) + (a(-1, 0, 1) - a(1, 0, -1)) +
                       (a(0, 1, 1) - a(0, -1, -1)) + (a(0, -1, 1) - a(0, 1, -1))) +
                 p3 * ((a(1, 1, 1) - a(-1, -1, -1)) + (a(-1, -1, 1) - a(1, 1, -1)) +
                       (a(1, -1, 1) - a(-1, 1, -1)) + (a(-1, 1, 1) - a(1, -1, -1))));
}

// 1-D D1Q3 inverse transform: Hermite coefficients (m0, m1, m2) -> values at c = -1, 0, +1
template <typename R> __device__ __forceinline__ void d1q3_inv(R m0, R m1, R m2, R& vm, R& v0, R& vp) {
    R s = fmaf_t(m0, R(1.0 / 6.0), R(0.5) * m2);
    R d = R(0.5) * m1;
    vm = s - d;
    vp = s + d;
    v0 = fmaf_t(m0, R(2.0 / 3.0), -m2);
}

}  // namespace lbf
