// lbf_stream_kernel.cuh -- body of the fused step kernel (see lbf_stream.cuh).
//
// Per z plane q a CTA runs two barrier phases:
//   phase 1  the in-plane partials of phi(q+3) and theta(q+2) on the theta
//            region, and the moments prologue + collision of plane q on the
//            collision region (populations to shared memory).  The two sets
//            of work are independent, so one barrier covers both, and the
//            halo-ring collisions are placed on the warps with no theta work.
//            Before the barrier each thread issues the loads of its interior
//            node's fields of plane q+1.
//   phase 2  an asynchronous copy (cp.async) of phi(q+4) into its ring
//            slot; the theta partials of plane q+2; then every output node
//            pulls the populations of plane q and plane q-1 is written.  The
//            copy completes behind this phase.
#pragma once
#include "lbf_stream.cuh"

namespace lbf {

// Reciprocal and square root: in FP32 the hardware approximations (about 2 ulp)
// instead of the correctly rounded sequences, which cost several instructions
// and a branch each; FP64 stays correctly rounded.
template <typename R> __device__ __forceinline__ R rcp(R x);
template <> __device__ __forceinline__ float rcp<float>(float x) { return __fdividef(1.0f, x); }
template <> __device__ __forceinline__ double rcp<double>(double x) { return 1.0 / x; }
template <typename R> __device__ __forceinline__ R sqrt_a(R x);
template <> __device__ __forceinline__ float sqrt_a<float>(float x) { return x > 0.0f ? x * rsqrtf(x) : 0.0f; }
template <> __device__ __forceinline__ double sqrt_a<double>(double x) { return sqrt(x); }

template <typename R>
__device__ __forceinline__ void accum_slice(R (&acc)[10], R cz, R Y00, R Y01, R Y02, R Y10, R Y11, R Y20) {
    acc[0] += Y00;
    acc[1] += Y10;
    acc[2] += Y01;
    acc[3] += cz * Y00;
    acc[4] += Y20;
    acc[5] += Y02;
    acc[6] += (cz * cz) * Y00;
    acc[7] += Y11;
    acc[8] += cz * Y10;
    acc[9] += cz * Y01;
}

// asynchronous global -> shared copies of 4 or 8 bytes
template <int BYTES> __device__ __forceinline__ void cp_async(void* smem, const void* gmem) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    if constexpr (BYTES == 4) {
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
    } else {
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
    }
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Smagorinsky constant of the reference: the single-precision product 0.053 * 18.0
constexpr double SMAG_C = (double)(0.053f * 18.0f);

// The moments (and u_old) of a collision node go from global memory straight
// into registers: the tile-interior node's one plane ahead (NodeRaw, below),
// the ring nodes' at the point of use.  A cp.async prefetch of them into a
// shared staging area, one plane ahead, lost more than it hid: its
// shared-memory writes were bank-conflicted (13.6 M of the 19.8 M conflicts of a
// 256^3 FP32 launch) and the extra 52 B/node of shared traffic competed with the
// population exchange; without it the FP32 Laplace step ran 14.1 against 12.0
// GLUPS.

// ring slots of the separable phase-field stencils (see step_body)
constexpr int SXY_SLOTS = 5, GXY_SLOTS = 3, TH_SLOTS = 2, GT_SLOTS = 3, H_SLOTS = 3;

// vector of two R (the populations of cz = -1 and 0 of one (cx, cy) group)
template <typename R> struct Vec2;
template <> struct Vec2<float> { using type = float2; };
template <> struct Vec2<double> { using type = double2; };

// Pairs of independent values in one instruction: FP32 as f32x2 (FFMA2,
// FADD2, FMUL2 of sm_100: two lanes' operations per issue slot, each rounded
// as the scalar instruction), FP64 as two scalar operations
template <typename R> struct PK;
template <> struct PK<float> {
    using T = float2;
    static __device__ __forceinline__ float2 mk(float a, float b) { return make_float2(a, b); }
    static __device__ __forceinline__ float2 fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
    static __device__ __forceinline__ float2 add(float2 a, float2 b) { return __fadd2_rn(a, b); }
    static __device__ __forceinline__ float2 mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
};
template <> struct PK<double> {
    using T = double2;
    static __device__ __forceinline__ double2 mk(double a, double b) { return make_double2(a, b); }
    static __device__ __forceinline__ double2 fma(double2 a, double2 b, double2 c) {
        return make_double2(::fma(a.x, b.x, c.x), ::fma(a.y, b.y, c.y));
    }
    static __device__ __forceinline__ double2 add(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
    static __device__ __forceinline__ double2 mul(double2 a, double2 b) { return make_double2(a.x * b.x, a.y * b.y); }
};
// d1q3_inv with the second coefficient negated (m2n = -m2), the same
// roundings: scalar and packed
template <typename R> __device__ __forceinline__ void d1q3n(R m0, R m1, R m2n, R& vm, R& v0, R& vp) {
    const R s = fmaf_t(m0, R(1.0 / 6.0), R(-0.5) * m2n);
    const R d = R(0.5) * m1;
    vm = s - d;
    vp = s + d;
    v0 = fmaf_t(m0, R(2.0 / 3.0), m2n);
}
template <typename R, typename T = typename PK<R>::T>
__device__ __forceinline__ void d1q3n2(T m0, T m1, T m2n, T& vm, T& v0, T& vp) {
    using P = PK<R>;
    const T s = P::fma(m0, P::mk(R(1.0 / 6.0), R(1.0 / 6.0)), P::mul(P::mk(R(-0.5), R(-0.5)), m2n));
    const T d = P::mul(P::mk(R(0.5), R(0.5)), m1);
    vm = P::fma(d, P::mk(R(-1), R(-1)), s);
    vp = P::add(s, d);
    v0 = P::fma(m0, P::mk(R(2.0 / 3.0), R(2.0 / 3.0)), m2n);
}

template <int LAT, bool TC, typename S, typename R, int TYV> constexpr size_t stream_smem_bytes() {
    constexpr int R1N = Tile<TYV>::R1N, R2N = Tile<TYV>::R2N, R3N = Tile<TYV>::R3N;
    size_t b = sizeof(R) * size_t(24) * R1N;  // populations: 8 (cx, cy) groups x 3 cz (the centre stays in registers)
    if (TC)
        b += sizeof(R) * (size_t(PHI_SLOTS) * R3N + size_t(SXY_SLOTS) * R2N + size_t(GXY_SLOTS) * 2 * R2N +
                          size_t(TH_SLOTS) * 3 * R2N + size_t(GT_SLOTS) * 3 * R1N + size_t(H_SLOTS) * 3 * R1N);
    return b;
}

// One piece of a time step: tile (bx, by) of the box, planes z0 <= z < z1.
// REP: REPULSIVE_FLUX force in the moments prologue; OBS: obstacles (isfluid
// tests, the moment-space bounce-back, open-face moments).  Both are separate
// compilations, so the kernels without them carry no code for them: the
// obstacle code alone, never executed, costs a box without obstacles 5.6 %.
template <int LAT, bool HO, bool TC, typename S, typename R, int TYV, bool REP = false, bool OBS = true>
__device__ __forceinline__ void step_body(const StepParams<S, R>& p, const int bx, const int by, const int z0,
                                          const int z1) {
    using TL = Tile<TYV>;
    constexpr int TY = TL::TY, NT = TL::NT, NRING1 = TL::NRING1, NTH = TL::NTH, KTH = TL::KTH;
    constexpr int R1Y = TL::R1Y, R1N = TL::R1N, R2Y = TL::R2Y, R2N = TL::R2N, R3N = TL::R3N;
    using CD = Codec<S>;
    using SP = typename PhiStore<S>::type;
    using CP = Codec<SP>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    // post-collision populations of plane q, by (cx, cy) group g = 3 (cy+1) + (cx+1):
    // the output nodes that read one group of a node read all three cz of it
    using R2 = typename Vec2<R>::type;
    // (the centre group (0, 0) of a node is read only by the node's own
    // output, the thread that collided it: it stays in registers)
    R2* pops2 = reinterpret_cast<R2*>(smem_raw);                  // [8][R1N] (cz = -1, cz = 0)
    R* pops1 = reinterpret_cast<R*>(pops2 + 8 * R1N);             // [8][R1N] (cz = +1)
    R* phis = pops1 + 8 * R1N;                         // [PHI_SLOTS][R3N]     (TC)
    auto gslot = [](int g) { return g < 4 ? g : g - 1; };  // shared slot of group g != 4
    R* sxys = phis + (TC ? PHI_SLOTS * R3N : 0);       // [SXY_SLOTS][R2N]     (TC) S_x S_y phi
    R* gxys = sxys + (TC ? SXY_SLOTS * R2N : 0);       // [GXY_SLOTS][2][R2N]  (TC) D_x S_y phi, S_x D_y phi
    R* ths = gxys + (TC ? GXY_SLOTS * 2 * R2N : 0);    // [TH_SLOTS][3][R2N]   (TC) theta
    R* gts = ths + (TC ? TH_SLOTS * 3 * R2N : 0);      // [GT_SLOTS][3][R1N]   (TC) g~
    R* hs = gts + (TC ? GT_SLOTS * 3 * R1N : 0);       // [H_SLOTS][3][R1N]    (TC) theta partials

    const int t = threadIdx.x;
    const int tx = t % TX, ty = t / TX;
    const int X0 = bx * TX, Y0 = by * TY;
    // node indices inside one field fit in 32 bits (boxes hold < 2^31 nodes);
    // field bases (f * N) are 64-bit and uniform across the CTA
    const long long N = p.N;
    const int plane = (int)p.plane;
    const int nx = p.nx, ny = p.ny, nz = p.nz;
    const bool dr = TC && p.densratio;
    const bool obs = OBS && p.obstacles != 0;
    const R cssq = R(1.0 / 3.0);

    // ---- static per-thread node tables (x/y wrap does not change along z) ----
    // collision nodes: A = tile interior node t; B = ring node r for the threads
    // of the last warps (t >= NTH), r = t - NTH < NRING1
    const int nodeA = (ty + 1) * R1X + (tx + 1);
    int nodeB = -1;
    {
        const int r = t - NTH;
        if (r >= 0 && r < NRING1) {
            // one kind of ring node per warp: the inner 32 nodes of the top row,
            // of the bottom row, then the left and right columns with the corners
            if (r < TX) nodeB = r + 1;                                              // top row
            else if (r < 2 * TX) nodeB = (R1Y - 1) * R1X + (r - TX + 1);            // bottom row
            else if (r < 2 * TX + R1Y) nodeB = (r - 2 * TX) * R1X;                  // left column
            else nodeB = (r - 2 * TX - R1Y) * R1X + (R1X - 1);                      // right column
        }
    }
    // ring nodes stream into the tile along one axis only: the rows' along y
    // (cy = +1 from the top row, -1 from the bottom), the columns' along x
    // (cx = +1 from the left, -1 from the right; corners with them).  ring_col
    // is uniform across a warp (the ring warps hold 32 row nodes each, then
    // the columns).
    const bool ring_col = (t - NTH) >= 2 * TX;
    R ring_dir = R(0);
    if (nodeB >= 0) {
        const int bx = nodeB % R1X, by = nodeB / R1X;
        ring_dir = ring_col ? (bx == 0 ? R(1) : R(-1)) : (by == 0 ? R(1) : R(-1));
    }
    // wrapped: the node was reached across a periodic face in x or y
    auto r1_geom = [&](int node, int& off, bool& wrapped) -> bool {
        wrapped = false;
        if (node < 0) { off = 0; return false; }
        int hx = node % R1X, hy = node / R1X;
        bool ok = true;
        const int gx0 = X0 + hx - 1, gy0 = Y0 + hy - 1;
        int gx = wrap_coord(gx0, nx, p.pbx, ok);
        int gy = wrap_coord(gy0, ny, p.pby, ok);
        wrapped = gx != gx0 || gy != gy0;
        off = ok ? gy * nx + gx : 0;
        return ok;
    };
    int offA, offB;
    bool wrapA, wrapB;
    const bool okA = r1_geom(nodeA, offA, wrapA);
    const bool okB = r1_geom(nodeB, offB, wrapB);
    // phi mass correction of the input phi (compiled with the obstacle code only)
    double mcorr = 0.0;
    bool do_mcorr = false;
    if constexpr (OBS && TC) do_mcorr = mass_corr(p.mass, mcorr);
    const int ox = X0 + tx, oy = Y0 + ty;
    const bool out_ok = (ox < nx) && (oy < ny);
    const int out_off = oy * nx + ox;


    // theta nodes (R2): slot n = t + k NTH of the first NTH threads; phi nodes
    // (R3): t, t + NT, t + 2 NT.  Slot n maps to the first TX columns of each
    // row of the theta region, one row per warp, then to the remaining
    // R2X - TX columns of every row: a warp's loads from the rings then stay
    // in one row, 32 consecutive words, instead of straddling two rows of the
    // wider rings (a two-way bank conflict).  Storage stays row-major.
    auto r2_node = [](int n, int& hx, int& hy) {
        constexpr int MAIN = TX * Tile<TYV>::R2Y;
        if (n < MAIN) {
            hy = n / TX; hx = n % TX;
        } else {
            const int e = n - MAIN;
            hy = e / (R2X - TX); hx = TX + e % (R2X - TX);
        }
    };
    int r2_off[KTH];
    bool r2_ok[KTH];
#pragma unroll
    for (int k = 0; k < KTH; ++k) {
        r2_off[k] = 0;
        r2_ok[k] = false;
    }
    int r3_off[3] = {0, 0, 0};
    bool r3_ok[3] = {false, false, false};
    if constexpr (TC) {
#pragma unroll
        for (int k = 0; k < KTH; ++k) {
            int n = t + k * NTH;
            if (t < NTH && n < R2N) {
                int hx, hy;
                r2_node(n, hx, hy);
                bool ok = true;
                int gx = wrap_coord(X0 + hx - 2, nx, p.pbx, ok);
                int gy = wrap_coord(Y0 + hy - 2, ny, p.pby, ok);
                r2_ok[k] = ok;
                r2_off[k] = ok ? gy * nx + gx : 0;
            }
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            int n = t + k * NT;
            if (n < R3N) {
                int hx = n % R3X, hy = n / R3X;
                bool ok = true;
                int gx = wrap_coord(X0 + hx - 3, nx, p.pbx, ok);
                int gy = wrap_coord(Y0 + hy - 3, ny, p.pby, ok);
                r3_ok[k] = ok;
                r3_off[k] = ok ? gy * nx + gx : 0;
            }
        }
    }

    auto zwrap = [&](int q, bool& ok) { return wrap_coord(q, nz, p.pbz, ok); };
    auto phi_slot = [&](int q) { return (int)((unsigned)(q - z0 + 3) % (unsigned)PHI_SLOTS); };
    auto sxy_slot = [&](int q) { return (int)((unsigned)(q - z0 + 3) % (unsigned)SXY_SLOTS); };
    auto gxy_slot = [&](int q) { return (int)((unsigned)(q - z0 + 3) % (unsigned)GXY_SLOTS); };
    auto th_slot = [&](int q) { return (int)((unsigned)(q - z0 + 3) % (unsigned)TH_SLOTS); };
    auto gt_slot = [&](int q) { return (int)((unsigned)(q - z0 + 3) % (unsigned)GT_SLOTS); };
    auto h_slot = [&](int q) { return (int)((unsigned)(q - z0 + 3) % (unsigned)H_SLOTS); };
    // D1Q3 weights: the D3Q27 weights of the isotropic stencils factor as W(cx) W(cy) W(cz)
    const R W0 = R(2.0 / 3.0), W1 = R(1.0 / 6.0);

    // phi plane q into its ring slot (zero outside the box); asynchronous or direct
    auto load_phi_plane = [&](int q, bool async) {
        bool zok = true;
        const int wz = zwrap(q, zok);
        R* dst = phis + phi_slot(q) * R3N;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const int n = t + k * NT;
            if (n < R3N) {
                const bool ok = zok && r3_ok[k];
                const int g = wz * plane + r3_off[k];
                if (async && ok) {
                    cp_async<sizeof(SP)>(dst + n, p.pin + g);
                } else {
                    dst[n] = ok ? CP::ld(p.pin, g, R(1)) : R(0);
                }
            }
        }
    };
    // Separable phase-field stencils.  The isotropic gradient, Laplacian and
    // divergence of the reference (lb_cuda_auxfields_module.f90:72-135,
    // 1136-1157) use the D3Q27 weights w = W(cx) W(cy) W(cz), W(0) = 2/3,
    // W(+-1) = 1/6, so each is a product of 1-D operators: S = W-weighted sum,
    // D = W(1) x central difference.  Per plane the theta region keeps the
    // in-plane partials S_x S_y phi, D_x S_y phi, S_x D_y phi; the z operator
    // then combines three planes of them at the same (x, y):
    //   grad phi = 3 (S_z D_x S_y, S_z S_x D_y, D_z S_x S_y) phi
    //   lap phi  = 6 (S_z S_x S_y phi - phi)
    // and likewise div theta = 3 (S_z (D_x S_y th_x + S_x D_y th_y) + D_z S_x S_y th_z)
    // from in-plane partials of theta on the collision region.  The same sums
    // as the reference, in another order.  The in-plane smoothings are kept
    // relative to the node's own value (S_x S_y f - f_c, from the differences
    // f - f_c), and z differences are taken of those and of the centre values
    // separately: a z difference of two smoothed planes of values near 1
    // would lose the digits that a small gradient needs in FP32.

    // in-plane partials of phi(q) on this thread's theta-region nodes
    auto planar_plane = [&](int q) {
        const R* f = phis + phi_slot(q) * R3N;
        R* sx = sxys + sxy_slot(q) * R2N;
        R* gg = gxys + gxy_slot(q) * (2 * R2N);
#pragma unroll
        for (int k = 0; k < KTH; ++k) {
            const int n = t + k * NTH;
            if (t >= NTH || n >= R2N) continue;
            int hx, hy;
            r2_node(n, hx, hy);
            const int m = hy * R2X + hx;
            const R* c = f + (hy + 1) * R3X + (hx + 1);
            const R fc = c[0];
            R sr[3], dr_[3];
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                const R a = c[(r - 1) * R3X - 1], b = c[(r - 1) * R3X], e = c[(r - 1) * R3X + 1];
                sr[r] = W1 * ((a - fc) + (e - fc)) + W0 * (b - fc);
                dr_[r] = e - a;
            }
            sx[m] = W1 * (sr[0] + sr[2]) + W0 * sr[1];  // S_x S_y phi - phi_c
            gg[m] = W1 * (W1 * (dr_[0] + dr_[2]) + W0 * dr_[1]);
            gg[R2N + m] = W1 * (sr[2] - sr[0]);
        }
    };
    // theta = phi(1-phi) n on the theta region and g~ = n |g| on the collision
    // region of plane q (compute_norm_interface, lb_cuda_auxfields_module.f90:72-119)
    // from the partials of planes q-1..q+1
    // Obstacles: isfluid of this thread's theta nodes in plane q (0 outside
    // the box), loaded a plane before theta_plane uses it so the load's
    // latency passes behind the pull phase; a load at the point of use
    // stalled every theta warp at once (a box with obstacles stepped 33 %
    // slower than without, with no solid node)
    auto theta_isf = [&](int q, int8_t (&s)[KTH]) {
        bool zk = true;
        const int wz = zwrap(q, zk);
#pragma unroll
        for (int k = 0; k < KTH; ++k) {
            const int n = t + k * NTH;
            s[k] = (t < NTH && n < R2N && zk && r2_ok[k]) ? p.isf[wz * plane + r2_off[k]] : int8_t(0);
        }
    };
    int8_t th_isf[KTH];
#pragma unroll
    for (int k = 0; k < KTH; ++k) th_isf[k] = 1;
    auto theta_plane = [&](int q) {
        bool zok = true;
        const int wz = zwrap(q, zok);
        const R* f0 = phis + phi_slot(q - 1) * R3N;
        const R* f1 = phis + phi_slot(q) * R3N;
        const R* f2 = phis + phi_slot(q + 1) * R3N;
        const R* s0 = sxys + sxy_slot(q - 1) * R2N;
        const R* s2 = sxys + sxy_slot(q + 1) * R2N;
        const R* g0 = gxys + gxy_slot(q - 1) * (2 * R2N);
        const R* g1 = gxys + gxy_slot(q) * (2 * R2N);
        const R* g2 = gxys + gxy_slot(q + 1) * (2 * R2N);
        R* th = ths + th_slot(q) * (3 * R2N);
        R* gt = gts + gt_slot(q) * (3 * R1N);
#pragma unroll
        for (int k = 0; k < KTH; ++k) {
            const int n = t + k * NTH;
            if (t >= NTH || n >= R2N) continue;
            int hx, hy;
            r2_node(n, hx, hy);
            const int m = hy * R2X + hx;
            bool fluid = zok && r2_ok[k];
            if (fluid && obs) fluid = (th_isf[k] == 1 || th_isf[k] == -1);
            R th0 = 0, th1 = 0, th2 = 0, gv0 = 0, gv1 = 0, gv2 = 0;
            if (fluid) {
                const R gx = R(3) * (W1 * (g0[m] + g2[m]) + W0 * g1[m]);
                const R gy = R(3) * (W1 * (g0[R2N + m] + g2[R2N + m]) + W0 * g1[R2N + m]);
                const int c3 = (hy + 1) * R3X + (hx + 1);
                const R gz = R(3) * W1 * ((s2[m] - s0[m]) + (f2[c3] - f0[c3]));
                const R mg = sqrt_a<R>(gx * gx + gy * gy + gz * gz);
                const R rden = rcp<R>(mg + R(1.0e-9));
                const R nxv = gx * rden, nyv = gy * rden, nzv = gz * rden;
                const R ph = f1[c3];
                const R pp = ph * (R(1) - ph);
                th0 = pp * nxv; th1 = pp * nyv; th2 = pp * nzv;
                gv0 = nxv * mg; gv1 = nyv * mg; gv2 = nzv * mg;
            }
            th[0 * R2N + m] = th0;
            th[1 * R2N + m] = th1;
            th[2 * R2N + m] = th2;
            if (hx >= 1 && hx <= R2X - 2 && hy >= 1 && hy <= R2Y - 2) {
                const int n1 = (hy - 1) * R1X + (hx - 1);
                gt[0 * R1N + n1] = gv0;
                gt[1 * R1N + n1] = gv1;
                gt[2 * R1N + n1] = gv2;
            }
        }
    };
    // in-plane partials of theta(q) at this thread's collision nodes:
    // D_x S_y th_x + S_x D_y th_y and S_x S_y th_z
    auto theta_partials = [&](int q) {
        const R* th = ths + th_slot(q) * (3 * R2N);
        R* h = hs + h_slot(q) * (3 * R1N);
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const int node = k ? nodeB : nodeA;
            if (node < 0) continue;
            const int hx = node % R1X, hy = node / R1X;
            const R* c = th + (hy + 1) * R2X + (hx + 1);
            const R zc = c[2 * R2N];
            R dx[3], sy[3], sz[3];
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                const int o = (r - 1) * R2X;
                dx[r] = c[o + 1] - c[o - 1];
                sy[r] = W1 * (c[R2N + o - 1] + c[R2N + o + 1]) + W0 * c[R2N + o];
                sz[r] = W1 * ((c[2 * R2N + o - 1] - zc) + (c[2 * R2N + o + 1] - zc)) + W0 * (c[2 * R2N + o] - zc);
            }
            h[node] = W1 * (W1 * (dx[0] + dx[2]) + W0 * dx[1]) + W1 * (sy[2] - sy[0]);
            h[R1N + node] = W1 * (sz[0] + sz[2]) + W0 * sz[1];  // S_x S_y th_z - th_z,c
            h[2 * R1N + node] = zc;
        }
    };

    // stored moments, u_old and isfluid of one collision node, not yet decoded.
    // The tile-interior node's are loaded one plane ahead, at the end of the
    // collision phase of the plane before (after its collisions), so their
    // latency passes behind its barrier and the pull phase; the ring nodes
    // load theirs at the point of use.
    using LY = Layout<S>;
    struct NodeRaw {
        S m[10];      // with 16-bit storage only m[4..9] (Pi - u u)
        float v32[4];  // P, u, v, w of the 16-bit formats
        S uo[3];
        int8_t isf;
    };
    auto fetch = [&](int gi, NodeRaw& r) {
        if constexpr (LY::split) {
#pragma unroll
            for (int f = 0; f < 4; ++f) r.v32[f] = __ldg(p.pres_in + f * N + gi);
#pragma unroll
            for (int f = 4; f < 10; ++f) r.m[f] = CD::raw(p.min + LY::off(f, N), gi);
        } else {
#pragma unroll
            for (int f = 0; f < 10; ++f) r.m[f] = CD::raw(p.min + f * N, gi);
        }
        if (dr) {
#pragma unroll
            for (int f = 0; f < 3; ++f) r.uo[f] = CD::raw(p.uin + f * N, gi);
        }
        if (obs) r.isf = p.isf[gi];
    };
    NodeRaw nxt;
    auto prefetch_a = [&](int q) {
        bool zk = true;
        const int wz = zwrap(q, zk);
        if (zk && okA) fetch(wz * plane + offA, nxt);
    };

    // accumulators of the raw moments {sum g, sum g c, sum g c c} for output planes
    // q-1 (am), q (a0), q+1 (ap); A2[i] = (am[i], a0[i]), one pair, accumulated
    // with packed instructions from the population pairs (cz = -1, 0).  With
    // the packed x and y transforms of the collision: 2.9 % fewer
    // instructions, 1.8 % per step at 256^3
    using PA = typename PK<R>::T;
    PA A2[10];
    R ap[10];
#pragma unroll
    for (int i = 0; i < 10; ++i) {
        A2[i] = PK<R>::mk(R(0), R(0));
        ap[i] = R(0);
    }

    // ---- prologue: phi(z0-3..z0+2), theta(z0-2..z0) ----
    if constexpr (TC) {
        // partials of phi(z0-3..z0+1), theta(z0-2..z0), theta partials (z0-2, z0-1)
        // (theta reads only this thread's own partials; the partial slots are
        // reused as soon as a theta plane no longer needs them)
        for (int q = z0 - 3; q <= z0 + 1; ++q) load_phi_plane(q, false);
        __syncthreads();
        planar_plane(z0 - 3);
        planar_plane(z0 - 2);
        planar_plane(z0 - 1);
        if (obs) theta_isf(z0 - 2, th_isf);
        theta_plane(z0 - 2);
        planar_plane(z0);
        if (obs) theta_isf(z0 - 1, th_isf);
        theta_plane(z0 - 1);
        planar_plane(z0 + 1);
        __syncthreads();
        theta_partials(z0 - 2);
        theta_partials(z0 - 1);
        __syncthreads();
        if (obs) theta_isf(z0, th_isf);
        theta_plane(z0);               // into the slot of theta(z0-2)
        if (obs) theta_isf(z0 + 1, th_isf);  // for the loop's first theta plane
        load_phi_plane(z0 + 2, true);  // into the slot of phi(z0-3), no longer read
    }
    prefetch_a(z0 - 1);
    cp_async_wait_all();
    __syncthreads();
    // theta partials of the first loop plane; the loop computes each later
    // plane's in the pull phase of the plane before
    if constexpr (TC) theta_partials(z0);

    for (int q = z0 - 1; q <= z1; ++q) {
        bool zok = true;
        const int wz = zwrap(q, zok);
        const int zoff = wz * plane;
        const bool q_inner = (q >= z0) && (q < z1);

        // ================= phase 1 =================
        // partials of phi(q+3), then theta(q+2) from the partials of planes
        // q+1..q+3 (this thread's own nodes)
        if constexpr (TC) {
            planar_plane(q + 3);
            theta_plane(q + 2);
        }

        R c4m = R(0), c40 = R(0), c4p = R(0);  // centre group of the interior node
        // unrolled: the interior node's copy of the collision reads the
        // prefetched registers in place (one shared copy of the loop body
        // costs moves and selects between the two sources: 6 % more
        // instructions and 3.6 % more time on the FP32 Laplace step)
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const int node = k ? nodeB : nodeA;
            if (node < 0) continue;
            const bool inb = zok && (k ? okB : okA);
            const int gi = zoff + (k ? offB : offA);
            NodeRaw cur;
            if (k == 0) cur = nxt;
            else if (inb) fetch(gi, cur);
            int isf = 1;
            if (inb && obs) isf = cur.isf;
            const bool live = inb && (isf != 0);
            const bool interior = (k == 0) && out_ok && q_inner;
            R fpop[27];
            bool ring_done = false;  // a ring node's populations are stored already
            R sP = 0, spxx = 0, spyy = 0, spzz = 0, spxy = 0, spxz = 0, spyz = 0, som = 0;
            if (live) {
                R P, u, v, w, pxx, pyy, pzz, pxy, pxz, pyz;
                if constexpr (LY::split) {
                    P = (R)cur.v32[0]; u = (R)cur.v32[1]; v = (R)cur.v32[2]; w = (R)cur.v32[3];
                } else {
                    P = CD::dec(cur.m[0], p.inv_scale[0]);
                    u = CD::dec(cur.m[1], p.inv_scale[1]);
                    v = CD::dec(cur.m[2], p.inv_scale[2]);
                    w = CD::dec(cur.m[3], p.inv_scale[3]);
                }
                pxx = CD::dec(cur.m[4], p.inv_scale[4]);
                pyy = CD::dec(cur.m[5], p.inv_scale[5]);
                pzz = CD::dec(cur.m[6], p.inv_scale[6]);
                pxy = CD::dec(cur.m[7], p.inv_scale[7]);
                pxz = CD::dec(cur.m[8], p.inv_scale[8]);
                pyz = CD::dec(cur.m[9], p.inv_scale[9]);
                if constexpr (CD::scaled) {
                    // 16-bit storage keeps Pi - u u, the deviation from equilibrium
                    pxx += u * u; pyy += v * v; pzz += w * w;
                    pxy += u * v; pxz += u * w; pyz += v * w;
                }
                R phi = 0, lap = 0, divt = 0, gfx = 0, gfy = 0, gfz = 0;
                R phi_u = 0;         // phi before the mass correction
                bool stale = false;  // the collision reads phi_u (see below)
                if constexpr (TC) {
                    const int hx = node % R1X, hy = node / R1X;
                    const int c2 = (hy + 1) * R2X + (hx + 1);
                    const int c3 = (hy + 2) * R3X + (hx + 2);
                    phi = phis[phi_slot(q) * R3N + c3];
                    const R phm = phis[phi_slot(q - 1) * R3N + c3], php = phis[phi_slot(q + 1) * R3N + c3];
                    const R* sm = sxys + sxy_slot(q - 1) * R2N;
                    const R* s0 = sxys + sxy_slot(q) * R2N;
                    const R* sp = sxys + sxy_slot(q + 1) * R2N;
                    // S_z S_x S_y phi - phi, with W0 - 1 = -2 W1
                    lap = R(6) * (W1 * (sm[c2] + sp[c2]) + W0 * s0[c2] + W1 * ((phm - phi) + (php - phi)));
                    const R* hm = hs + h_slot(q - 1) * (3 * R1N);
                    const R* h0 = hs + h_slot(q) * (3 * R1N);
                    const R* hp = hs + h_slot(q + 1) * (3 * R1N);
                    divt = R(3) * ((W1 * (hm[node] + hp[node]) + W0 * h0[node]) +
                                   W1 * ((hp[R1N + node] - hm[R1N + node]) + (hp[2 * R1N + node] - hm[2 * R1N + node])));
                    const R* g1 = gts + gt_slot(q) * (3 * R1N);
                    gfx = g1[0 * R1N + node];
                    gfy = g1[1 * R1N + node];
                    gfz = g1[2 * R1N + node];
                    if constexpr (OBS) {
                        // from here on the input phi after the mass correction (the
                        // gradient, theta and Laplacian above are compute_norm's, from
                        // the uncorrected phi)
                        if (do_mcorr) {
                            phi_u = phi;
                            phi = (R)mass_corrected<SP>((double)phi, mcorr);
                            // a node reached across a periodic face is, in the
                            // reference's fused kernel, a halo copy: its moments and
                            // forces were exchanged after the moments kernel (corrected
                            // phi), its phi before the correction
                            stale = phi != phi_u && ((k ? wrapB : wrapA) || q < 0 || q >= nz);
                        }
                    }
                }
                // ---- moments prologue: lb_cuda_moments_module.f90:104-339 ----
                R inv = R(1), mask = R(0), fxv, fyv, fzv;
                if constexpr (TC) mask = R(4) * phi * (R(1) - phi);
                if (dr) {
                    const R rhophi = p.rho_r * phi + (R(1) - phi) * p.rho_b;
                    inv = rcp<R>(rhophi);
                    fxv = rhophi * p.fx; fyv = rhophi * p.fy; fzv = rhophi * p.fz;
                } else {
                    fxv = p.fx; fyv = p.fy; fzv = p.fz;
                }
                R grx = 0, gry = 0, grz = 0, cv = 0, omega;
                R visc_l = p.visc1;  // local viscosity (mixture with two components)
                if constexpr (TC) {
                    const R chem = R(4) * p.beta * phi * (phi - R(1)) * (phi - R(0.5)) - p.kapp * lap;
                    fxv += chem * gfx;
                    fyv += chem * gfy;
                    fzv += chem * gfz;
                    if constexpr (REP) {
                        // REPULSIVE_FLUX (lb_cuda_moments_module.f90:148-160): rho_phi F_rep,
                        // each component capped at 1e-3, times rho_phi
                        const R rh = dr ? p.rho_r * phi + (R(1) - phi) * p.rho_b : R(1);
                        const R cap = R(1.0e-3);
                        R t0 = p.rep[gi] * rh, t1 = p.rep[N + gi] * rh, t2 = p.rep[2 * N + gi] * rh;
                        t0 = t0 > cap ? cap : (t0 < -cap ? -cap : t0);
                        t1 = t1 > cap ? cap : (t1 < -cap ? -cap : t1);
                        t2 = t2 > cap ? cap : (t2 < -cap ? -cap : t2);
                        fxv += t0 * rh;
                        fyv += t1 * rh;
                        fzv += t2 * rh;
                    }
                }
                if (dr) {
                    const R drho = p.rho_r - p.rho_b;
                    grx = drho * gfx; gry = drho * gfy; grz = drho * gfz;
                    const R mp = mask * P * cssq;
                    fxv -= mp * grx; fyv -= mp * gry; fzv -= mp * grz;
                }
                R tfx = fxv, tfy = fyv, tfz = fzv;
                if (dr) {
                    const R uo = CD::dec(cur.uo[0], p.inv_scale[F_UOLD + 0]);
                    const R vo = CD::dec(cur.uo[1], p.inv_scale[F_UOLD + 1]);
                    const R wo = CD::dec(cur.uo[2], p.inv_scale[F_UOLD + 2]);
                    const R qxx = pxx - uo * uo, qyy = pyy - vo * vo, qzz = pzz - wo * wo;
                    const R qxy = pxy - uo * vo, qxz = pxz - uo * wo, qyz = pyz - vo * wo;
                    const R visc = (p.rho_r * p.visc1 * phi + (R(1) - phi) * p.visc2 * p.rho_b) * inv;
                    visc_l = visc;
                    omega = rcp<R>(visc * R(3) + R(0.5));
                    // mask * visc / (tau cs^2), with 1/tau = omega
                    cv = mask * visc * omega * R(3);
                    fxv -= cv * (qxx * grx + qxy * gry + qxz * grz);
                    fyv -= cv * (qyy * gry + qxy * grx + qyz * grz);
                    fzv -= cv * (qzz * grz + qxz * grx + qyz * gry);
                    const R tmp = -p.sharp_c * divt;
                    u += R(0.5) * fxv * inv;
                    v += R(0.5) * fyv * inv;
                    w += R(0.5) * fzv * inv;
                    const R dd = (p.rho_r - p.rho_b) * (p.tau_diff * lap + tmp);
                    const R den = rcp<R>(R(1) - R(0.5) * dd * inv);
                    u *= den; v *= den; w *= den;
                    tfx -= dd * u; tfy -= dd * v; tfz -= dd * w;
                    fxv -= dd * u; fyv -= dd * v; fzv -= dd * w;
                } else {
                    u += R(0.5) * fxv * inv;
                    v += R(0.5) * fyv * inv;
                    w += R(0.5) * fzv * inv;
                    if constexpr (TC) {
                        const R visc = (p.rho_r * p.visc1 * phi + (R(1) - phi) * p.visc2 * p.rho_b) * inv;
                        visc_l = visc;
                        omega = rcp<R>(visc * R(3) + R(0.5));
                    } else {
                        omega = p.omega;
                    }
                }
                pxx += fxv * u * inv;
                pyy += fyv * v * inv;
                pzz += fzv * w * inv;
                pxy += R(0.5) * (fyv * u + fxv * v) * inv;
                pxz += R(0.5) * (fzv * u + fxv * w) * inv;
                pyz += R(0.5) * (fzv * v + fyv * w) * inv;
                if (dr) {
                    const R qxx = pxx - u * u, qyy = pyy - v * v, qzz = pzz - w * w;
                    const R qxy = pxy - u * v, qxz = pxz - u * w, qyz = pyz - v * w;
                    tfx -= cv * (qxx * grx + qxy * gry + qxz * grz);
                    tfy -= cv * (qyy * gry + qxy * grx + qyz * grz);
                    tfz -= cv * (qzz * grz + qxz * grx + qyz * gry);
                }
                // ---- outputs of this node that leave the kernel ----
                if (interior) {
                    if (p.write_u) {
                        CD::st(p.uout + 0 * N, gi, u, p.scale[F_UOLD + 0]);
                        CD::st(p.uout + 1 * N, gi, v, p.scale[F_UOLD + 1]);
                        CD::st(p.uout + 2 * N, gi, w, p.scale[F_UOLD + 2]);
                    }
                    if constexpr (TC) {
                        // update_phifields: lb_cuda_update_phi_module.f90:77-93
                        const R phi_new = phi - u * R(0.5) * gfx - v * R(0.5) * gfy - w * R(0.5) * gfz +
                                          p.tau_diff * lap - p.sharp_c * divt;
                        CP::st(p.pout, gi, phi_new, p.scale[F_PHI]);
                    }
                }
                if constexpr (OBS && TC) {
                    if (stale) {
                        // density and viscosity of the collision from the halo copy's
                        // uncorrected phi (lb_cuda_fused_module.f90:590-620)
                        const R rh = dr ? p.rho_r * phi_u + (R(1) - phi_u) * p.rho_b : R(1);
                        if (dr) inv = rcp<R>(rh);
                        visc_l = (p.rho_r * p.visc1 * phi_u + (R(1) - phi_u) * p.visc2 * p.rho_b) * inv;
                        omega = rcp<R>(visc_l * R(3) + R(0.5));
                    }
                }
                // ---- collision: lb_cuda_fused_module.f90:531-713 ----
                const R Xn = pxx - u * u, Yn = pyy - v * v, Zn = pzz - w * w;
                const R XYn = pxy - u * v, XZn = pxz - u * w, YZn = pyz - v * w;
                const R Fx = tfx * inv, Fy = tfy * inv, Fz = tfz * inv;
                if (p.smag) {
                    // SMAGORINSKI (lb_cuda_fused_module.f90:609-616): relaxation time from the
                    // Frobenius norm of the non-equilibrium stress; the moments prologue above
                    // keeps the molecular one, as the reference's moments kernel does
                    const R QQ = Xn * Xn + Yn * Yn + Zn * Zn + R(2) * (XYn * XYn + XZn * XZn + YZn * YZn);
                    const R v3 = R(3) * visc_l;
                    const R tau = R(0.5) + R(1.0 / 6.0) * (v3 + sqrt_a<R>(v3 * v3 + R(SMAG_C) * sqrt_a<R>(R(2) * QQ) * inv));
                    omega = rcp<R>(tau);
                }
                sP = P;
                spxx = Xn; spyy = Yn; spzz = Zn; spxy = XYn; spxz = XZn; spyz = YZn; som = omega;
                const R om1 = R(1) - omega;
                const R m0 = P;
                const R mx = u + R(0.5) * Fx, my = v + R(0.5) * Fy, mz = w + R(0.5) * Fz;
                const R mxx = u * u + om1 * Xn + u * Fx;
                const R myy = v * v + om1 * Yn + v * Fy;
                const R mzz = w * w + om1 * Zn + w * Fz;
                const R mxy = u * v + om1 * XYn + R(0.5) * (u * Fy + v * Fx);
                const R mxz = u * w + om1 * XZn + R(0.5) * (u * Fz + w * Fx);
                const R myz = v * w + om1 * YZn + R(0.5) * (v * Fz + w * Fy);
                if constexpr (LAT == 27) {
                    R M[3][3][3];
                    M[0][0][0] = m0;
                    M[1][0][0] = mx; M[0][1][0] = my; M[0][0][1] = mz;
                    M[2][0][0] = mxx; M[0][2][0] = myy; M[0][0][2] = mzz;
                    M[1][1][0] = mxy; M[1][0][1] = mxz; M[0][1][1] = myz;
                    if constexpr (HO) {
                        const R X = Xn, Y = Yn, Z = Zn, XY = XYn, XZ = XZn, YZ = YZn;
                        const R u2 = u * u, v2 = v * v, w2 = w * w;
                        // rows 10..26 of the reference (lb_cuda_fused_module.f90:667-703)
                        M[2][1][0] = u2 * v + om1 * (R(2) * XY * u + X * v);
                        M[2][0][1] = u2 * w + om1 * (R(2) * XZ * u + X * w);
                        M[1][2][0] = u * v2 + om1 * (Y * u + R(2) * XY * v);
                        M[1][0][2] = u * w2 + om1 * (Z * u + R(2) * XZ * w);
                        M[0][1][2] = v * w2 + om1 * (Z * v + R(2) * YZ * w);
                        M[0][2][1] = v2 * w + om1 * (R(2) * YZ * v + Y * w);
                        M[1][1][1] = u * v * w + om1 * (YZ * u + XZ * v + XY * w);
                        M[2][2][0] = u2 * v2 + om1 * (Y * u2 + R(2) * v * (R(3) * XY * u + X * v));
                        M[2][0][2] = u2 * w2 + om1 * (Z * u2 + R(2) * w * (R(3) * XZ * u + X * w));
                        M[0][2][2] = v2 * w2 + om1 * (Z * v2 + R(2) * w * (R(3) * YZ * v + Y * w));
                        M[1][1][2] = u * v * w2 + om1 * (Z * u * v + w * (R(3) * YZ * u + R(3) * XZ * v + R(2) * XY * w));
                        M[1][2][1] = u * v2 * w +
                                     om1 * (R(2) * YZ * u * v + XZ * v2 + R(2) * Y * u * w + R(4) * XY * v * w);
                        M[2][1][1] = u2 * v * w +
                                     om1 * (YZ * u2 + R(2) * XZ * u * v + R(4) * XY * u * w + R(2) * X * v * w);
                        M[2][1][2] = u2 * v * w2 + om1 * (Z * u2 * v + R(3) * w * (YZ * u2 + R(2) * XZ * u * v +
                                                                                 R(2) * XY * u * w + X * v * w));
                        M[2][2][1] = u2 * v2 * w + om1 * (R(2) * u * v * (YZ * u + XZ * v) + R(2) * Y * u2 * w +
                                                          v * (R(10) * XY * u + R(3) * X * v) * w);
                        M[1][2][2] = u * v2 * w2 + om1 * (Z * u * v2 + R(3) * w * (R(2) * YZ * u * v + XZ * v2 +
                                                                                  Y * u * w + R(2) * XY * v * w));
                        M[2][2][2] = u2 * v2 * w2 +
                                     om1 * (Z * u2 * v2 + w * (R(6) * u * v * (YZ * u + XZ * v) + R(3) * Y * u2 * w +
                                                               R(2) * v * (R(7) * XY * u + R(2) * X * v) * w));
                    } else {
                        M[2][1][0] = M[2][0][1] = M[1][2][0] = M[1][0][2] = M[0][1][2] = M[0][2][1] = M[1][1][1] = R(0);
                        M[2][2][0] = M[2][0][2] = M[0][2][2] = M[1][1][2] = M[1][2][1] = M[2][1][1] = R(0);
                        M[2][1][2] = M[2][2][1] = M[1][2][2] = M[2][2][2] = R(0);
                    }
                    if (k == 1 && ring_col) {
                        // column ring node: the x transform at cx = ring_dir only,
                        // the same operations as the full transform for that value
                        R T[3][3];  // [b][c]
#pragma unroll
                        for (int b = 0; b < 3; ++b)
#pragma unroll
                            for (int c = 0; c < 3; ++c) {
                                const R sv = fmaf_t(M[0][b][c], R(1.0 / 6.0), R(0.5) * M[2][b][c]);
                                T[b][c] = sv + ring_dir * (R(0.5) * M[1][b][c]);
                            }
                        R Y[3][3];  // [b][c]
#pragma unroll
                        for (int c = 0; c < 3; ++c) d1q3_inv<R>(T[0][c], T[1][c], T[2][c], Y[0][c], Y[1][c], Y[2][c]);
                        const int xg = ring_dir > R(0) ? 2 : 0;
#pragma unroll
                        for (int b = 0; b < 3; ++b) {
                            R vm, v0, vp;
                            d1q3_inv<R>(Y[b][0], Y[b][1], Y[b][2], vm, v0, vp);
                            R2 v2;
                            v2.x = vm;
                            v2.y = v0;
                            pops2[gslot(3 * b + xg) * R1N + node] = v2;
                            pops1[gslot(3 * b + xg) * R1N + node] = vp;
                        }
                        ring_done = true;
                    } else {
                        // the x (a) and y (b) transforms packed over the pair
                        // c = 0, 1 of the z coefficient index, c = 2 alone; both
                        // take the second coefficient negated, carried by the
                        // sign (-1)^([a==2] + [b==2]) of the coefficients (exact:
                        // the values are those of the scalar transforms)
                        using PT = typename PK<R>::T;
                        PT P[3][3];
                        R Q[3][3];
#pragma unroll
                        for (int a = 0; a < 3; ++a)
#pragma unroll
                            for (int b = 0; b < 3; ++b) {
                                const R sg = ((a == 2) != (b == 2)) ? R(-1) : R(1);
                                P[a][b] = PK<R>::mk(sg * M[a][b][0], sg * M[a][b][1]);
                                Q[a][b] = sg * M[a][b][2];
                            }
                        // x transform: TP/TQ[a'][b], with the sign (-1)^[b==2]
                        PT TP[3][3];
                        R TQ[3][3];
#pragma unroll
                        for (int b = 0; b < 3; ++b) {
                            d1q3n2<R>(P[0][b], P[1][b], P[2][b], TP[0][b], TP[1][b], TP[2][b]);
                            d1q3n<R>(Q[0][b], Q[1][b], Q[2][b], TQ[0][b], TQ[1][b], TQ[2][b]);
                        }
                        if (k == 1) {
                            // row ring node: the y transform at cy = ring_dir only
                            const int yg = ring_dir > R(0) ? 2 : 0;
#pragma unroll
                            for (int a = 0; a < 3; ++a) {
                                R Y[3];
#pragma unroll
                                for (int c = 0; c < 3; ++c) {
                                    const R t0 = c == 0 ? TP[a][0].x : (c == 1 ? TP[a][0].y : TQ[a][0]);
                                    const R t1 = c == 0 ? TP[a][1].x : (c == 1 ? TP[a][1].y : TQ[a][1]);
                                    const R t2n = c == 0 ? TP[a][2].x : (c == 1 ? TP[a][2].y : TQ[a][2]);
                                    const R sv = fmaf_t(t0, R(1.0 / 6.0), R(-0.5) * t2n);
                                    Y[c] = sv + ring_dir * (R(0.5) * t1);
                                }
                                R vm, v0, vp;
                                d1q3_inv<R>(Y[0], Y[1], Y[2], vm, v0, vp);
                                R2 v2;
                                v2.x = vm;
                                v2.y = v0;
                                pops2[gslot(3 * yg + a) * R1N + node] = v2;
                                pops1[gslot(3 * yg + a) * R1N + node] = vp;
                            }
                            ring_done = true;
                        } else {
                            // y transform: MP/MQ[a][b'], then the z transform scalar
                            PT MP[3][3];
                            R MQ[3][3];
#pragma unroll
                            for (int a = 0; a < 3; ++a) {
                                d1q3n2<R>(TP[a][0], TP[a][1], TP[a][2], MP[a][0], MP[a][1], MP[a][2]);
                                d1q3n<R>(TQ[a][0], TQ[a][1], TQ[a][2], MQ[a][0], MQ[a][1], MQ[a][2]);
                            }
#pragma unroll
                            for (int a = 0; a < 3; ++a)
#pragma unroll
                                for (int b = 0; b < 3; ++b) {
                                    R vm, v0, vp;
                                    d1q3_inv<R>(MP[a][b].x, MP[a][b].y, MQ[a][b], vm, v0, vp);
                                    fpop[LINK(a - 1, b - 1, -1)] = vm;
                                    fpop[LINK(a - 1, b - 1, 0)] = v0;
                                    fpop[LINK(a - 1, b - 1, 1)] = vp;
                                }
                        }
                    }
                } else {
                    // D3Q19 / D3Q15: the second-order expansion link by link (D3Q27 indices)
                    const R base = m0 - R(1.5) * (mxx + myy + mzz);
#pragma unroll
                    for (int l = 0; l < 27; ++l) {
                        if (!IN<LAT>(l)) continue;
                        const int cx = EX(l), cy = EY(l), cz = EZ(l);
                        R s = base;
                        s += R(3) * (R(cx) * mx + R(cy) * my + R(cz) * mz);
                        s += R(4.5) * (R(cx * cx) * mxx + R(cy * cy) * myy + R(cz * cz) * mzz);
                        s += R(9) * (R(cx * cy) * mxy + R(cx * cz) * mxz + R(cy * cz) * myz);
                        fpop[l] = R(WL<LAT>(l)) * s;
                    }
                }
            } else {
#pragma unroll
                for (int l = 0; l < 27; ++l) fpop[l] = R(0);
            }
#pragma unroll
            for (int g = 0; g < 9; ++g) {
                if (ring_done) break;
                const int cx = g % 3 - 1, cy = g / 3 - 1;
                // links the lattice lacks carry 0 (D3Q19: no corners, D3Q15: no edges)
                R2 v;
                v.x = IN<LAT>(LINK(cx, cy, -1)) ? fpop[LINK(cx, cy, -1)] : R(0);
                v.y = IN<LAT>(LINK(cx, cy, 0)) ? fpop[LINK(cx, cy, 0)] : R(0);
                const R vp = IN<LAT>(LINK(cx, cy, 1)) ? fpop[LINK(cx, cy, 1)] : R(0);
                if (g == 4) {
                    // the centre group: only the interior node's own output reads it
                    if (k == 0) {
                        c4m = v.x;
                        c40 = v.y;
                        c4p = vp;
                    }
                    continue;
                }
                pops2[gslot(g) * R1N + node] = v;
                pops1[gslot(g) * R1N + node] = vp;
            }

            // ---- obstacle bounce-back: lb_cuda_boundary_module.f90:162-199 ----
            if (interior && obs && isf == -1) {
                const R om1 = R(1) - som;
                // neighbour x / y coordinates of the output node, computed here:
                // held in registers through the whole sweep they cost the
                // obstacle step 4 registers at its limit of 128 and 10.7 % of
                // its time on a box with obstacles
                int nbx[3], nby[3];
                bool nbx_ok[3], nby_ok[3];
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    bool okx = true, oky = true;
                    nbx[d] = wrap_coord(ox + d - 1, nx, p.pbx, okx);
                    nby[d] = wrap_coord(oy + d - 1, ny, p.pby, oky);
                    nbx_ok[d] = okx;
                    nby_ok[d] = oky;
                }
#pragma unroll
                for (int l = 1; l < 27; ++l) {
                    if (!IN<LAT>(l)) continue;
                    const int cx = EX(l), cy = EY(l), cz = EZ(l);
                    const int ix = 1 - cx, iy = 1 - cy;
                    bool zk = true;
                    const int zz = zwrap(q - cz, zk);
                    int s = 1;
                    if (nbx_ok[ix] && nby_ok[iy] && zk) s = p.isf[zz * plane + nby[iy] * nx + nbx[ix]];
                    if (s != 0) continue;
                    const R wl = R(WL<LAT>(l));
                    const R dx = R(cx), dy = R(cy), dz = R(cz);
                    const R fneq = wl * R(4.5) *
                                   ((dx * dx - cssq) * spxx + (dy * dy - cssq) * spyy + (dz * dz - cssq) * spzz +
                                    R(2) * (dx * dy) * spxy + R(2) * (dx * dz) * spxz + R(2) * (dy * dz) * spyz);
                    const R fp = wl * sP + om1 * fneq;
                    A2[0].y += fp;
                    A2[1].y += fp * dx; A2[2].y += fp * dy; A2[3].y += fp * dz;
                    A2[4].y += fp * (dx * dx); A2[5].y += fp * (dy * dy); A2[6].y += fp * (dz * dz);
                    A2[7].y += fp * (dx * dy); A2[8].y += fp * (dx * dz); A2[9].y += fp * (dy * dz);
                }
            }
        }
        // the interior node's fields of plane q+1, issued before the barrier
        // rather than after it: 0.9 % per step at 256^3
        prefetch_a(q + 1);
        __syncthreads();

        // ================= phase 2 =================
        // the slot of phi(q-1) was last read in phase 1
        if constexpr (TC) load_phi_plane(q + 4, true);
        if (TC && obs) theta_isf(q + 3, th_isf);  // for theta(q+3), next plane
        // the theta partials of plane q+2 at this thread's collision nodes
        // (theta(q+2) is complete since the barrier after phase 1).  Here
        // rather than in phase 1 they fill the shorter pull phase and shorten
        // the collision phase, whose barrier waits for the ring collisions
        // (1.7 % per step at 256^3); before the pull rather than after it,
        // 0.3 % more
        if constexpr (TC) theta_partials(q + 2);

        // the three cz populations of every (cx, cy) group from node x - c:
        // cz = -1, 0 as one pair (packed sums), cz = +1 alone
        using PP = typename PK<R>::T;
        PP gp[3][3];  // [cy][cx]
        R gs[3][3];
#pragma unroll
        for (int yc = 0; yc < 3; ++yc)
#pragma unroll
            for (int xc = 0; xc < 3; ++xc) {
                const int g = 3 * yc + xc;
                if (g == 4) {
                    gp[yc][xc] = PK<R>::mk(c4m, c40);
                    gs[yc][xc] = c4p;
                    continue;
                }
                const int src = (ty + 1 - (yc - 1)) * R1X + (tx + 1 - (xc - 1));
                const R2 v = pops2[gslot(g) * R1N + src];
                gp[yc][xc] = PK<R>::mk(v.x, v.y);
                gs[yc][xc] = pops1[gslot(g) * R1N + src];
            }
        {
            using P = PK<R>;
            const PP m1 = P::mk(R(-1), R(-1));
            PP S0[3], S1[3], S2[3];
#pragma unroll
            for (int yc = 0; yc < 3; ++yc) {
                const PP* g = gp[yc];
                S0[yc] = P::add(P::add(g[0], g[1]), g[2]);
                S1[yc] = P::fma(g[0], m1, g[2]);
                S2[yc] = P::add(g[2], g[0]);
            }
            const PP Y00 = P::add(P::add(S0[0], S0[1]), S0[2]);
            const PP Y01 = P::fma(S0[0], m1, S0[2]);
            const PP Y02 = P::add(S0[2], S0[0]);
            const PP Y10 = P::add(P::add(S1[0], S1[1]), S1[2]);
            const PP Y11 = P::fma(S1[0], m1, S1[2]);
            const PP Y20 = P::add(P::add(S2[0], S2[1]), S2[2]);
            // accum_slice for cz = -1 (x) and 0 (y)
            const PP cz = P::mk(R(-1), R(0)), cz2 = P::mk(R(1), R(0));
            A2[0] = P::add(A2[0], Y00);
            A2[1] = P::add(A2[1], Y10);
            A2[2] = P::add(A2[2], Y01);
            A2[3] = P::fma(cz, Y00, A2[3]);
            A2[4] = P::add(A2[4], Y20);
            A2[5] = P::add(A2[5], Y02);
            A2[6] = P::fma(cz2, Y00, A2[6]);
            A2[7] = P::add(A2[7], Y11);
            A2[8] = P::fma(cz, Y10, A2[8]);
            A2[9] = P::fma(cz, Y01, A2[9]);
        }
        {
            R S0[3], S1[3], S2[3];
#pragma unroll
            for (int yc = 0; yc < 3; ++yc) {
                const R* g = gs[yc];
                S0[yc] = g[0] + g[1] + g[2];
                S1[yc] = g[2] - g[0];
                S2[yc] = g[2] + g[0];
            }
            const R Y00 = S0[0] + S0[1] + S0[2];
            const R Y01 = S0[2] - S0[0];
            const R Y02 = S0[2] + S0[0];
            const R Y10 = S1[0] + S1[1] + S1[2];
            const R Y11 = S1[2] - S1[0];
            const R Y20 = S2[0] + S2[1] + S2[2];
            accum_slice<R>(ap, R(1), Y00, Y01, Y02, Y10, Y11, Y20);
        }
        R am[10];
#pragma unroll
        for (int i = 0; i < 10; ++i) am[i] = A2[i].x;
        if (q - 1 >= z0 && out_ok) {
            const int go = (q - 1) * plane + out_off;
            const R third = am[0] * cssq;
            if constexpr (CD::scaled) {
                am[4] -= am[1] * am[1]; am[5] -= am[2] * am[2]; am[6] -= am[3] * am[3];
                am[7] -= am[1] * am[2]; am[8] -= am[1] * am[3]; am[9] -= am[2] * am[3];
            }
            if constexpr (LY::split) {
#pragma unroll
                for (int f = 0; f < 4; ++f) p.pres_out[f * N + go] = (float)am[f];
            } else {
#pragma unroll
                for (int f = 0; f < 4; ++f) CD::st(p.mout + f * N, go, am[f], p.scale[f]);
            }
            CD::st(p.mout + LY::off(4, N), go, am[4] - third, p.scale[4]);
            CD::st(p.mout + LY::off(5, N), go, am[5] - third, p.scale[5]);
            CD::st(p.mout + LY::off(6, N), go, am[6] - third, p.scale[6]);
            CD::st(p.mout + LY::off(7, N), go, am[7], p.scale[7]);
            CD::st(p.mout + LY::off(8, N), go, am[8], p.scale[8]);
            CD::st(p.mout + LY::off(9, N), go, am[9], p.scale[9]);
        }
#pragma unroll
        for (int i = 0; i < 10; ++i) {
            A2[i] = PK<R>::mk(A2[i].y, ap[i]);
            ap[i] = R(0);
        }
        cp_async_wait_all();
        __syncthreads();
    }
}

// CTAs per SM the kernel is compiled for: two of 256 threads, one of 512, one in FP64
template <typename R, int TYV> constexpr int step_min_blocks() { return (sizeof(R) == 8 || TYV > 8) ? 1 : 2; }

// Column-planes of the planes zlo .. zlo + nzr - 1 of a box for a tile of
// TYV rows, column index = by * gx + bx, plane fastest.
template <int TYV, typename F>
__device__ __forceinline__ void run_share(const int nx, const int nzr, const int zlo, long long s0, long long s1,
                                          F&& body) {
    const int gx = (nx + TX - 1) / TX;
    while (s0 < s1) {
        const long long col = s0 / nzr;
        const int z0 = (int)(s0 - col * nzr);
        const int z1 = (int)min((long long)nzr, z0 + (s1 - s0));
        body((int)(col % gx), (int)(col / gx), zlo + z0, zlo + z1);
        s0 += z1 - z0;
    }
}

// Single box.  zseg > 0: one CTA per (tile x, tile y, z segment of zseg
// planes).  zseg < 0: split columns -- CTA i < ncols advances planes [0, L)
// of column i and CTA ncols + i planes [L, nzr), L = -zseg: when the columns
// fill less than one wave of CTA slots, the long segments run in step on
// ncols SMs (their halo re-reads hit in L2) while the other SMs work through
// the short tails.  zseg = 0: persistent schedule -- the box's columns x planes are
// cut into gridDim.x equal contiguous shares (a share may end inside one
// column and continue at the bottom of the next), so every CTA does the same
// work and pays the pipeline fill of a segment start only once or twice.
// Both schedules are expressed as a range of column-planes walked by ONE call
// site of step_body, so the kernel holds a single compiled copy of the step:
// separately inlined copies may contract floating-point operations
// differently and give results that differ in the last bit.
template <int LAT, bool HO, bool TC, typename S, typename R, int TYV, bool REP = false, bool OBS = true>
__global__ void __launch_bounds__(TX * TYV, step_min_blocks<R, TYV>()) stream_kernel(const StepParams<S, R> p) {
    long long s0, s1;
    const int nzr = p.zhi - p.zlo;
    if (p.zseg < 0) {
        const int L = min(-p.zseg, nzr);
        const long long ncols = (long long)((p.nx + TX - 1) / TX) * ((p.ny + TYV - 1) / TYV);
        const bool head = blockIdx.x < ncols;
        const long long col = head ? blockIdx.x : blockIdx.x - ncols;
        s0 = col * nzr + (head ? 0 : L);
        s1 = col * nzr + (head ? L : nzr);
    } else if (p.zseg > 0) {
        const long long col = (long long)blockIdx.y * ((p.nx + TX - 1) / TX) + blockIdx.x;
        const int z0 = blockIdx.z * p.zseg;
        s0 = col * nzr + z0;
        s1 = s0 + min(p.zseg, nzr - z0);
    } else {
        const long long W = (long long)((p.nx + TX - 1) / TX) * ((p.ny + TYV - 1) / TYV) * nzr;
        const long long share = (W + gridDim.x - 1) / gridDim.x;
        s0 = (long long)blockIdx.x * share;
        s1 = min(W, s0 + share);
    }
    run_share<TYV>(p.nx, nzr, p.zlo, s0, s1,
                   [&](int bx, int by, int z0, int z1) { step_body<LAT, HO, TC, S, R, TYV, REP, OBS>(p, bx, by, z0, z1); });
}

// Many boxes in one launch: CTA i advances box work[i].x over column-planes
// [work[i].y, work[i].z) of that box (column-major: plane fastest), with the
// box's own parameters and fields.  Each node's arithmetic is the same as in
// stream_kernel, so a box gives the same bits alone and in a batch.
template <int LAT, bool HO, bool TC, typename S, typename R, int TYV, bool REP = false, bool OBS = true>
__global__ void __launch_bounds__(TX * TYV, step_min_blocks<R, TYV>())
    stream_kernel_batched(const StepParams<S, R>* __restrict__ boxes, const int4* __restrict__ work) {
    __shared__ StepParams<S, R> sp;
    const int4 w = work[blockIdx.x];
    if (threadIdx.x == 0) sp = boxes[w.x];
    __syncthreads();
    run_share<TYV>(sp.nx, sp.nz, 0, w.y, w.z,
                   [&](int bx, int by, int z0, int z1) { step_body<LAT, HO, TC, S, R, TYV, REP, OBS>(sp, bx, by, z0, z1); });
}

}  // namespace lbf
