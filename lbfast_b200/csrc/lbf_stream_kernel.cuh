// lbf_stream_kernel.cuh -- body of the fused step kernel (see lbf_stream.cuh).
#pragma once
#include "lbf_stream.cuh"

namespace lbf {

// Per-node state after the moments prologue (lb_cuda_moments_module.f90:104-339).
template <typename R> struct NodeState {
    R P, u, v, w, pxx, pyy, pzz, pxy, pxz, pyz;  // post-prologue moments
    R Fx, Fy, Fz;                                // force / rho_phi, as the collision reads it
    R omega;
};

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

template <int LAT, bool HO, bool TC, typename S, typename R>
__global__ void __launch_bounds__(NT, 2) stream_kernel(const StepParams<S, R> p) {
    using CD = Codec<S>;
    using SP = typename PhiStore<S>::type;
    using CP = Codec<SP>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R* pops = reinterpret_cast<R*>(smem_raw);  // [LAT][R1N]
    R* phis = pops + LAT * R1N;                // [PHI_SLOTS][R3N]          (TC)
    R* ths = phis + PHI_SLOTS * R3N;           // [TH_SLOTS][TH_COMP][R2N]  (TC)

    const int t = threadIdx.x;
    const int tx = t % TX, ty = t / TX;
    const int X0 = blockIdx.x * TX, Y0 = blockIdx.y * TY;
    const int z0 = blockIdx.z * p.zseg;
    const int z1 = min(z0 + p.zseg, p.nz);
    const long long N = p.N, plane = p.plane;
    const int nx = p.nx, ny = p.ny, nz = p.nz;
    const bool dr = TC && p.densratio;
    const bool obs = p.obstacles != 0;
    const R cssq = R(1.0 / 3.0);

    // ---- static per-thread node tables (x/y wrap does not change along z) ----
    // R1 node of pass 0 (tile interior) and pass 1 (ring of the collision region)
    const int r1n0 = (ty + 1) * R1X + (tx + 1);
    int r1n1 = -1;
    if (t < NRING1) {
        if (t < R1X) r1n1 = t;                                       // top row
        else if (t < 2 * R1X) r1n1 = (R1Y - 1) * R1X + (t - R1X);    // bottom row
        else if (t < 2 * R1X + TY) r1n1 = (t - 2 * R1X + 1) * R1X;   // left column
        else r1n1 = (t - 2 * R1X - TY + 1) * R1X + (R1X - 1);        // right column
    }
    auto r1_geom = [&](int node, int& off) -> bool {
        if (node < 0) { off = 0; return false; }
        int hx = node % R1X, hy = node / R1X;
        bool ok = true;
        int gx = wrap_coord(X0 + hx - 1, nx, p.pbx, ok);
        int gy = wrap_coord(Y0 + hy - 1, ny, p.pby, ok);
        off = ok ? gy * nx + gx : 0;
        return ok;
    };
    int r1off0, r1off1;
    const bool r1ok0 = r1_geom(r1n0, r1off0);
    const bool r1ok1 = r1_geom(r1n1, r1off1);
    // output node of this thread
    const int ox = X0 + tx, oy = Y0 + ty;
    const bool out_ok = (ox < nx) && (oy < ny);
    const long long out_off = (long long)oy * nx + ox;

    // neighbour x / y offsets of the output node, for the bounce-back isfluid tests
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

    int r2_off[2] = {0, 0};
    bool r2_ok[2] = {false, false};
    int r3_off[3] = {0, 0, 0};
    bool r3_ok[3] = {false, false, false};
    if constexpr (TC) {
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            int n = t + k * NT;
            if (n < R2N) {
                int hx = n % R2X, hy = n / R2X;
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
    auto phi_slot = [&](int q) { return (q - z0 + 3 + 5 * PHI_SLOTS) % PHI_SLOTS; };
    auto th_slot = [&](int q) { return (q - z0 + 2 + 3 * TH_SLOTS) % TH_SLOTS; };

    // stage A: phi plane q into its ring slot (zero outside the box)
    auto load_phi_plane = [&](int q) {
        bool zok = true;
        int wz = zwrap(q, zok);
        R* dst = phis + phi_slot(q) * R3N;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            int n = t + k * NT;
            if (n < R3N) {
                R v = R(0);
                if (zok && r3_ok[k]) v = CP::ld(p.pin, (long long)wz * plane + r3_off[k], p.inv_scale[F_PHI]);
                dst[n] = v;
            }
        }
    };
    // stage B: theta = phi(1-phi) n and g~ = n |g| on the R2 region of plane q
    auto theta_plane = [&](int q) {
        bool zok = true;
        int wz = zwrap(q, zok);
        const R* f0 = phis + phi_slot(q - 1) * R3N;
        const R* f1 = phis + phi_slot(q) * R3N;
        const R* f2 = phis + phi_slot(q + 1) * R3N;
        R* dst = ths + th_slot(q) * (TH_COMP * R2N);
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            int n = t + k * NT;
            if (n >= R2N) continue;
            int hx = n % R2X, hy = n / R2X;
            int c3 = (hy + 1) * R3X + (hx + 1);
            bool fluid = zok && r2_ok[k];
            if (fluid && obs) {
                int s = p.isf[(long long)wz * plane + r2_off[k]];
                fluid = (s == 1 || s == -1);
            }
            R th0 = 0, th1 = 0, th2 = 0, g0 = 0, g1 = 0, g2 = 0;
            if (fluid) {
                auto A = [&](int a, int b, int c) -> R {
                    const R* f = c < 0 ? f0 : (c > 0 ? f2 : f1);
                    return f[c3 + b * R3X + a];
                };
                R gx, gy, gz;
                iso_grad<R>(A, gx, gy, gz);
                R mg = sqrt(gx * gx + gy * gy + gz * gz);
                R den = mg + R(1.0e-9);
                R nxv = gx / den, nyv = gy / den, nzv = gz / den;
                R ph = f1[c3];
                R pp = ph * (R(1) - ph);
                th0 = pp * nxv; th1 = pp * nyv; th2 = pp * nzv;
                g0 = nxv * mg; g1 = nyv * mg; g2 = nzv * mg;
            }
            dst[0 * R2N + n] = th0;
            dst[1 * R2N + n] = th1;
            dst[2 * R2N + n] = th2;
            dst[3 * R2N + n] = g0;
            dst[4 * R2N + n] = g1;
            dst[5 * R2N + n] = g2;
        }
    };

    // accumulators of the raw moments {sum g, sum g c, sum g c c} for output planes
    // q-1 (am), q (a0), q+1 (ap)
    R am[10], a0[10], ap[10];
#pragma unroll
    for (int i = 0; i < 10; ++i) am[i] = a0[i] = ap[i] = R(0);

    if constexpr (TC) {
        for (int q = z0 - 3; q <= z0 + 1; ++q) load_phi_plane(q);
        __syncthreads();
        theta_plane(z0 - 2);
        theta_plane(z0 - 1);
        __syncthreads();
    }

    for (int q = z0 - 1; q <= z1; ++q) {
        if constexpr (TC) {
            // A: prefetch phi(q+3) into the slot of phi(q-2) (last read by stage C of
            //    the previous iteration, which ended with a barrier).
            // B: theta(q+1) from phi(q..q+2) into the slot of theta(q-2).
            load_phi_plane(q + 3);
            theta_plane(q + 1);
            __syncthreads();
        }
        bool zok = true;
        const int wz = zwrap(q, zok);
        const long long zoff = (long long)wz * plane;
        const bool q_inner = (q >= z0) && (q < z1);

        // ---------------- stage C: prologue + collision on the R1 region ----------------
        for (int pass = 0; pass < 2; ++pass) {
            const int node = pass ? r1n1 : r1n0;
            if (node < 0) break;
            const bool inb = zok && (pass ? r1ok1 : r1ok0);
            const long long gi = zoff + (pass ? r1off1 : r1off0);
            int isf = 1;
            if (inb && obs) isf = p.isf[gi];
            R fpop[27];
            bool live = inb && (isf != 0);
            NodeState<R> st;
            R phi_new = 0;
            bool interior = (pass == 0) && out_ok && q_inner;
            if (live) {
                // input moments
                R P = CD::ld(p.min, 0 * N + gi, p.inv_scale[0]);
                R u = CD::ld(p.min, 1 * N + gi, p.inv_scale[1]);
                R v = CD::ld(p.min, 2 * N + gi, p.inv_scale[2]);
                R w = CD::ld(p.min, 3 * N + gi, p.inv_scale[3]);
                R pxx = CD::ld(p.min, 4 * N + gi, p.inv_scale[4]);
                R pyy = CD::ld(p.min, 5 * N + gi, p.inv_scale[5]);
                R pzz = CD::ld(p.min, 6 * N + gi, p.inv_scale[6]);
                R pxy = CD::ld(p.min, 7 * N + gi, p.inv_scale[7]);
                R pxz = CD::ld(p.min, 8 * N + gi, p.inv_scale[8]);
                R pyz = CD::ld(p.min, 9 * N + gi, p.inv_scale[9]);
                R phi = 0, lap = 0, divt = 0, gfx = 0, gfy = 0, gfz = 0;
                if constexpr (TC) {
                    const int hx = node % R1X, hy = node / R1X;
                    const int c3 = (hy + 2) * R3X + (hx + 2);
                    const int c2 = (hy + 1) * R2X + (hx + 1);
                    const R* f0 = phis + phi_slot(q - 1) * R3N;
                    const R* f1 = phis + phi_slot(q) * R3N;
                    const R* f2 = phis + phi_slot(q + 1) * R3N;
                    auto A = [&](int a, int b, int c) -> R {
                        const R* f = c < 0 ? f0 : (c > 0 ? f2 : f1);
                        return f[c3 + b * R3X + a];
                    };
                    phi = f1[c3];
                    lap = iso_lap<R>(A);
                    const R* t0 = ths + th_slot(q - 1) * (TH_COMP * R2N);
                    const R* t1 = ths + th_slot(q) * (TH_COMP * R2N);
                    const R* t2 = ths + th_slot(q + 1) * (TH_COMP * R2N);
                    auto TXa = [&](int a, int b, int c) -> R {
                        const R* f = c < 0 ? t0 : (c > 0 ? t2 : t1);
                        return f[0 * R2N + c2 + b * R2X + a];
                    };
                    auto TYa = [&](int a, int b, int c) -> R {
                        const R* f = c < 0 ? t0 : (c > 0 ? t2 : t1);
                        return f[1 * R2N + c2 + b * R2X + a];
                    };
                    auto TZa = [&](int a, int b, int c) -> R {
                        const R* f = c < 0 ? t0 : (c > 0 ? t2 : t1);
                        return f[2 * R2N + c2 + b * R2X + a];
                    };
                    divt = iso_div<R>(TXa, TYa, TZa);
                    gfx = t1[3 * R2N + c2];
                    gfy = t1[4 * R2N + c2];
                    gfz = t1[5 * R2N + c2];
                }
                // ---- moments prologue: lb_cuda_moments_module.f90:104-339 ----
                R rhophi = R(1), inv = R(1), mask = R(0), fxv, fyv, fzv;
                if constexpr (TC) mask = R(4) * phi * (R(1) - phi);
                if (dr) {
                    rhophi = p.rho_r * phi + (R(1) - phi) * p.rho_b;
                    inv = R(1) / rhophi;
                    fxv = rhophi * p.fx; fyv = rhophi * p.fy; fzv = rhophi * p.fz;
                } else {
                    fxv = p.fx; fyv = p.fy; fzv = p.fz;
                }
                R grx = 0, gry = 0, grz = 0, cv = 0, omega;
                if constexpr (TC) {
                    R chem = R(4) * p.beta * phi * (phi - R(1)) * (phi - R(0.5)) - p.kapp * lap;
                    fxv += chem * gfx;
                    fyv += chem * gfy;
                    fzv += chem * gfz;
                }
                if (dr) {
                    const R drho = p.rho_r - p.rho_b;
                    grx = drho * gfx; gry = drho * gfy; grz = drho * gfz;
                    R mp = mask * P * cssq;
                    fxv -= mp * grx; fyv -= mp * gry; fzv -= mp * grz;
                }
                R tfx = fxv, tfy = fyv, tfz = fzv;
                if (dr) {
                    R uo = CD::ld(p.uin, 0 * N + gi, p.inv_scale[F_UOLD + 0]);
                    R vo = CD::ld(p.uin, 1 * N + gi, p.inv_scale[F_UOLD + 1]);
                    R wo = CD::ld(p.uin, 2 * N + gi, p.inv_scale[F_UOLD + 2]);
                    R qxx = pxx - uo * uo, qyy = pyy - vo * vo, qzz = pzz - wo * wo;
                    R qxy = pxy - uo * vo, qxz = pxz - uo * wo, qyz = pyz - vo * wo;
                    R visc = (p.rho_r * p.visc1 * phi + (R(1) - phi) * p.visc2 * p.rho_b) * inv;
                    R tau = visc * R(3) + R(0.5);
                    omega = R(1) / tau;
                    cv = mask * visc / (tau * cssq);
                    fxv -= cv * (qxx * grx + qxy * gry + qxz * grz);
                    fyv -= cv * (qyy * gry + qxy * grx + qyz * grz);
                    fzv -= cv * (qzz * grz + qxz * grx + qyz * gry);
                    R tmp = -p.sharp_c * divt;
                    u += R(0.5) * fxv * inv;
                    v += R(0.5) * fyv * inv;
                    w += R(0.5) * fzv * inv;
                    R dd = (p.rho_r - p.rho_b) * (p.tau_diff * lap + tmp);
                    R den = R(1) / (R(1) - R(0.5) * dd * inv);
                    u *= den; v *= den; w *= den;
                    tfx -= dd * u; tfy -= dd * v; tfz -= dd * w;
                    fxv -= dd * u; fyv -= dd * v; fzv -= dd * w;
                } else {
                    u += R(0.5) * fxv * inv;
                    v += R(0.5) * fyv * inv;
                    w += R(0.5) * fzv * inv;
                    if constexpr (TC) {
                        R visc = (p.rho_r * p.visc1 * phi + (R(1) - phi) * p.visc2 * p.rho_b) * inv;
                        omega = R(1) / (visc * R(3) + R(0.5));
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
                    R qxx = pxx - u * u, qyy = pyy - v * v, qzz = pzz - w * w;
                    R qxy = pxy - u * v, qxz = pxz - u * w, qyz = pyz - v * w;
                    tfx -= cv * (qxx * grx + qxy * gry + qxz * grz);
                    tfy -= cv * (qyy * gry + qxy * grx + qyz * grz);
                    tfz -= cv * (qzz * grz + qxz * grx + qyz * gry);
                }
                // ---- outputs of this node that leave the kernel ----
                if (interior) {
                    if (p.write_u) {
                        CD::st(p.uout, 0 * N + gi, u, p.scale[F_UOLD + 0]);
                        CD::st(p.uout, 1 * N + gi, v, p.scale[F_UOLD + 1]);
                        CD::st(p.uout, 2 * N + gi, w, p.scale[F_UOLD + 2]);
                    }
                    if constexpr (TC) {
                        // update_phifields: lb_cuda_update_phi_module.f90:77-93
                        phi_new = phi - u * R(0.5) * gfx - v * R(0.5) * gfy - w * R(0.5) * gfz + p.tau_diff * lap -
                                  p.sharp_c * divt;
                        CP::st(p.pout, gi, phi_new, p.scale[F_PHI]);
                    }
                }
                // ---- collision: lb_cuda_fused_module.f90:531-713 ----
                st.P = P;
                st.u = u; st.v = v; st.w = w;
                st.pxx = pxx - u * u; st.pyy = pyy - v * v; st.pzz = pzz - w * w;
                st.pxy = pxy - u * v; st.pxz = pxz - u * w; st.pyz = pyz - v * w;
                st.Fx = tfx * inv; st.Fy = tfy * inv; st.Fz = tfz * inv;
                st.omega = omega;
                const R om1 = R(1) - omega;
                // Hermite coefficients up to second order
                const R m0 = P;
                const R mx = u + R(0.5) * st.Fx, my = v + R(0.5) * st.Fy, mz = w + R(0.5) * st.Fz;
                const R mxx = u * u + om1 * st.pxx + u * st.Fx;
                const R myy = v * v + om1 * st.pyy + v * st.Fy;
                const R mzz = w * w + om1 * st.pzz + w * st.Fz;
                const R mxy = u * v + om1 * st.pxy + R(0.5) * (u * st.Fy + v * st.Fx);
                const R mxz = u * w + om1 * st.pxz + R(0.5) * (u * st.Fz + w * st.Fx);
                const R myz = v * w + om1 * st.pyz + R(0.5) * (v * st.Fz + w * st.Fy);
                if constexpr (LAT == 27) {
                    // M[a][b][c]: coefficient with x/y/z multiplicities a, b, c
                    R M[3][3][3];
                    M[0][0][0] = m0;
                    M[1][0][0] = mx; M[0][1][0] = my; M[0][0][1] = mz;
                    M[2][0][0] = mxx; M[0][2][0] = myy; M[0][0][2] = mzz;
                    M[1][1][0] = mxy; M[1][0][1] = mxz; M[0][1][1] = myz;
                    if constexpr (HO) {
                        const R X = st.pxx, Y = st.pyy, Z = st.pzz, XY = st.pxy, XZ = st.pxz, YZ = st.pyz;
                        const R u2 = u * u, v2 = v * v, w2 = w * w;
                        // recursive non-equilibrium terms, rows 10..26 (lb_cuda_fused_module.f90:686-703)
                        M[2][1][0] = u2 * v + om1 * (R(2) * XY * u + X * v);                          // 10 xxy
                        M[2][0][1] = u2 * w + om1 * (R(2) * XZ * u + X * w);                          // 11 xxz
                        M[1][2][0] = u * v2 + om1 * (Y * u + R(2) * XY * v);                          // 12 xyy
                        M[1][0][2] = u * w2 + om1 * (Z * u + R(2) * XZ * w);                          // 13 xzz
                        M[0][1][2] = v * w2 + om1 * (Z * v + R(2) * YZ * w);                          // 14 yzz
                        M[0][2][1] = v2 * w + om1 * (R(2) * YZ * v + Y * w);                          // 15 yyz
                        M[1][1][1] = u * v * w + om1 * (YZ * u + XZ * v + XY * w);                    // 16 xyz
                        M[2][2][0] = u2 * v2 + om1 * (Y * u2 + R(2) * v * (R(3) * XY * u + X * v));   // 17
                        M[2][0][2] = u2 * w2 + om1 * (Z * u2 + R(2) * w * (R(3) * XZ * u + X * w));   // 18
                        M[0][2][2] = v2 * w2 + om1 * (Z * v2 + R(2) * w * (R(3) * YZ * v + Y * w));   // 19
                        M[1][1][2] = u * v * w2 +
                                     om1 * (Z * u * v + w * (R(3) * YZ * u + R(3) * XZ * v + R(2) * XY * w));  // 20
                        M[1][2][1] = u * v2 * w +
                                     om1 * (R(2) * YZ * u * v + XZ * v2 + R(2) * Y * u * w + R(4) * XY * v * w);  // 21
                        M[2][1][1] = u2 * v * w +
                                     om1 * (YZ * u2 + R(2) * XZ * u * v + R(4) * XY * u * w + R(2) * X * v * w);  // 22
                        M[2][1][2] = u2 * v * w2 +
                                     om1 * (Z * u2 * v + R(3) * w * (YZ * u2 + R(2) * XZ * u * v + R(2) * XY * u * w +
                                                                     X * v * w));  // 23
                        M[2][2][1] = u2 * v2 * w + om1 * (R(2) * u * v * (YZ * u + XZ * v) + R(2) * Y * u2 * w +
                                                          v * (R(10) * XY * u + R(3) * X * v) * w);  // 24
                        M[1][2][2] = u * v2 * w2 +
                                     om1 * (Z * u * v2 + R(3) * w * (R(2) * YZ * u * v + XZ * v2 + Y * u * w +
                                                                     R(2) * XY * v * w));  // 25
                        M[2][2][2] = u2 * v2 * w2 +
                                     om1 * (Z * u2 * v2 + w * (R(6) * u * v * (YZ * u + XZ * v) + R(3) * Y * u2 * w +
                                                               R(2) * v * (R(7) * XY * u + R(2) * X * v) * w));  // 26
                    } else {
                        M[2][1][0] = M[2][0][1] = M[1][2][0] = M[1][0][2] = M[0][1][2] = M[0][2][1] = M[1][1][1] = R(0);
                        M[2][2][0] = M[2][0][2] = M[0][2][2] = M[1][1][2] = M[1][2][1] = M[2][1][1] = R(0);
                        M[2][1][2] = M[2][2][1] = M[1][2][2] = M[2][2][2] = R(0);
                    }
                    // x pass: T[cx][b][c]
                    R T[3][3][3];
#pragma unroll
                    for (int b = 0; b < 3; ++b)
#pragma unroll
                        for (int c = 0; c < 3; ++c) d1q3_inv<R>(M[0][b][c], M[1][b][c], M[2][b][c], T[0][b][c], T[1][b][c], T[2][b][c]);
                    // y pass: U[cx][cy][c] (reuse M)
#pragma unroll
                    for (int a = 0; a < 3; ++a)
#pragma unroll
                        for (int c = 0; c < 3; ++c) d1q3_inv<R>(T[a][0][c], T[a][1][c], T[a][2][c], M[a][0][c], M[a][1][c], M[a][2][c]);
                    // z pass: populations
#pragma unroll
                    for (int a = 0; a < 3; ++a)
#pragma unroll
                        for (int b = 0; b < 3; ++b) {
                            R vm, v0, vp;
                            d1q3_inv<R>(M[a][b][0], M[a][b][1], M[a][b][2], vm, v0, vp);
                            fpop[LINK(a - 1, b - 1, -1)] = vm;
                            fpop[LINK(a - 1, b - 1, 0)] = v0;
                            fpop[LINK(a - 1, b - 1, 1)] = vp;
                        }
                } else {
                    // D3Q19: f*_l = w_l [m0 + 3 c.m1 + 4.5 H2(c):m2]
                    const R base = m0 - R(1.5) * (mxx + myy + mzz);
#pragma unroll
                    for (int l = 0; l < 19; ++l) {
                        const int cx = EX(l), cy = EY(l), cz = EZ(l);
                        R s = base;
                        s += R(3) * (R(cx) * mx + R(cy) * my + R(cz) * mz);
                        s += R(4.5) * (R(cx * cx) * mxx + R(cy * cy) * myy + R(cz * cz) * mzz);
                        s += R(9) * (R(cx * cy) * mxy + R(cx * cz) * mxz + R(cy * cz) * myz);
                        fpop[l] = R(WL<19>(l)) * s;
                    }
                }
            } else {
#pragma unroll
                for (int l = 0; l < LAT; ++l) fpop[l] = R(0);
            }
#pragma unroll
            for (int l = 0; l < LAT; ++l) pops[l * R1N + node] = fpop[l];

            // ---- obstacle bounce-back: lb_cuda_boundary_module.f90:162-199 ----
            if (interior && obs && isf == -1) {
                const R om1 = R(1) - st.omega;
#pragma unroll
                for (int l = 1; l < LAT; ++l) {
                    const int cx = EX(l), cy = EY(l), cz = EZ(l);
                    // upstream node x - c_l
                    const int ix = 1 - cx, iy = 1 - cy;
                    bool ok = nbx_ok[ix] && nby_ok[iy];
                    bool zk = true;
                    int zz = zwrap(q - cz, zk);
                    int s = 1;
                    if (ok && zk) s = p.isf[(long long)zz * plane + (long long)nby[iy] * nx + nbx[ix]];
                    if (s != 0) continue;
                    const R wl = R(WL<LAT>(l));
                    const R dx = R(cx), dy = R(cy), dz = R(cz);
                    R fneq = wl * R(4.5) *
                             ((dx * dx - cssq) * st.pxx + (dy * dy - cssq) * st.pyy + (dz * dz - cssq) * st.pzz +
                              R(2) * (dx * dy) * st.pxy + R(2) * (dx * dz) * st.pxz + R(2) * (dy * dz) * st.pyz);
                    R fp = wl * st.P + om1 * fneq;
                    a0[0] += fp;
                    a0[1] += fp * dx; a0[2] += fp * dy; a0[3] += fp * dz;
                    a0[4] += fp * (dx * dx); a0[5] += fp * (dy * dy); a0[6] += fp * (dz * dz);
                    a0[7] += fp * (dx * dy); a0[8] += fp * (dx * dz); a0[9] += fp * (dy * dz);
                }
            }
        }
        __syncthreads();

        // ---------------- stage D: pull populations of plane q ----------------
#pragma unroll
        for (int zc = 0; zc < 3; ++zc) {
            const int cz = zc - 1;
            // x sums for each cy
            R S0[3], S1[3], S2[3];
#pragma unroll
            for (int yc = 0; yc < 3; ++yc) {
                const int cy = yc - 1;
                R g[3];
#pragma unroll
                for (int xc = 0; xc < 3; ++xc) {
                    const int cx = xc - 1;
                    const int l = LINK(cx, cy, cz);
                    if (LAT == 19 && (cx * cx + cy * cy + cz * cz) == 3) {
                        g[xc] = R(0);
                    } else {
                        g[xc] = pops[l * R1N + (ty + 1 - cy) * R1X + (tx + 1 - cx)];
                    }
                }
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
            if (zc == 0) accum_slice<R>(am, R(cz), Y00, Y01, Y02, Y10, Y11, Y20);
            else if (zc == 1) accum_slice<R>(a0, R(cz), Y00, Y01, Y02, Y10, Y11, Y20);
            else accum_slice<R>(ap, R(cz), Y00, Y01, Y02, Y10, Y11, Y20);
        }
        if (q - 1 >= z0 && out_ok) {
            const long long go = (long long)(q - 1) * plane + out_off;
            const R third = am[0] * cssq;
            CD::st(p.mout, 0 * N + go, am[0], p.scale[0]);
            CD::st(p.mout, 1 * N + go, am[1], p.scale[1]);
            CD::st(p.mout, 2 * N + go, am[2], p.scale[2]);
            CD::st(p.mout, 3 * N + go, am[3], p.scale[3]);
            CD::st(p.mout, 4 * N + go, am[4] - third, p.scale[4]);
            CD::st(p.mout, 5 * N + go, am[5] - third, p.scale[5]);
            CD::st(p.mout, 6 * N + go, am[6] - third, p.scale[6]);
            CD::st(p.mout, 7 * N + go, am[7], p.scale[7]);
            CD::st(p.mout, 8 * N + go, am[8], p.scale[8]);
            CD::st(p.mout, 9 * N + go, am[9], p.scale[9]);
        }
#pragma unroll
        for (int i = 0; i < 10; ++i) {
            am[i] = a0[i];
            a0[i] = ap[i];
            ap[i] = R(0);
        }
        if constexpr (!TC) __syncthreads();
    }
}

}  // namespace lbf
