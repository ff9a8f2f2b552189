// lbf_repulsive.cu -- REPULSIVE_FLUX (lb_cuda_repulsive_module.f90:19-292):
// a film-repulsion force between facing interfaces, computed before each step
// from the step's phi and read by the fused step's moments prologue
// (lb_cuda_moments_module.f90:148-160).  Two passes: the unit normals of the
// phi gradient on fluid nodes (compute_norm's aux 1-3,
// lb_cuda_auxfields_module.f90:72-112), then per interfacial node the window
// scan for the facing partner and the pair's force (the reference's
// thinfilm_scan_mark_kernel and repulsive_flux_normal_kernel in one pass: the
// partner's offset is not kept).  FP64, as the reference's (real(kind=db)).
#include <type_traits>

#include "lbf_internal.h"
#include "lbf_stream.cuh"

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

// index of (i, j, k) folded into the box on periodic axes; -1 beyond a
// non-periodic face (the reference's halo there: isfluid 1, phi 0, aux 0)
__device__ __forceinline__ long long wrap_idx(const RepulsiveArgs& a, int i, int j, int k) {
    bool ok = true;
    const int x = wrap_coord(i, a.nx, a.pbx, ok), y = wrap_coord(j, a.ny, a.pby, ok);
    const int z = wrap_coord(k, a.nz, a.pbz, ok);
    return ok ? ((long long)z * a.ny + y) * a.nx + x : -1;
}

// n = g / (|g| + 1e-9) on fluid nodes, 0 elsewhere (3 x N, FP64)
template <typename SP> __global__ void rep_normals_kernel(const RepulsiveArgs a) {
    const long long N = (long long)a.nx * a.ny * a.nz;
    const SP* ph = static_cast<const SP*>(a.phi);
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < N; g += (long long)gridDim.x * blockDim.x) {
        double n0 = 0, n1 = 0, n2 = 0;
        const int f = a.isf ? a.isf[g] : 1;
        if (f == 1 || f == -1) {
            const int x = (int)(g % a.nx), y = (int)((g / a.nx) % a.ny), z = (int)(g / ((long long)a.nx * a.ny));
            double gx, gy, gz;
            iso_grad<double>(
                [&](int p, int q, int r) {
                    const long long c = wrap_idx(a, x + p, y + q, z + r);
                    return c < 0 ? 0.0 : (double)ph[c];
                },
                gx, gy, gz);
            const double den = sqrt(gx * gx + gy * gy + gz * gz) + 1.0e-9;
            n0 = gx / den; n1 = gy / den; n2 = gz / den;
        }
        a.nrm[g] = n0; a.nrm[N + g] = n1; a.nrm[2 * N + g] = n2;
    }
}

// the force of each node (3 x N in the arithmetic type R; 0 where no pair)
template <typename SP, typename R> __global__ void rep_force_kernel(const RepulsiveArgs a) {
    const long long N = (long long)a.nx * a.ny * a.nz;
    const SP* ph = static_cast<const SP*>(a.phi);
    R* out = static_cast<R*>(a.force);
    const double eps = 1.0e-9;
    // the pair search reads the step's input phi after the mass correction
    // (thinfilm_scan_mark_cuda runs after bcs_mesoscopic_phifields,
    // integrator_module.f90:297-328); the normals above are compute_norm's,
    // from the uncorrected phi.  Every node of the search is a fluid node.
    double corr = 0.0;
    const bool mc = mass_corr(a.mass, corr);
    auto PH = [&](long long i) {
        const double v = (double)ph[i];
        return mc ? mass_corrected<SP>(v, corr) : v;
    };
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < N; g += (long long)gridDim.x * blockDim.x) {
        double fo[3] = {0, 0, 0};
        const int f = a.isf ? a.isf[g] : 1;
        const double loc_phi = (f == 1 || f == -1) ? PH(g) : (double)ph[g];
        double qloc = fmin(fmax(loc_phi, 0.0), 1.0);
        qloc = qloc * (1.0 - qloc);
        if ((f == 1 || f == -1) && qloc >= a.q_th) {
            const int x = (int)(g % a.nx), y = (int)((g / a.nx) % a.ny), z = (int)(g / ((long long)a.nx * a.ny));
            const double nix = a.nrm[g], niy = a.nrm[N + g], niz = a.nrm[2 * N + g];
            // scan and mark (lb_cuda_repulsive_module.f90:63-150): nearest facing
            // partner of similar q, ties to the larger facing factor; x outermost
            double best_r2 = 1.0e300, best_face = -1.0;
            int bi = 0, bj = 0, bk = 0;
            bool found = false;
            for (int di = -3; di <= 3; ++di)
                for (int dj = -3; dj <= 3; ++dj)
                    for (int dk = -3; dk <= 3; ++dk) {
                        if (di == 0 && dj == 0 && dk == 0) continue;
                        const long long nb = wrap_idx(a, x + di, y + dj, z + dk);
                        const int fn = nb < 0 ? 1 : (a.isf ? a.isf[nb] : 1);
                        if (fn != 1 && fn != -1) continue;
                        const double r2 = (double)(di * di + dj * dj + dk * dk);
                        double qn = nb < 0 ? 0.0 : PH(nb);
                        qn = fmin(fmax(qn, 0.0), 1.0);
                        qn = qn * (1.0 - qn);
                        if (qn < a.q_th || fabs(qn - qloc) > 0.1 * fmax(qloc, 1.0e-12)) continue;
                        const double dotn = nb < 0 ? 0.0 : nix * a.nrm[nb] + niy * a.nrm[N + nb] + niz * a.nrm[2 * N + nb];
                        if (dotn > a.cos_opp_t) continue;
                        const double face = 0.5 * (1.0 - dotn);
                        if (r2 < best_r2 - 1.0e-14) {
                            best_r2 = r2; best_face = face; bi = di; bj = dj; bk = dk; found = true;
                        } else if (fabs(r2 - best_r2) <= 1.0e-14 && face > best_face) {
                            best_face = face; bi = di; bj = dj; bk = dk; found = true;
                        }
                    }
            // normal repulsive flux (lb_cuda_repulsive_module.f90:194-289)
            const double q1 = loc_phi * (1.0 - loc_phi);
            if (found && q1 > eps) {
                double dx = bi, dy = bj, dz = bk;
                const double r = sqrt(dx * dx + dy * dy + dz * dz);
                dx /= r; dy /= r; dz /= r;
                const long long nb = wrap_idx(a, x + bi, y + bj, z + bk);
                const double n2x = nb < 0 ? 0.0 : a.nrm[nb], n2y = nb < 0 ? 0.0 : a.nrm[N + nb];
                const double n2z = nb < 0 ? 0.0 : a.nrm[2 * N + nb];
                const double face = fmax(0.0, -(nix * n2x + niy * n2y + niz * n2z));
                if (face > eps) {
                    double nsx = nix - n2x, nsy = niy - n2y, nsz = niz - n2z;
                    const double nsm = sqrt(nsx * nsx + nsy * nsy + nsz * nsz);
                    if (nsm <= eps) {
                        nsx = dx; nsy = dy; nsz = dz;
                    } else {
                        nsx /= nsm; nsy /= nsm; nsz /= nsm;
                    }
                    if (dx * nsx + dy * nsy + dz * nsz < 0) { nsx = -nsx; nsy = -nsy; nsz = -nsz; }
                    const double phi2 = nb < 0 ? 0.0 : PH(nb);
                    const double qpair = 0.5 * (q1 + phi2 * (1.0 - phi2));
                    const double qcl = fmin(fmax(qpair, eps), 0.25 - eps);
                    const double arg = 1.0 / (2.0 * sqrt(qcl));
                    if (arg > 1.0) {
                        const double wfilm = a.width * log(arg + sqrt(arg * arg - 1.0));
                        if (wfilm > 0) {
                            const double wd = 1.0 / (1.0 + pow(wfilm, 4.0));
                            const double s = a.a_rep * wd * qcl * face;
                            const double fx = s * nsx, fy = s * nsy, fz = s * nsz;
                            const double cap = 1.5 * (fabs(fx) + fabs(fy) + fabs(fz));
                            const double sc = fmin(1.0, loc_phi / fmax(cap, 1.0e-9));
                            fo[0] = fx * sc; fo[1] = fy * sc; fo[2] = fz * sc;
                        }
                    }
                }
            }
        }
        out[g] = (R)fo[0]; out[N + g] = (R)fo[1]; out[2 * N + g] = (R)fo[2];
    }
}

}  // namespace

cudaError_t launch_repulsive(int storage, const RepulsiveArgs& a, cudaStream_t st) {
    const long long N = (long long)a.nx * a.ny * a.nz;
    return by_storage(storage, [&](auto tag) {
        using S = decltype(tag);
        using SP = typename PhiStore<S>::type;
        using R = typename std::conditional<sizeof(S) == 8, double, float>::type;
        rep_normals_kernel<SP><<<grid_for(N, 256), 256, 0, st>>>(a);
        rep_force_kernel<SP, R><<<grid_for(N, 128), 128, 0, st>>>(a);
        return cudaGetLastError();
    });
}

}  // namespace lbf
