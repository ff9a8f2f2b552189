// lbf_misc.cu -- the small kernels around the fused step: wetting ghost phi,
// field conversions at the host boundary, copy_print extraction and FP64
// reductions.
#include <type_traits>

#include "lbf_internal.h"
#include "lbf_stream.cuh"

namespace lbf {

size_t storage_bytes(int storage) {
    switch (storage) {
        case 0: return 4;
        case 1: return 2;
        case 2: return 2;
        case 3: return 8;
    }
    return 0;
}
size_t phi_bytes(int storage) { return storage == 3 ? 8 : 4; }

template <typename S> struct Arith { using R = float; };
template <> struct Arith<double> { using R = double; };

template <typename Fn> static cudaError_t by_storage(int storage, Fn&& fn) {
    switch (storage) {
        case 0: return fn(float{});
        case 1: return fn(__half{});
        case 2: return fn(__nv_bfloat16{});
        case 3: return fn(double{});
    }
    return cudaErrorInvalidValue;
}

static inline int blocks_for(long long n, int bs) {
    long long b = (n + bs - 1) / bs;
    if (b > 148LL * 64) b = 148LL * 64;  // grid-stride beyond this
    return (int)(b < 1 ? 1 : b);
}

// ---------------------------------------------------------------------------
// Wetting ghost phi at solid nodes: PHI_int_boundary_kernel,
// lb_cuda_boundary_module.f90:218-459.  The wall normal and the donor depend
// only on isfluid and are precomputed on the host; here the donor's gradient
// (compute_norm_interface at the donor, lb_cuda_auxfields_module.f90:72-112)
// and the extrapolation (:404-454) are evaluated.  The result goes to `wout`
// and is written into phi only after every reader of the pre-wetting phi has
// run (see lbf_step).
// ---------------------------------------------------------------------------
template <typename SP, typename R>
__global__ void wetting_kernel(const WetArgs a) {
    using CP = Codec<SP>;
    const SP* pin = static_cast<const SP*>(a.pin);
    SP* wout = static_cast<SP*>(a.wout);
    const long long plane = (long long)a.nx * a.ny;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        if (a.scatter_dst) {
            static_cast<SP*>(a.scatter_dst)[a.s_idx[i]] = static_cast<const SP*>(a.scatter_src)[i];
        }
        const int flag = a.flag[i];
        if (flag == WET_OPENCOPY) {
            // wall node of an open face: the phi of its neighbour on the plane
            // next to it replaces the wetting value (boundary_cds_module.f90:1351-1663)
            const long long d = (long long)a.donor[3 * i + 2] * plane + (long long)a.donor[3 * i + 1] * a.nx +
                                a.donor[3 * i];
            wout[i] = pin[d];
            continue;
        }
        const R old = CP::ld(pin, a.s_idx[i], R(1));
        R ghost;
        if (flag == WET_OUTSIDE || (a.prime && flag == WET_HIGHWRAP)) {
            // donor on a never-written halo layer: phi = 0 and aux = 0 there
            ghost = R(0);
        } else {
            const int dx = a.donor[3 * i], dy = a.donor[3 * i + 1], dz = a.donor[3 * i + 2];
            const R phid = CP::ld(pin, (long long)dz * plane + (long long)dy * a.nx + dx, R(1));
            R gx = 0, gy = 0, gz = 0;
            if (!a.prime) {
                auto A = [&](int ox, int oy, int oz) -> R {
                    bool ok = true;
                    int x = wrap_coord(dx + ox, a.nx, a.pbx, ok);
                    int y = wrap_coord(dy + oy, a.ny, a.pby, ok);
                    int z = wrap_coord(dz + oz, a.nz, a.pbz, ok);
                    return ok ? CP::ld(pin, (long long)z * plane + (long long)y * a.nx + x, R(1)) : R(0);
                };
                R g0, g1, g2;
                iso_grad<R>(A, g0, g1, g2);
                R mg = sqrt(g0 * g0 + g1 * g1 + g2 * g2);
                R den = mg + R(1.0e-9);
                gx = (g0 / den) * mg;
                gy = (g1 / den) * mg;
                gz = (g2 / den) * mg;
            }
            const R wx = (R)a.wn[3 * i], wy = (R)a.wn[3 * i + 1], wz = (R)a.wn[3 * i + 2];
            const R gdw = gx * wx + gy * wy + gz * wz;
            const R tx = gx - gdw * wx, ty = gy - gdw * wy, tz = gz - gdw * wz;
            const R tmag = sqrt(tx * tx + ty * ty + tz * tz);
            const R dn = -tmag * (R)a.cot_theta;
            const R bx = tx + dn * wx, by = ty + dn * wy, bz = tz + dn * wz;
            const R sx = (R)a.shift[3 * i], sy = (R)a.shift[3 * i + 1], sz = (R)a.shift[3 * i + 2];
            ghost = phid + (bx * sx + by * sy + bz * sz) * (R(4) * old * (R(1) - old));
        }
        ghost = max(R(0), min(R(1), ghost));
        CP::st(wout, i, ghost, R(1));
    }
}

cudaError_t launch_wetting(int storage, const WetArgs& a, cudaStream_t st) {
    if (a.n <= 0) return cudaSuccess;
    return by_storage(storage, [&](auto tag) {
        using S = decltype(tag);
        using SP = typename PhiStore<S>::type;
        using R = typename Arith<S>::R;
        wetting_kernel<SP, R><<<blocks_for(a.n, 256), 256, 0, st>>>(a);
        return cudaGetLastError();
    });
}

template <typename SP>
__global__ void wet_apply_kernel(int n, const long long* s_idx, const SP* src, SP* dst) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[s_idx[i]] = src[i];
}

cudaError_t launch_wet_apply(int storage, int n, const long long* s_idx, const void* src, void* dst, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    return by_storage(storage, [&](auto tag) {
        using S = decltype(tag);
        using SP = typename PhiStore<S>::type;
        wet_apply_kernel<SP><<<blocks_for(n, 256), 256, 0, st>>>(n, s_idx, static_cast<const SP*>(src),
                                                                   static_cast<SP*>(dst));
        return cudaGetLastError();
    });
}

// ---------------------------------------------------------------------------
// conversions between host arrays (float/double) and stored fields
// ---------------------------------------------------------------------------
template <typename T, typename S, typename R>
__global__ void convert_in_kernel(const T* src, S* dst, long long n, R scale) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        Codec<S>::st(dst, i, (R)src[i], scale);
}
template <typename S, typename T, typename R>
__global__ void convert_out_kernel(const S* src, T* dst, long long n, R inv) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[i] = (T)Codec<S>::ld(src, i, inv);
}

cudaError_t launch_convert_in(int storage, bool is_phi, const void* src, int src_dtype, void* dst, long long n,
                              double scale, cudaStream_t st) {
    return by_storage(storage, [&](auto tag) {
        using S0 = decltype(tag);
        using R = typename Arith<S0>::R;
        auto go = [&](auto stag) {
            using S = decltype(stag);
            if (src_dtype == 1)
                convert_in_kernel<double, S, R><<<blocks_for(n, 256), 256, 0, st>>>(static_cast<const double*>(src),
                                                                                    static_cast<S*>(dst), n, (R)scale);
            else
                convert_in_kernel<float, S, R><<<blocks_for(n, 256), 256, 0, st>>>(static_cast<const float*>(src),
                                                                                   static_cast<S*>(dst), n, (R)scale);
            return cudaGetLastError();
        };
        if (is_phi) return go(typename PhiStore<S0>::type{});
        return go(S0{});
    });
}

cudaError_t launch_convert_out(int storage, bool is_phi, const void* src, void* dst, int dst_dtype, long long n,
                               double inv_scale, cudaStream_t st) {
    return by_storage(storage, [&](auto tag) {
        using S0 = decltype(tag);
        using R = typename Arith<S0>::R;
        auto go = [&](auto stag) {
            using S = decltype(stag);
            if (dst_dtype == 1)
                convert_out_kernel<S, double, R><<<blocks_for(n, 256), 256, 0, st>>>(
                    static_cast<const S*>(src), static_cast<double*>(dst), n, (R)inv_scale);
            else
                convert_out_kernel<S, float, R><<<blocks_for(n, 256), 256, 0, st>>>(
                    static_cast<const S*>(src), static_cast<float*>(dst), n, (R)inv_scale);
            return cudaGetLastError();
        };
        if (is_phi) return go(typename PhiStore<S0>::type{});
        return go(S0{});
    });
}

// ---------------------------------------------------------------------------
// copy_print (print_module.f90:638-776)
// ---------------------------------------------------------------------------
template <typename S, typename R>
__global__ void print_kernel(const PrintArgs a) {
    using SP = typename PhiStore<S>::type;
    // with 16-bit storage P is a float array (PhiStore<S> is float there too)
    using SPres = typename std::conditional<Codec<S>::scaled, float, S>::type;
    const SPres* P = static_cast<const SPres*>(a.P);
    const S* V = static_cast<const S*>(a.vel);
    const SP* ph = static_cast<const SP*>(a.phi);
    // the copy_print of a step reads its input phi after the mass correction
    double corr = 0.0;
    const bool mc = mass_corr(a.mass, corr);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < a.N; i += (long long)gridDim.x * blockDim.x) {
        R press = Codec<SPres>::ld(P, i, (R)a.sP);
        if (a.rho) {
            R r;
            if (a.mode == 0) r = press;
            else {
                R f = Codec<SP>::ld(ph, i, R(1));
                if (mc && (!a.isf || a.isf[i] == 1 || a.isf[i] == -1)) f = (R)mass_corrected<SP>((double)f, corr);
                r = a.mode == 1 ? f : (R)a.rho_r * f + (R(1) - f) * (R)a.rho_b;
            }
            a.rho[i] = (float)r;
        }
        if (a.press) a.press[i] = (float)press;
        if (a.vel_out && a.vel32) {
            a.vel_out[3 * i + 0] = a.vel32[i];
            a.vel_out[3 * i + 1] = a.vel32[a.N + i];
            a.vel_out[3 * i + 2] = a.vel32[2 * a.N + i];
        } else if (a.vel_out) {
            a.vel_out[3 * i + 0] = (float)Codec<S>::ld(V, i, (R)a.su[0]);
            a.vel_out[3 * i + 1] = (float)Codec<S>::ld(V, a.N + i, (R)a.su[1]);
            a.vel_out[3 * i + 2] = (float)Codec<S>::ld(V, 2 * a.N + i, (R)a.su[2]);
        }
    }
}

cudaError_t launch_print(int storage, const PrintArgs& a, cudaStream_t st) {
    return by_storage(storage, [&](auto tag) {
        using S = decltype(tag);
        using R = typename Arith<S>::R;
        print_kernel<S, R><<<blocks_for(a.N, 256), 256, 0, st>>>(a);
        return cudaGetLastError();
    });
}

// ---------------------------------------------------------------------------
// FP64 sums over fluid nodes (phi_sum_count_kernel, lb_cuda_boundary_module.f90:461-515,
// with a block-level tree instead of one atomic per node)
// ---------------------------------------------------------------------------
template <typename S>
__global__ void reduce_kernel(long long N, const S* mom, const float* pres, const typename PhiStore<S>::type* phi,
                              const int8_t* isf, double s0, double s1, double s2, double s3, double* out) {
    using SP = typename PhiStore<S>::type;
    double acc[5] = {0, 0, 0, 0, 0};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        if (isf) {
            int f = isf[i];
            if (f != 1 && f != -1) continue;
        }
        if (phi) acc[0] += (double)Codec<SP>::ld(phi, i, 1.0);
        if (Layout<S>::split) {
            acc[1] += (double)pres[i];
            acc[2] += (double)pres[N + i];
            acc[3] += (double)pres[2 * N + i];
            acc[4] += (double)pres[3 * N + i];
        } else {
            acc[1] += (double)Codec<S>::ld(mom, i, s0);
            acc[2] += (double)Codec<S>::ld(mom, N + i, s1);
            acc[3] += (double)Codec<S>::ld(mom, 2 * N + i, s2);
            acc[4] += (double)Codec<S>::ld(mom, 3 * N + i, s3);
        }
    }
    __shared__ double red[5][256];
#pragma unroll
    for (int k = 0; k < 5; ++k) red[k][threadIdx.x] = acc[k];
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s)
#pragma unroll
            for (int k = 0; k < 5; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < 5; ++k) atomicAdd(out + k, red[k][0]);
}

// ---------------------------------------------------------------------------
// 16-bit upload: group maxima and Pi - u u on the device
// ---------------------------------------------------------------------------
constexpr int PIN_A[6] = {1, 2, 3, 1, 1, 2}, PIN_B[6] = {1, 2, 3, 2, 3, 3};

template <typename T> __global__ void upload_maxabs_kernel(long long N, const T* f, unsigned* out) {
    const int ua[6] = {1, 2, 3, 1, 1, 2}, ub[6] = {1, 2, 3, 2, 3, 3};
    float mu = 0.f, mpi = 0.f;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        double m[10];
#pragma unroll
        for (int k = 0; k < 10; ++k) m[k] = (double)f[k * N + i];
#pragma unroll
        for (int k = 1; k <= 3; ++k)
            if (isfinite(m[k])) mu = fmaxf(mu, (float)fabs(m[k]));
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            const double v = m[4 + c] - m[ua[c]] * m[ub[c]];
            if (isfinite(v)) mpi = fmaxf(mpi, (float)fabs(v));
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mu = fmaxf(mu, __shfl_xor_sync(0xffffffffu, mu, o));
        mpi = fmaxf(mpi, __shfl_xor_sync(0xffffffffu, mpi, o));
    }
    // non-negative floats order as their bit patterns
    if ((threadIdx.x & 31) == 0) {
        atomicMax(out, __float_as_uint(mu));
        atomicMax(out + 1, __float_as_uint(mpi));
    }
}

template <typename T, typename S>
__global__ void upload_pin_kernel(long long N, const T* f, int a, int b, int c, S* dst, float scale) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        const double v = (double)f[(4 + c) * N + i] - (double)f[a * N + i] * (double)f[b * N + i];
        Codec<S>::st(dst, i, (float)v, scale);
    }
}

cudaError_t launch_upload_maxabs(int src_dtype, long long N, const void* staged10, unsigned* d_max, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(d_max, 0, 2 * sizeof(unsigned), st);
    if (e != cudaSuccess) return e;
    if (src_dtype == 1)
        upload_maxabs_kernel<double><<<blocks_for(N, 256), 256, 0, st>>>(N, static_cast<const double*>(staged10), d_max);
    else
        upload_maxabs_kernel<float><<<blocks_for(N, 256), 256, 0, st>>>(N, static_cast<const float*>(staged10), d_max);
    return cudaGetLastError();
}

cudaError_t launch_upload_pin(int storage, int src_dtype, long long N, const void* staged10, int c, void* dst,
                              double scale, cudaStream_t st) {
    auto go = [&](auto stag) {
        using S = decltype(stag);
        if (src_dtype == 1)
            upload_pin_kernel<double, S><<<blocks_for(N, 256), 256, 0, st>>>(
                N, static_cast<const double*>(staged10), PIN_A[c], PIN_B[c], c, static_cast<S*>(dst), (float)scale);
        else
            upload_pin_kernel<float, S><<<blocks_for(N, 256), 256, 0, st>>>(
                N, static_cast<const float*>(staged10), PIN_A[c], PIN_B[c], c, static_cast<S*>(dst), (float)scale);
        return cudaGetLastError();
    };
    if (storage == 1) return go(__half());
    if (storage == 2) return go(__nv_bfloat16());
    return cudaErrorInvalidValue;
}

// vel32 holds u, v, w (FP32); moment field a in 1..3 is vel32[(a - 1) N]
template <typename S, typename T>
__global__ void download_pi_kernel(long long N, const S* m, const float* vel32, float sc, int a, int b, int c, T* dst) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        const double ua = (double)vel32[(a - 1) * N + i];
        const double ub = (double)vel32[(b - 1) * N + i];
        const double pn = (double)Codec<S>::ld(m + c * N, i, sc);
        dst[i] = (T)(pn + ua * ub);
    }
}

cudaError_t launch_download_pi(int storage, int dst_dtype, long long N, const void* mom, const float* vel32,
                               const double* inv_scale, int c, void* dst, cudaStream_t st) {
    const int a = PIN_A[c], b = PIN_B[c];
    auto go = [&](auto stag) {
        using S = decltype(stag);
        const S* m = static_cast<const S*>(mom);
        if (dst_dtype == 1)
            download_pi_kernel<S, double><<<blocks_for(N, 256), 256, 0, st>>>(
                N, m, vel32, (float)inv_scale[4 + c], a, b, c, static_cast<double*>(dst));
        else
            download_pi_kernel<S, float><<<blocks_for(N, 256), 256, 0, st>>>(
                N, m, vel32, (float)inv_scale[4 + c], a, b, c, static_cast<float*>(dst));
        return cudaGetLastError();
    };
    if (storage == 1) return go(__half());
    if (storage == 2) return go(__nv_bfloat16());
    return cudaErrorInvalidValue;
}

// ---------------------------------------------------------------------------
// phi mass correction (phi_sum_count_kernel + apply_lagrangian_phi_kernel,
// lb_cuda_boundary_module.f90:459-563): FP64 sums, tree per block, one atomic
// per block
// ---------------------------------------------------------------------------
template <typename SP>
__global__ void mass_sum_kernel(long long N, const SP* phi, const int8_t* isf, double* out, bool count) {
    double acc = 0, cnt = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        if (isf) {
            const int f = isf[i];
            if (f != 1 && f != -1) continue;
        }
        const double v = (double)phi[i];
        acc += v;
        if (v > 0.5 && v < 0.9) cnt += 1.0;
    }
    __shared__ double red[2][256];
    red[0][threadIdx.x] = acc;
    red[1][threadIdx.x] = cnt;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) {
            red[0][threadIdx.x] += red[0][threadIdx.x + s];
            red[1][threadIdx.x] += red[1][threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        atomicAdd(out, red[0][0]);
        if (count) atomicAdd(out + 1, red[1][0]);
    }
}

template <typename SP>
__global__ void mass_apply_kernel(long long N, SP* phi, const int8_t* isf, const double* m) {
    if (m[1] <= 0.0) return;
    const double corr = (m[2] + m[3] - m[0]) / m[1];
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        if (isf) {
            const int f = isf[i];
            if (f != 1 && f != -1) continue;
        }
        const double v = (double)phi[i];
        if (v > 0.5 && v < 0.9) phi[i] = (SP)(v + corr);
    }
}

cudaError_t launch_mass(int storage, MassMode mode, long long N, void* phi, const int8_t* isf, double* d_mass,
                        cudaStream_t st) {
    const bool initial = mode == MASS_INITIAL;
    cudaError_t e = cudaMemsetAsync(initial ? d_mass + 2 : d_mass, 0, (initial ? 1 : 2) * sizeof(double), st);
    if (e != cudaSuccess) return e;
    return by_storage(storage, [&](auto tag) {
        using SP = typename PhiStore<decltype(tag)>::type;
        SP* f = static_cast<SP*>(phi);
        mass_sum_kernel<SP><<<blocks_for(N, 256), 256, 0, st>>>(N, f, isf, initial ? d_mass + 2 : d_mass, !initial);
        if (mode == MASS_APPLY) mass_apply_kernel<SP><<<blocks_for(N, 256), 256, 0, st>>>(N, f, isf, d_mass);
        return cudaGetLastError();
    });
}

cudaError_t launch_reduce(int storage, long long N, const void* mom, const float* pres, const void* phi,
                          const int8_t* isf, const double* inv_scale, double* d_out, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(d_out, 0, 5 * sizeof(double), st);
    if (e != cudaSuccess) return e;
    return by_storage(storage, [&](auto tag) {
        using S = decltype(tag);
        using SP = typename PhiStore<S>::type;
        reduce_kernel<S><<<blocks_for(N, 256), 256, 0, st>>>(N, static_cast<const S*>(mom), pres,
                                                              static_cast<const SP*>(phi), isf, inv_scale[0],
                                                              inv_scale[1], inv_scale[2], inv_scale[3], d_out);
        return cudaGetLastError();
    });
}

}  // namespace lbf
