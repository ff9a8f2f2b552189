// lbf_host.cpp -- host-side set-up and output of the LBFAST driver, behind
// the C ABI (include/lbfast_gpu.h): isfluid marking, initial conditions and
// the raw/XDMF writer.  These run once per run (or per output frame) on the
// CPU, as in the reference.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/lbfast_gpu.h"

namespace {
const int EXh[27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, 1, -1, -1, 1, 1, -1};
const int EYh[27] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, -1, 1, -1, 1};
const int EZh[27] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1};

inline long long lin(int i, int j, int k, int lx, int ly) { return ((long long)k * ly + j) * lx + i; }

// Fortran NINT: round half away from zero
inline double nint_f(double a) { return a >= 0 ? std::floor(a + 0.5) : -std::floor(-a + 0.5); }
}  // namespace

extern "C" {

// LBFAST.f90:258-325
int lbf_mark_isfluid(int lx, int ly, int lz, int pbc_x, int pbc_y, int pbc_z, int lattice, int obstacles,
                     const int8_t* raw, int8_t* out) {
    if (lx < 1 || ly < 1 || lz < 1 || !out) return LBF_E_ARG;
    if (lattice != 19 && lattice != 27) return LBF_E_UNSUPPORTED;
    const long long N = (long long)lx * ly * lz;
    std::vector<int8_t> isf(N);
    for (long long c = 0; c < N; ++c) isf[c] = raw ? (raw[c] != 0 ? 1 : 0) : 1;
    if (obstacles) {
        for (int k = 0; k < lz; ++k)
            for (int j = 0; j < ly; ++j)
                for (int i = 0; i < lx; ++i) {
                    bool wall = (!pbc_x && (i == 0 || i == lx - 1)) || (!pbc_y && (j == 0 || j == ly - 1)) ||
                                (!pbc_z && (k == 0 || k == lz - 1));
                    if (wall) isf[lin(i, j, k, lx, ly)] = 0;
                }
    }
    const int dims[3] = {lx, ly, lz};
    const int pb[3] = {pbc_x, pbc_y, pbc_z};
    const int nl = lattice == 27 ? 27 : 19;
    for (long long c = 0; c < N; ++c) out[c] = isf[c];
    for (int k = 0; k < lz; ++k)
        for (int j = 0; j < ly; ++j)
            for (int i = 0; i < lx; ++i) {
                long long c = lin(i, j, k, lx, ly);
                if (isf[c] != 1) continue;
                for (int l = 1; l < nl; ++l) {
                    int q[3] = {i + EXh[l], j + EYh[l], k + EZh[l]};
                    int v = 1;  // halo in a non-periodic direction keeps isfluid = 1
                    bool inside = true;
                    for (int d = 0; d < 3; ++d) {
                        if (q[d] < 0 || q[d] >= dims[d]) {
                            if (pb[d]) q[d] = (q[d] + dims[d]) % dims[d];
                            else inside = false;
                        }
                    }
                    if (inside) v = isf[lin(q[0], q[1], q[2], lx, ly)];
                    if (v != 1 && v != -1) out[c] = -1;
                }
            }
    return LBF_OK;
}

// init_conditions_module.f90:492-541
int lbf_seed_solid_phi(int lx, int ly, int lz, int lattice, const int8_t* isfluid, double* phi) {
    if (!isfluid || !phi) return LBF_E_ARG;
    const int nl = lattice == 27 ? 27 : 19;
    for (int k = 0; k < lz; ++k)
        for (int j = 0; j < ly; ++j)
            for (int i = 0; i < lx; ++i) {
                long long c = lin(i, j, k, lx, ly);
                if (isfluid[c] != 0) continue;
                double num = 0, den = 0;
                for (int l = 1; l < nl; ++l) {
                    int ni = i + EXh[l], nj = j + EYh[l], nk = k + EZh[l];
                    if (ni < 0 || ni >= lx || nj < 0 || nj >= ly || nk < 0 || nk >= lz) continue;
                    long long n = lin(ni, nj, nk, lx, ly);
                    if (isfluid[n] == 0) continue;
                    int d2 = EXh[l] * EXh[l] + EYh[l] * EYh[l] + EZh[l] * EZh[l];
                    double sc = d2 == 1 ? 1.0 : d2 == 2 ? 0.70710678118654752440 : 0.57735026918962576450;
                    num += sc * phi[n];
                    den += sc;
                }
                phi[c] = num / den;  // 0/0 (no fluid neighbour) stays NaN, as in the reference
            }
    return LBF_OK;
}

// init_conditions_module.f90:298-314
int lbf_ic_taylor_green(int lx, int ly, int lz, double u0, double* m) {
    if (!m) return LBF_E_ARG;
    const double pi = 3.1415926535897932384626433832795028841971;
    const long long N = (long long)lx * ly * lz;
    for (int k = 0; k < lz; ++k)
        for (int j = 0; j < ly; ++j)
            for (int i = 0; i < lx; ++i) {
                long long c = lin(i, j, k, lx, ly);
                double x = 2 * pi * i / lx, y = 2 * pi * j / ly, z = 2 * pi * k / lz;
                double u = u0 * std::sin(x) * std::cos(y) * std::cos(z);
                double v = -u0 * std::cos(x) * std::sin(y) * std::cos(z);
                double w = 0.0;
                double press = ((u0 * u0 / 16.0) * (std::cos(2 * x) + std::cos(2 * y)) * (2.0 + std::cos(2 * z))) /
                               (1.0 / 3.0);
                double vals[10] = {press, u, v, w, u * u, v * v, w * w, u * v, u * w, v * w};
                for (int f = 0; f < 10; ++f) m[f * N + c] = vals[f];
            }
    return LBF_OK;
}

// init_conditions_module.f90:394-426 with pbc_images (:591-600)
int lbf_ic_droplet(int lx, int ly, int lz, const double center[3], double radius, double width, double sigma,
                   double rho_r, double rho_b, int densratio, const int8_t* isfluid, double* m, double* phi) {
    if (!center || !m || !phi || radius <= 0 || width <= 0) return LBF_E_ARG;
    const long long N = (long long)lx * ly * lz;
    for (long long c = 0; c < 10 * N; ++c) m[c] = 0.0;
    for (long long c = 0; c < N; ++c) phi[c] = 0.0;
    for (int k = 0; k < lz; ++k)
        for (int j = 0; j < ly; ++j)
            for (int i = 0; i < lx; ++i) {
                long long c = lin(i, j, k, lx, ly);
                if (isfluid && isfluid[c] != 1 && isfluid[c] != -1) continue;
                double d[3] = {(i + 1) - center[0], (j + 1) - center[1], (k + 1) - center[2]};
                const int L[3] = {lx, ly, lz};
                for (int a = 0; a < 3; ++a) d[a] = d[a] - L[a] * nint_f(d[a] / L[a]);
                double r = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
                double ph = 0.5 * (1.0 - std::tanh((r - radius) / (0.5 * width)));
                double rp = densratio ? rho_r * ph + (1.0 - ph) * rho_b : 1.0;
                m[c] = ph * (sigma * 2.0) / radius / (rp * (1.0 / 3.0));
                phi[c] = ph;
            }
    return LBF_OK;
}

// print_raw_sync, print_module.f90:2007-2180 (float32 stream files + XDMF)
int lbf_write_raw_xdmf(const char* dir, int iframe, int lx, int ly, int lz, const float* rho, const float* vel,
                       const float* press) {
    if (!dir) return LBF_E_ARG;
    const long long N = (long long)lx * ly * lz;
    char num[16];
    std::snprintf(num, sizeof(num), "%06d", iframe < 0 ? 0 : (iframe > 999999 ? 999999 : iframe));
    const bool little = [] {
        unsigned int one = 1;
        return *reinterpret_cast<unsigned char*>(&one) == 1;
    }();
    struct Item {
        const char* name;
        const float* data;
        int ncomp;
        const char* grid;
        const char* attr;
    };
    const Item items[3] = {{"rho", rho, 1, "ScalarField", "Scalar"},
                           {"vel", vel, 3, "VelocityField", "Vector"},
                           {"press", press, 1, "ScalarField", "Scalar"}};
    for (const Item& it : items) {
        if (!it.data) continue;
        std::string base = std::string("out_") + it.name + "_" + num;
        std::string raw = std::string(dir) + "/" + base + ".raw";
        std::string xdmf = std::string(dir) + "/" + base + ".xdmf";
        FILE* f = std::fopen(raw.c_str(), "wb");
        if (!f) return LBF_E_IO;
        size_t w = std::fwrite(it.data, sizeof(float), (size_t)(N * it.ncomp), f);
        std::fclose(f);
        if (w != (size_t)(N * it.ncomp)) return LBF_E_IO;
        f = std::fopen(xdmf.c_str(), "w");
        if (!f) return LBF_E_IO;
        std::fprintf(f, "<?xml version=\"1.0\" ?>\n<Xdmf Version=\"3.0\">\n  <Domain>\n    <!-- Uniform Grid -->\n");
        std::fprintf(f, "    <Grid Name=\"%s\" GridType=\"Uniform\">\n\n", it.grid);
        std::fprintf(f, "      <!-- Topology: 3D grid -->\n");
        std::fprintf(f, "      <Topology TopologyType=\"3DCoRectMesh\" Dimensions=\"%d %d %d\"/>\n\n", lz, ly, lx);
        std::fprintf(f, "      <!-- Geometry: origin and spacing (dx, dy, dz) -->\n");
        std::fprintf(f, "      <Geometry GeometryType=\"ORIGIN_DXDYDZ\">\n");
        std::fprintf(f, "        <DataItem Dimensions=\"3\" Format=\"XML\" Precision=\"4\">0.0 0.0 0.0</DataItem>\n");
        std::fprintf(f, "        <DataItem Dimensions=\"3\" Format=\"XML\" Precision=\"4\">1.0 1.0 1.0</DataItem>\n");
        std::fprintf(f, "      </Geometry>\n\n");
        std::fprintf(f, "      <!-- %s field associated with the grid -->\n", it.attr);
        std::fprintf(f, "      <Attribute Name=\"%s\" AttributeType=\"%s\" Center=\"Node\">\n", it.name, it.attr);
        if (it.ncomp == 1)
            std::fprintf(f, "        <DataItem Format=\"Binary\" NumberType=\"Float\" Precision=\"4\" Dimensions=\"%d %d %d\" Endian=\"%s\">\n",
                         lz, ly, lx, little ? "Little" : "Big");
        else
            std::fprintf(f, "        <DataItem Format=\"Binary\" NumberType=\"Float\" Precision=\"4\" Dimensions=\"%d %d %d 3\" Endian=\"%s\">\n",
                         lz, ly, lx, little ? "Little" : "Big");
        std::fprintf(f, "          %s.raw\n        </DataItem>\n      </Attribute>\n\n    </Grid>\n  </Domain>\n</Xdmf>\n",
                     base.c_str());
        std::fclose(f);
    }
    return LBF_OK;
}

}  // extern "C"
