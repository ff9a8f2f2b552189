// lbf_host.cpp -- host-side set-up and output of the LBFAST driver, behind
// the C ABI (include/lbfast_gpu.h): isfluid marking, initial conditions and
// the raw/XDMF writer.  These run once per run (or per output frame) on the
// CPU, as in the reference.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/lbfast_gpu.h"

namespace {
const int EXh[27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, 1, -1, -1, 1, 1, -1};
const int EYh[27] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, -1, 1, -1, 1};
const int EZh[27] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1};

inline long long lin(int i, int j, int k, int lx, int ly) { return ((long long)k * ly + j) * lx + i; }

// is D3Q27 link l a link of the lattice: D3Q19 = links 0-18 (vars_module.f90:666-684),
// D3Q15 = links 0-6 and 19-26 (vars_module.f90:685-703), in the reference's order
inline bool link_in(int lat, int l) { return lat == 27 || (lat == 19 ? l < 19 : (l < 7 || l >= 19)); }

// Fortran NINT: round half away from zero
inline double nint_f(double a) { return a >= 0 ? std::floor(a + 0.5) : -std::floor(-a + 0.5); }
}  // namespace

extern "C" {

// LBFAST.f90:258-325
int lbf_mark_isfluid(int lx, int ly, int lz, int pbc_x, int pbc_y, int pbc_z, int lattice, int obstacles,
                     const int8_t* raw, int8_t* out) {
    if (lx < 1 || ly < 1 || lz < 1 || !out) return LBF_E_ARG;
    if (lattice != 15 && lattice != 19 && lattice != 27) return LBF_E_UNSUPPORTED;
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
    for (long long c = 0; c < N; ++c) out[c] = isf[c];
    for (int k = 0; k < lz; ++k)
        for (int j = 0; j < ly; ++j)
            for (int i = 0; i < lx; ++i) {
                long long c = lin(i, j, k, lx, ly);
                if (isf[c] != 1) continue;
                for (int l = 1; l < 27; ++l) {
                    if (!link_in(lattice, l)) continue;
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
    for (int k = 0; k < lz; ++k)
        for (int j = 0; j < ly; ++j)
            for (int i = 0; i < lx; ++i) {
                long long c = lin(i, j, k, lx, ly);
                if (isfluid[c] != 0) continue;
                double num = 0, den = 0;
                for (int l = 1; l < 27; ++l) {
                    if (!link_in(lattice, l)) continue;
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

}  // extern "C"

namespace {
// droplet of init_conditions_module.f90:355-426; xscale = 0.5 is the LAMBTEST
// ellipsoid (dist3dout(1)*HALF, :362)
int droplet(int lx, int ly, int lz, const double center[3], double radius, double width, double sigma,
            double rho_r, double rho_b, int densratio, const int8_t* isfluid, double* m, double* phi, double xscale) {
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
                d[0] *= xscale;
                double r = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
                double ph = 0.5 * (1.0 - std::tanh((r - radius) / (0.5 * width)));
                double rp = densratio ? rho_r * ph + (1.0 - ph) * rho_b : 1.0;
                m[c] = ph * (sigma * 2.0) / radius / (rp * (1.0 / 3.0));
                phi[c] = ph;
            }
    return LBF_OK;
}
}  // namespace

extern "C" {

// init_conditions_module.f90:394-426 with pbc_images (:591-600)
int lbf_ic_droplet(int lx, int ly, int lz, const double center[3], double radius, double width, double sigma,
                   double rho_r, double rho_b, int densratio, const int8_t* isfluid, double* m, double* phi) {
    return droplet(lx, ly, lz, center, radius, width, sigma, rho_r, rho_b, densratio, isfluid, m, phi, 1.0);
}

// init_conditions_module.f90:355-393
int lbf_ic_lamb(int lx, int ly, int lz, const double center[3], double radius, double width, double sigma,
                double rho_r, double rho_b, int densratio, const int8_t* isfluid, double* m, double* phi) {
    return droplet(lx, ly, lz, center, radius, width, sigma, rho_r, rho_b, densratio, isfluid, m, phi, 0.5);
}

}  // extern "C"

namespace {
// IEEE 754 binary32 -> binary16, round to nearest even (overflow to
// infinity, NaN kept quiet): the value the reference's real(kind=2) print
// arrays hold under PRINTHALF
uint16_t float_to_half_rne(float x) {
    uint32_t b;
    std::memcpy(&b, &x, sizeof b);
    const uint32_t sign = (b >> 16) & 0x8000u;
    const uint32_t ex = (b >> 23) & 0xffu;
    uint32_t man = b & 0x7fffffu;
    if (ex == 0xffu) return (uint16_t)(sign | 0x7c00u | (man ? 0x200u | (man >> 13) : 0u));
    const int e = (int)ex - 127 + 15;  // biased binary16 exponent
    if (e >= 31) return (uint16_t)(sign | 0x7c00u);
    if (e <= 0) {
        // subnormal (or zero) in binary16: shift the full significand
        if (e < -10) return (uint16_t)sign;
        man |= 0x800000u;
        const int shift = 14 - e;  // 24-bit significand -> 10-bit field
        uint32_t h = man >> shift;
        const uint32_t rem = man & ((1u << shift) - 1u), half = 1u << (shift - 1);
        if (rem > half || (rem == half && (h & 1u))) ++h;
        return (uint16_t)(sign | h);
    }
    uint32_t h = ((uint32_t)e << 10) | (man >> 13);
    const uint32_t rem = man & 0x1fffu;
    if (rem > 0x1000u || (rem == 0x1000u && (h & 1u))) ++h;  // a carry into the exponent is correct
    return (uint16_t)(sign | h);
}

std::vector<uint16_t> to_half(const float* d, long long n) {
    std::vector<uint16_t> out((size_t)n);
    for (long long i = 0; i < n; ++i) out[(size_t)i] = float_to_half_rne(d[i]);
    return out;
}

// print_raw_sync, print_module.f90:2007-2180 (float32 stream files + XDMF;
// PRINTHALF: binary16 bit patterns, declared UInt of precision 2)
int write_raw_xdmf(const char* dir, int iframe, int lx, int ly, int lz, const float* rho, const float* vel,
                   const float* press, bool half) {
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
        size_t w;
        if (half) {
            const std::vector<uint16_t> h16 = to_half(it.data, N * it.ncomp);
            w = std::fwrite(h16.data(), sizeof(uint16_t), h16.size(), f);
        } else {
            w = std::fwrite(it.data, sizeof(float), (size_t)(N * it.ncomp), f);
        }
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
        const char* ntype = half ? "UInt" : "Float";
        const int prec = half ? 2 : 4;
        if (it.ncomp == 1)
            std::fprintf(f, "        <DataItem Format=\"Binary\" NumberType=\"%s\" Precision=\"%d\" Dimensions=\"%d %d %d\" Endian=\"%s\">\n",
                         ntype, prec, lz, ly, lx, little ? "Little" : "Big");
        else
            std::fprintf(f, "        <DataItem Format=\"Binary\" NumberType=\"%s\" Precision=\"%d\" Dimensions=\"%d %d %d 3\" Endian=\"%s\">\n",
                         ntype, prec, lz, ly, lx, little ? "Little" : "Big");
        std::fprintf(f, "          %s.raw\n        </DataItem>\n      </Attribute>\n\n    </Grid>\n  </Domain>\n</Xdmf>\n",
                     base.c_str());
        std::fclose(f);
    }
    return LBF_OK;
}
}  // namespace

extern "C" {

int lbf_write_raw_xdmf(const char* dir, int iframe, int lx, int ly, int lz, const float* rho, const float* vel,
                       const float* press) {
    return write_raw_xdmf(dir, iframe, lx, ly, lz, rho, vel, press, false);
}

int lbf_write_raw_xdmf_half(const char* dir, int iframe, int lx, int ly, int lz, const float* rho, const float* vel,
                            const float* press) {
    return write_raw_xdmf(dir, iframe, lx, ly, lz, rho, vel, press, true);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Fortran namelist reader for the reference's `simulation` / `fluid` groups
// (LBFAST.f90:32-60): `&group`, `key = value[, value...]`, `!` comments,
// `.true.` / `.false.`, reals with e or d exponents, terminated by `&end` or `/`.
// ---------------------------------------------------------------------------
namespace {

std::string lower(std::string s) {
    for (char& c : s) c = (char)std::tolower((unsigned char)c);
    return s;
}
std::string trim(const std::string& s) {
    size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
    return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
}

struct NmlError {
    std::string msg;
};

// one assignment: key, raw values, first element index (key(i) = ..., 1 otherwise)
struct NmlItem {
    std::string first;
    std::vector<std::string> second;
    int idx;
};

// split "a = 1, b = 2.0" style text into key -> list of raw values
std::vector<NmlItem> parse_group(const std::string& body) {
    std::vector<NmlItem> out;
    // tokens separated by commas / whitespace; a key is a token followed by '='
    std::string s = body;
    for (char& c : s)
        if (c == '\n' || c == '\r' || c == '\t') c = ' ';
    size_t i = 0;
    std::string key;
    std::vector<std::string> vals;
    int idx = 1;
    auto flush = [&]() {
        if (!key.empty()) out.push_back({key, vals, idx});
        key.clear();
        vals.clear();
        idx = 1;
    };
    while (i < s.size()) {
        while (i < s.size() && (s[i] == ' ' || s[i] == ',')) ++i;
        if (i >= s.size()) break;
        size_t j = i;
        while (j < s.size() && s[j] != ' ' && s[j] != ',' && s[j] != '=') ++j;
        std::string tok = s.substr(i, j - i);
        size_t k = j;
        while (k < s.size() && s[k] == ' ') ++k;
        if (k < s.size() && s[k] == '=') {
            flush();
            key = lower(tok);
            size_t p = key.find('(');
            if (p != std::string::npos) {  // element assignment key(i)=
                const size_t q = key.find(')');
                const std::string e = key.substr(p + 1, q == std::string::npos ? std::string::npos : q - p - 1);
                char* end = nullptr;
                const long v = std::strtol(e.c_str(), &end, 10);
                if (end == e.c_str() || *end != '\0') throw NmlError{"bad element index in `" + tok + "`"};
                idx = (int)v;
                key = key.substr(0, p);
            }
            i = k + 1;
        } else {
            if (key.empty()) throw NmlError{"value `" + tok + "` without a key"};
            vals.push_back(tok);
            i = j;
        }
    }
    flush();
    return out;
}

double to_real(const std::string& v, const std::string& key) {
    std::string t = lower(v);
    std::replace(t.begin(), t.end(), 'd', 'e');
    char* end = nullptr;
    double x = std::strtod(t.c_str(), &end);
    if (end == t.c_str() || *end != '\0') throw NmlError{"bad real `" + v + "` for " + key};
    return x;
}
int to_int(const std::string& v, const std::string& key) {
    char* end = nullptr;
    long x = std::strtol(v.c_str(), &end, 10);
    if (end == v.c_str() || *end != '\0') throw NmlError{"bad integer `" + v + "` for " + key};
    return (int)x;
}
int to_bool(const std::string& v, const std::string& key) {
    std::string t = lower(v);
    if (t == ".true." || t == "t" || t == ".t.") return 1;
    if (t == ".false." || t == "f" || t == ".f.") return 0;
    throw NmlError{"bad logical `" + v + "` for " + key};
}

// body of group `name` (text between `&name` and `&end` or `/`), comments removed
std::string group_body(const std::string& text, const std::string& name) {
    std::istringstream in(text);
    std::string line, body;
    bool inside = false;
    while (std::getline(in, line)) {
        size_t c = line.find('!');
        if (c != std::string::npos) line = line.substr(0, c);
        std::string t = lower(trim(line));
        if (!inside) {
            if (t.rfind("&" + name, 0) == 0) {
                inside = true;
                body += line.substr(line.find('&') + 1 + name.size()) + "\n";
            }
            continue;
        }
        if (t.rfind("&end", 0) == 0 || t == "/") return body;
        size_t slash = line.find('/');
        if (slash != std::string::npos) return body + line.substr(0, slash);
        body += line + "\n";
    }
    if (!inside) throw NmlError{"namelist group &" + name + " not found"};
    throw NmlError{"namelist group &" + name + " is not terminated"};
}

}  // namespace

extern "C" int lbf_read_namelists(const char* path, lbf_params* p, lbf_run* run) {
    if (!path || !p || !run) return LBF_E_ARG;
    std::ifstream f(path);
    if (!f) {
        std::fprintf(stderr, "lbf_read_namelists: cannot open %s\n", path);
        return LBF_E_IO;
    }
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string text = ss.str();
    // DOBENCHMARK defaults, LBFAST.f90:159-191
    run->nsteps = 100; run->stamp = 100; run->stamp2D = 10; run->stamp_term = 2147483647; run->stepskip = 1;
    run->lreadisfluid = 0; run->lreadinit = 0; run->lprint = 1; run->lvtk = 0; run->lraw = 1; run->lrestart = 0;
    run->lwriterestart = 0; run->openbc = 0; run->nplanes = 0; run->every_time_check = 1000;
    run->iprobe = run->jprobe = run->kprobe = 0;
    run->time_limit = -1.0;
    run->uwall = 0.0;
    run->width = 0.0;
    run->center[0] = run->center[1] = run->center[2] = 0.0;
    p->lx = p->ly = p->lz = 512;
    p->pbc_x = p->pbc_y = p->pbc_z = 1;
    p->fx = p->fy = p->fz = 0.0;
    p->rho_r = p->rho_b = 1.0;  // vars_module.f90:775
    p->visc1 = p->visc2 = 0.0;
    p->sigma = 0.0;
    p->width = 0.0;
    p->tau_diff = 0.0;
    p->wettab_r = 90.0;
    p->openbc = 0;  // vars_module.f90:238-255
    p->a_rep = p->cos_opp_t = p->q_th = 0.0;
    for (int a = 0; a < 3; ++a)
        for (int sd = 0; sd < 2; ++sd) {
            p->openbc_type[a][sd] = 0;
            p->openbc_press[a][sd] = 0.0;
            for (int d = 0; d < 3; ++d) p->openbc_vel[a][sd][d] = 0.0;
        }
    try {
        for (auto& kv : parse_group(group_body(text, "simulation"))) {
            const std::string& k = kv.first;
            const auto& v = kv.second;
            if (v.empty()) throw NmlError{"no value for " + k};
            const std::string& a = v[0];
            if (k == "nsteps") run->nsteps = to_int(a, k);
            else if (k == "stamp") run->stamp = to_int(a, k);
            else if (k == "stamp2d") run->stamp2D = to_int(a, k);
            else if (k == "stamp_term") run->stamp_term = to_int(a, k);
            else if (k == "stepskip") run->stepskip = to_int(a, k);
            else if (k == "lreadisfluid") run->lreadisfluid = to_bool(a, k);
            else if (k == "lreadinit") run->lreadinit = to_bool(a, k);
            else if (k == "lx") p->lx = to_int(a, k);
            else if (k == "ly") p->ly = to_int(a, k);
            else if (k == "lz") p->lz = to_int(a, k);
            else if (k == "lprint") run->lprint = to_bool(a, k);
            else if (k == "lvtk") run->lvtk = to_bool(a, k);
            else if (k == "lraw") run->lraw = to_bool(a, k);
            else if (k == "lrestart") run->lrestart = to_bool(a, k);
            else if (k == "lwriterestart") run->lwriterestart = to_bool(a, k);
            else if (k == "pbc_x") p->pbc_x = to_int(a, k);
            else if (k == "pbc_y") p->pbc_y = to_int(a, k);
            else if (k == "pbc_z") p->pbc_z = to_int(a, k);
            else if (k == "openbc") { run->openbc = to_int(a, k); p->openbc = run->openbc; }
            else if (k == "iprobe") run->iprobe = to_int(a, k);
            else if (k == "jprobe") run->jprobe = to_int(a, k);
            else if (k == "kprobe") run->kprobe = to_int(a, k);
            else if (k == "nplanes") run->nplanes = to_int(a, k);
            else if (k == "time_limit") run->time_limit = to_real(a, k);
            else if (k == "every_time_check") run->every_time_check = to_int(a, k);
            else if (k == "lasync" || k == "lweakscaling") to_bool(a, k);
            else if (k.rfind("openbc_", 0) == 0 && k.size() >= 9 && k[k.size() - 2] == '_' &&
                     (k.back() == 'x' || k.back() == 'y' || k.back() == 'z')) {
                // openbc_type_x(2), openbc_press_y(2), openbc_u_z(2), ... (vars_module.f90:240-255)
                const int axis = k.back() - 'x';
                const std::string what = k.substr(7, k.size() - 9);
                for (size_t m = 0; m < v.size(); ++m) {
                    const int side = kv.idx - 1 + (int)m;
                    if (side < 0 || side > 1) throw NmlError{"element out of range (1:2) for " + k};
                    if (what == "type") p->openbc_type[axis][side] = to_int(v[m], k);
                    else if (what == "press") p->openbc_press[axis][side] = to_real(v[m], k);
                    else if (what == "u") p->openbc_vel[axis][side][0] = to_real(v[m], k);
                    else if (what == "v") p->openbc_vel[axis][side][1] = to_real(v[m], k);
                    else if (what == "w") p->openbc_vel[axis][side][2] = to_real(v[m], k);
                    else throw NmlError{"unknown key `" + k + "` in &simulation"};
                }
            }
            else throw NmlError{"unknown key `" + k + "` in &simulation"};
        }
        bool have_radius = false;
        for (auto& kv : parse_group(group_body(text, "fluid"))) {
            const std::string& k = kv.first;
            const auto& v = kv.second;
            if (v.empty()) throw NmlError{"no value for " + k};
            const std::string& a = v[0];
            if (k == "fx") p->fx = to_real(a, k);
            else if (k == "fy") p->fy = to_real(a, k);
            else if (k == "fz") p->fz = to_real(a, k);
            else if (k == "visc1") p->visc1 = to_real(a, k);
            else if (k == "visc2") p->visc2 = to_real(a, k);
            else if (k == "radius") { run->radius = to_real(a, k); have_radius = true; }
            else if (k == "width") { run->width = to_real(a, k); p->width = run->width; }
            else if (k == "center") {
                if (v.size() != 3) throw NmlError{"center needs 3 values"};
                for (int d = 0; d < 3; ++d) run->center[d] = to_real(v[d], k);
            } else if (k == "tau_diff") p->tau_diff = to_real(a, k);
            else if (k == "sigma") p->sigma = to_real(a, k);
            else if (k == "wettab_r") p->wettab_r = to_real(a, k);
            else if (k == "rho_r") p->rho_r = to_real(a, k);
            else if (k == "rho_b") p->rho_b = to_real(a, k);
            else if (k == "uwall") run->uwall = to_real(a, k);
            else if (k == "a_rep") p->a_rep = to_real(a, k);  // REPULSIVE_FLUX (LBFAST.f90:57-58)
            else if (k == "cosoppt") p->cos_opp_t = to_real(a, k);
            else if (k == "q_th") p->q_th = to_real(a, k);
            else if (k == "wettab_b" || k == "mu_max" || k == "ks" || k == "k_elastic" || k == "lambda_rel" ||
                     k == "rhoin" || k == "rhoout") {
                for (auto& x : v) to_real(x, k);
            } else if (k == "npoint" || k == "ndir") { for (auto& x : v) to_int(x, k); }
            else throw NmlError{"unknown key `" + k + "` in &fluid"};
        }
        if (!have_radius) run->radius = p->lx / 4;  // DOBENCHMARK: radius = lx/4 (integer division)
    } catch (const NmlError& e) {
        std::fprintf(stderr, "lbf_read_namelists: %s: %s\n", path, e.msg.c_str());
        return LBF_E_ARG;
    }
    return LBF_OK;
}

// ---- VTK ImageData (print_module.f90:22-244 header_vtk / footer_vtk, 2789-2814) ----
// One .vti file per variable: a fixed-width XML header whose last byte is the
// '_' that opens the appended raw data, the data byte count as int32, the
// float32 values (vectors interleaved per node), and a 30-byte footer.
namespace {
std::string rjust(long long v, int w) {
    std::string s = std::to_string(v);
    return s.size() >= (size_t)w ? s : std::string(w - s.size(), ' ') + s;
}

int write_vti(const std::string& path, const char* name8, int ncomp, int lx, int ly, int lz, const float* data,
              bool half) {
    const long long N = (long long)lx * ly * lz;
    const std::string ext = rjust(1, 6) + " " + rjust(lx, 6) + " " + rjust(1, 6) + " " + rjust(ly, 6) + " " +
                            rjust(1, 6) + " " + rjust(lz, 6);
    // the reference assigns each line to a fixed-width field (padding with blanks)
    auto field = [](std::string s, size_t w) {
        s.resize(w - 1, ' ');
        return s + '\n';
    };
    std::string h;
    h += field("<?xml version=\"1.0\"?>", 22);
    h += field("<VTKFile type=\"ImageData\" version=\"0.1\" byte_order=\"LittleEndian\">", 67);
    h += field("  <ImageData WholeExtent=\"" + ext + "\">", 70);
    h += field("    <Piece Extent=\"" + ext + "\">", 63);
    h += field("      <PointData>", 18);
    // PRINTHALF declares the binary16 bit patterns as UnsignedShort (a field of 121)
    h += field(std::string("        <DataArray type=\"") + (half ? "UnsignedShort" : "Float32") + "\" Name=\"" + name8 +
                   "\" NumberOfComponents=\"" + std::to_string(ncomp) + "\" format=\"appended\" offset=\"" +
                   rjust(0, 12) + "\"/>",
               half ? 121 : 115);
    h += field("      </PointData>", 19);
    h += field("    </Piece>", 13);
    h += field("  </ImageData>", 15);
    h += field("  <AppendedData encoding=\"raw\">", 32);
    h += "_";
    const std::string foot = std::string("\n") + "  </AppendedData>\n" + "</VTKFile>\n";
    std::FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return LBF_E_IO;
    const int32_t nbytes = (int32_t)(ncomp * N * (long long)(half ? sizeof(uint16_t) : sizeof(float)));
    bool ok = std::fwrite(h.data(), 1, h.size(), f) == h.size();
    ok = ok && std::fwrite(&nbytes, sizeof nbytes, 1, f) == 1;
    if (half) {
        const std::vector<uint16_t> h16 = to_half(data, ncomp * N);
        ok = ok && std::fwrite(h16.data(), sizeof(uint16_t), h16.size(), f) == h16.size();
    } else {
        ok = ok && std::fwrite(data, sizeof(float), ncomp * N, f) == (size_t)(ncomp * N);
    }
    ok = ok && std::fwrite(foot.data(), 1, foot.size(), f) == foot.size();
    if (std::fclose(f) != 0) ok = false;
    return ok ? LBF_OK : LBF_E_IO;
}
}  // namespace

namespace {
int write_vtk(const char* dir, int iframe, int lx, int ly, int lz, const float* rho, const float* vel,
              const float* press, bool half) {
    if (!dir || !rho || !vel || lx < 1 || ly < 1 || lz < 1) return LBF_E_ARG;
    char num[16];
    std::snprintf(num, sizeof(num), "%06d", iframe < 0 ? 0 : (iframe > 999999 ? 999999 : iframe));
    std::string d = dir;
    if (!d.empty() && d.back() != '/') d += '/';
    int rc = write_vti(d + "out_rho_" + num + ".vti", "rho     ", 1, lx, ly, lz, rho, half);
    if (rc == LBF_OK) rc = write_vti(d + "out_vel_" + num + ".vti", "vel     ", 3, lx, ly, lz, vel, half);
    if (rc == LBF_OK && press) rc = write_vti(d + "out_press_" + num + ".vti", "press   ", 1, lx, ly, lz, press, half);
    return rc;
}
}  // namespace

int lbf_write_vtk(const char* dir, int iframe, int lx, int ly, int lz, const float* rho, const float* vel,
                  const float* press) {
    return write_vtk(dir, iframe, lx, ly, lz, rho, vel, press, false);
}

int lbf_write_vtk_half(const char* dir, int iframe, int lx, int ly, int lz, const float* rho, const float* vel,
                       const float* press) {
    return write_vtk(dir, iframe, lx, ly, lz, rho, vel, press, true);
}

// ---- restart.raw (print_module.f90:1030-1474 and 1474-1677) ----
// The reference's restart is one time level in float32, stream-unformatted:
// the ten moment fields in the order of its hfields indices 1,2,3,4,5,8,9,6,10,7
// (P, u, v, w, Pxx, Pxy, Pxz, Pyy, Pyz, Pzz), then phi for two components, then
// iframe and iframe2D as int32.  mom10 here is ordered P, u, v, w, Pxx, Pyy,
// Pzz, Pxy, Pxz, Pyz.
namespace {
const int kRestartOrder[10] = {0, 1, 2, 3, 4, 7, 8, 5, 9, 6};

std::string restart_path(const char* dir) {
    std::string d = dir ? dir : ".";
    if (!d.empty() && d.back() != '/') d += '/';
    return d + "restart.raw";
}
}  // namespace

int lbf_write_restart_raw(const char* dir, int lx, int ly, int lz, const float* mom10, const float* phi, int iframe,
                          int iframe2D) {
    if (!mom10 || lx < 1 || ly < 1 || lz < 1) return LBF_E_ARG;
    const long long N = (long long)lx * ly * lz;
    std::FILE* f = std::fopen(restart_path(dir).c_str(), "wb");
    if (!f) return LBF_E_IO;
    bool ok = true;
    for (int k = 0; k < 10 && ok; ++k) ok = std::fwrite(mom10 + kRestartOrder[k] * N, sizeof(float), N, f) == (size_t)N;
    if (ok && phi) ok = std::fwrite(phi, sizeof(float), N, f) == (size_t)N;
    const int32_t fr[2] = {iframe, iframe2D};
    if (ok) ok = std::fwrite(fr, sizeof(int32_t), 2, f) == 2;
    if (std::fclose(f) != 0) ok = false;
    return ok ? LBF_OK : LBF_E_IO;
}

int lbf_read_restart_raw(const char* dir, int lx, int ly, int lz, float* mom10, float* phi, int* iframe,
                         int* iframe2D) {
    if (!mom10 || lx < 1 || ly < 1 || lz < 1) return LBF_E_ARG;
    const long long N = (long long)lx * ly * lz;
    std::FILE* f = std::fopen(restart_path(dir).c_str(), "rb");
    if (!f) return LBF_E_IO;
    std::fseek(f, 0, SEEK_END);
    const long long size = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    const long long want = (long long)sizeof(float) * N * (phi ? 11 : 10) + 8;
    bool ok = size == want;
    for (int k = 0; k < 10 && ok; ++k) ok = std::fread(mom10 + kRestartOrder[k] * N, sizeof(float), N, f) == (size_t)N;
    if (ok && phi) ok = std::fread(phi, sizeof(float), N, f) == (size_t)N;
    int32_t fr[2] = {0, 0};
    if (ok) ok = std::fread(fr, sizeof(int32_t), 2, f) == 2;
    std::fclose(f);
    if (!ok) return LBF_E_IO;
    if (iframe) *iframe = fr[0];
    if (iframe2D) *iframe2D = fr[1];
    return LBF_OK;
}
