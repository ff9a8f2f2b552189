// lbfast_main.cpp -- driver program in the shape of LBFAST.f90 on top of the
// C ABI (include/lbfast_gpu.h).
//
//   lbfast [-DLATTICE=15|19|27] [-DHIGHORDER] [-DTWOCOMPONENT] [-DDENSRATIO]
//          [-DINTERNAL_OBSTACLES] [-DWETTABILITY] [-DPRINTPHI] [-DWRITEPRESS] [-DSMAGORINSKI] [-DBOUNCE_BACK]
//          [-DREPULSIVE_FLUX]
//          [-DTAYLORGREEN|-DLAPLACE|-DLAMBTEST] [--storage=f32|f16|bf16|f64]
//          input.inp
//
// The reference selects physics with compile-time macros (defines.h:1-74); here
// the same names are run-time flags, with the implications of defines.h:38-74
// (LAPLACE and LAMBTEST imply TWOCOMPONENT, DENSRATIO, PRINTPHI, WRITEPRESS;
// TAYLORGREEN implies one component).  The run follows LBFAST.f90:193-533 and
// integrator_module.f90:82-863: namelists, isfluid (isfluid.raw when
// lreadisfluid, walls at non-periodic faces with INTERNAL_OBSTACLES, -1
// marking), initial fields of the DOBENCHMARK branch (or rho/u/v/w/phi.raw
// when lreadinit), the time loop with copy_print + raw/XDMF output every
// `stamp` steps and the probe line every `stamp_term` steps, the wall-clock
// time limit, and the GLUPS report.
#include <sys/stat.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "lbfast_gpu.h"

namespace {

struct Flags {
    int lattice = 27;
    bool highorder = false, twocomponent = false, densratio = false, obstacles = false;
    bool printphi = false, writepress = false, wettability = false, smagorinsky = false, bounce_back = false;
    bool repulsive = false;
    bool taylorgreen = false, laplace = false, lambtest = false;
    int storage = LBF_STORE_F32;
    std::string input;
};

void die(const char* what, int rc) {
    char buf[512];
    lbf_last_error(buf, sizeof(buf));
    std::fprintf(stderr, "lbfast: %s failed (%d): %s\n", what, rc, buf);
    std::exit(1);
}

#define CHECK(call)                  \
    do {                             \
        int rc_ = (call);            \
        if (rc_ != LBF_OK) die(#call, rc_); \
    } while (0)

bool read_f32(const char* path, std::vector<float>& out) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return false;
    size_t n = std::fread(out.data(), sizeof(float), out.size(), f);
    std::fclose(f);
    return n == out.size();
}

Flags parse_flags(int argc, char** argv) {
    Flags fl;
    for (int i = 1; i < argc; ++i) {
        std::string a = argv[i];
        if (a == "-DLATTICE=27") fl.lattice = 27;
        else if (a == "-DLATTICE=19") fl.lattice = 19;
        else if (a == "-DLATTICE=15") fl.lattice = 15;
        else if (a == "-DHIGHORDER") fl.highorder = true;
        else if (a == "-DTWOCOMPONENT") fl.twocomponent = true;
        else if (a == "-DDENSRATIO") fl.densratio = true;
        else if (a == "-DINTERNAL_OBSTACLES") fl.obstacles = true;
        else if (a == "-DWETTABILITY") fl.wettability = true;
        else if (a == "-DSMAGORINSKI") fl.smagorinsky = true;
        else if (a == "-DBOUNCE_BACK") fl.bounce_back = true;
        else if (a == "-DREPULSIVE_FLUX") fl.repulsive = true;
        else if (a == "-DPRINTPHI") fl.printphi = true;
        else if (a == "-DWRITEPRESS") fl.writepress = true;
        else if (a == "-DTAYLORGREEN") fl.taylorgreen = true;
        else if (a == "-DLAPLACE") fl.laplace = true;
        else if (a == "-DLAMBTEST") fl.lambtest = true;
        else if (a.rfind("--storage=", 0) == 0) {
            std::string s = a.substr(10);
            fl.storage = s == "f16" ? LBF_STORE_F16 : s == "bf16" ? LBF_STORE_BF16 : s == "f64" ? LBF_STORE_F64 : LBF_STORE_F32;
        } else if (!a.empty() && a[0] != '-') fl.input = a;
        else {
            std::fprintf(stderr, "lbfast: unknown option %s\n", a.c_str());
            std::exit(2);
        }
    }
    if (fl.input.empty()) {
        std::fprintf(stderr, "the command line should be\n[executable] [flags] [input]\n");
        std::exit(2);
    }
    // defines.h:38-74
    if (fl.laplace || fl.lambtest) fl.twocomponent = fl.densratio = fl.printphi = fl.writepress = true;
    if (fl.taylorgreen) fl.twocomponent = fl.densratio = false;
    if (fl.highorder && fl.lattice != 27) {
        std::fprintf(stderr, "HIGHORDER: if the macro HIGHORDER is defined you MUST USE LATTICE 27\n");
        std::exit(2);
    }
    if (fl.densratio && !fl.twocomponent) fl.densratio = false;
    return fl;
}

}  // namespace

int main(int argc, char** argv) {
    Flags fl = parse_flags(argc, argv);
    lbf_params p;
    std::memset(&p, 0, sizeof(p));
    p.lattice = fl.lattice;
    p.highorder = fl.highorder;
    p.twocomponent = fl.twocomponent;
    p.densratio = fl.densratio;
    p.obstacles = fl.obstacles;
    p.storage = fl.storage;
    p.printphi = fl.printphi;
    p.smagorinsky = fl.smagorinsky;
    p.bounce_back = fl.bounce_back;
    p.repulsive_flux = fl.repulsive;
    p.visc2 = 0.0;
    p.wettab_r = 90.0;
    lbf_run run;
    CHECK(lbf_read_namelists(fl.input.c_str(), &p, &run));
    if (!p.twocomponent) p.visc2 = p.visc1;
    // without WETTABILITY the reference's wetting uses a 90 degree contact angle
    // (lb_cuda_boundary_module.f90:264,275) whatever the namelist says
    if (!fl.wettability) p.wettab_r = 90.0;
    const int lx = p.lx, ly = p.ly, lz = p.lz;
    const long long N = (long long)lx * ly * lz;
    std::printf("file  = %s\n", fl.input.c_str());
    std::printf("lbfast-b200 %s: D3Q%d%s, %s component(s), box %d x %d x %d\n", lbf_version(), p.lattice,
                p.highorder ? " high-order" : "", p.twocomponent ? "two" : "one", lx, ly, lz);

    // ---- geometry: LBFAST.f90:258-325 ----
    std::vector<int8_t> raw(N, 1), isf(N);
    if (run.lreadisfluid) {
        std::vector<float> a(N);
        if (!read_f32("isfluid.raw", a)) {
            std::fprintf(stderr, "ERROR: unable to read the file: isfluid.raw\n");
            return 1;
        }
        for (long long c = 0; c < N; ++c) raw[c] = (int8_t)(int)a[c];
    }
    if (!fl.obstacles) std::fill(raw.begin(), raw.end(), 1);  // LBFAST.f90:298-300
    CHECK(lbf_mark_isfluid(lx, ly, lz, p.pbc_x, p.pbc_y, p.pbc_z, p.lattice, p.obstacles, raw.data(), isf.data()));

    // ---- initial fields: init_conditions_module.f90:177-541 ----
    std::vector<double> mom(10 * N, 0.0), phi(N, 0.0);
    if (fl.taylorgreen) {
        CHECK(lbf_ic_taylor_green(lx, ly, lz, run.uwall, mom.data()));
    } else if (fl.lambtest) {
        CHECK(lbf_ic_lamb(lx, ly, lz, run.center, run.radius, run.width, p.sigma, p.rho_r, p.rho_b, p.densratio,
                          isf.data(), mom.data(), phi.data()));
    } else {
        CHECK(lbf_ic_droplet(lx, ly, lz, run.center, run.radius, run.width > 0 ? run.width : 1.0,
                             p.twocomponent ? p.sigma : 0.0, p.rho_r, p.rho_b, p.densratio, isf.data(), mom.data(),
                             phi.data()));
        if (!p.twocomponent) {
            // one-component branch: loc_press = 0.01 * fcut_tanh(...) (:443-448)
            for (long long c = 0; c < N; ++c) mom[c] = 0.01 * phi[c];
        }
    }
    if (p.obstacles && p.twocomponent) CHECK(lbf_seed_solid_phi(lx, ly, lz, p.lattice, isf.data(), phi.data()));
    if (run.lreadinit) {
        std::vector<float> a(N);
        const char* names[5] = {"rho.raw", "u.raw", "v.raw", "w.raw", "phi.raw"};
        for (int f = 0; f < (p.twocomponent ? 5 : 4); ++f) {
            if (!read_f32(names[f], a)) {
                std::fprintf(stderr, "ERROR: unable to read the file: %s\n", names[f]);
                return 1;
            }
            double* dst = f < 4 ? mom.data() + (long long)f * N : phi.data();
            for (long long c = 0; c < N; ++c) dst[c] = a[c];
        }
    }

    // ---- restart: integrator_module.f90:167-176 (replaces the initial fields) ----
    int iframe = 0, iframe2D = 0;
    if (run.lrestart) {
        std::vector<float> m32(10 * N), p32(N);
        if (lbf_read_restart_raw("output", lx, ly, lz, m32.data(), p.twocomponent ? p32.data() : nullptr, &iframe,
                                 &iframe2D) != LBF_OK) {
            std::fprintf(stderr, "ERROR: unable to read the file: output/restart.raw\n");
            return 1;
        }
        std::copy(m32.begin(), m32.end(), mom.begin());
        if (p.twocomponent) std::copy(p32.begin(), p32.end(), phi.begin());
        std::printf("restart read: iframe %d\n", iframe);
    }

    lbf_handle* h = nullptr;
    CHECK(lbf_create(&p, &h));
    if (p.obstacles) CHECK(lbf_set_isfluid(h, isf.data()));
    CHECK(lbf_set_fields(h, mom.data(), p.twocomponent ? phi.data() : nullptr, LBF_F64));

    // ---- output set-up: print_module.f90:277-445 ----
    std::vector<float> rho(N), vel(3 * N), press(N);
    const bool do_raw = run.lprint && run.lraw;
    const bool do_vtk = run.lprint && run.lvtk;
    if (do_raw || do_vtk || run.lwriterestart) mkdir("output", 0755);
    if (run.nplanes > 0) std::fprintf(stderr, "lbfast: nplanes ignored (2-D plane output is not provided)\n");
    if (run.lprint && !run.lrestart) {
        CHECK(lbf_get_print_fields(h, rho.data(), vel.data(), press.data()));
        if (do_raw)
            CHECK(lbf_write_raw_xdmf("output", iframe, lx, ly, lz, rho.data(), vel.data(),
                                     fl.writepress && p.twocomponent ? press.data() : nullptr));
        if (do_vtk)
            CHECK(lbf_write_vtk("output", iframe, lx, ly, lz, rho.data(), vel.data(),
                                fl.writepress && p.twocomponent ? press.data() : nullptr));
    }

    // ---- time loop: integrator_module.f90:266-827 (steps come in FLIP/FLOP pairs) ----
    const int nsteps = run.nsteps + (run.nsteps % 2);
    CHECK(lbf_sync(h));
    auto t0 = std::chrono::steady_clock::now();
    for (int step = 1; step <= nsteps; ++step) {
        CHECK(lbf_step(h, 1));
        const bool at_stamp = run.stamp > 0 && step % run.stamp == 0;
        const bool at_term = run.stamp_term > 0 && step % run.stamp_term == 0;
        if (run.lprint && (at_stamp || at_term)) {
            CHECK(lbf_get_print_fields(h, rho.data(), vel.data(), press.data()));
            if (at_stamp) {
                ++iframe;
                if (do_raw)
                    CHECK(lbf_write_raw_xdmf("output", iframe, lx, ly, lz, rho.data(), vel.data(),
                                             fl.writepress && p.twocomponent ? press.data() : nullptr));
                if (do_vtk)
                    CHECK(lbf_write_vtk("output", iframe, lx, ly, lz, rho.data(), vel.data(),
                                        fl.writepress && p.twocomponent ? press.data() : nullptr));
            }
            if (at_term) {
                int i = run.iprobe - 1, j = run.jprobe - 1, k = run.kprobe - 1;
                if (i >= 0 && i < lx && j >= 0 && j < ly && k >= 0 && k < lz) {
                    long long c = ((long long)k * ly + j) * lx + i;
                    std::printf("stamp step : %6d %6d%6d%6d; probe values : %2d %16.8g %16.8g %16.8g %16.8g\n", step,
                                run.iprobe, run.jprobe, run.kprobe, isf[c], rho[c], vel[3 * c], vel[3 * c + 1],
                                vel[3 * c + 2]);
                }
            }
        }
        if (run.time_limit > 0 && run.every_time_check > 0 && step % run.every_time_check == 0) {
            CHECK(lbf_sync(h));
            double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            if (el > run.time_limit) {
                std::printf("Time limit %16.2f sec reached at step %16d after %16.2f sec\n", run.time_limit, step, el);
                run.lwriterestart = 1;  // integrator_module.f90:819
                break;
            }
        }
    }
    CHECK(lbf_sync(h));
    double tot = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    double glups = (double)lx * ly * lz * (double)run.nsteps / tot * 1e-9;  // LBFAST.f90:499-500
    double sums[5];
    CHECK(lbf_reduce(h, sums));
    // ---- write restart: integrator_module.f90:834-840 ----
    if (run.lwriterestart) {
        std::vector<float> m32(10 * N), p32(N);
        CHECK(lbf_get_fields(h, m32.data(), p.twocomponent ? p32.data() : nullptr, nullptr, LBF_F32));
        CHECK(lbf_write_restart_raw("output", lx, ly, lz, m32.data(), p.twocomponent ? p32.data() : nullptr, iframe,
                                    iframe2D));
    }
    std::printf(" time elapsed: %g s\n", tot);
    std::printf(" glups: %g\n", glups);
    std::printf(" sums (phi, P, u, v, w): %.12g %.12g %.12g %.12g %.12g\n", sums[0], sums[1], sums[2], sums[3], sums[4]);
    CHECK(lbf_destroy(h));
    std::printf("program correctly closed\n");
    return 0;
}
