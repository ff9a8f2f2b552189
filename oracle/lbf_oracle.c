/*
 * lbf_oracle.c -- CPU restatement of the LBFAST per-timestep path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA path in
 * lbfast_b200/csrc: it is built by oracle/Makefile and loaded only by
 * tests/, __graft_entry__.smoke() and the CPU-baseline leg of bench.py.
 * Nothing in the product links, loads or calls it.
 *
 * Parity status: UNPINNED against a reference binary.  The reference is
 * CUDA Fortran + OpenACC (lauricella/LBFAST) and no Fortran compiler exists
 * on this machine or on the GPU hosts, and the reference ships no golden
 * vectors or tests.  This restatement is pinned instead against the
 * reference's own analytic benchmark checks (statistics.f90: Taylor-Green
 * viscous decay, Laplace pressure jump), against the reference's D3Q27
 * Minv_mrt table (tests/golden/minv_mrt.npy, parsed from vars_module.f90)
 * and against mass/momentum invariants.
 *
 * What it restates (reference file:line, paths within the LBFAST project):
 *   step order            integrator_module.f90:266-544 (FLIP; FLOP swaps buffers)
 *   pre-loop wetting      integrator_module.f90:186-190
 *   periodic halo copy    mpi_module.f90:646-710, 2203-2274 (one node layer)
 *   compute_norm          lb_cuda_auxfields_module.f90:19-139
 *   div(theta)            lb_cuda_auxfields_module.f90:1085-1164
 *   wetting ghost phi     lb_cuda_boundary_module.f90:218-459
 *   moments (force, u, Pi) lb_cuda_moments_module.f90:19-341
 *   fused collide+stream  lb_cuda_fused_module.f90:426-750
 *   update_phi            lb_cuda_update_phi_module.f90:19-104
 *   obstacle bounce-back  lb_cuda_boundary_module.f90:19-216
 *   BOUNCE_BACK           lb_cuda_fused_module.f90:20-424 (half-way, in the streaming)
 *   REPULSIVE_FLUX        lb_cuda_repulsive_module.f90:19-292; lb_cuda_moments_module.f90:148-160
 *   open boundaries       boundary_cds_module.f90:57-1311 (moments), 1351-1663 (phi), 1667-1885 (flux)
 *   copy_print            print_module.f90:638-776
 *   lattice tables        vars_module.f90:319-338 (D3Q27), 666-684 (D3Q19), 685-703 (D3Q15)
 *   parameter derivation  LBFAST.f90:212-219
 *
 * The fields live on a padded grid with one halo layer (the reference's
 * halo tiles, minus the tiling).  Periodic directions are wrapped by
 * explicit halo copies at the same points of the step where the reference
 * calls exchange_*_intpbc; non-periodic halos keep isfluid = 1 and zero
 * field values, as the reference's never-written halo memory does.
 *
 * Built twice: REAL=double (the FP64 oracle) and REAL=float (the stand-in
 * for the reference's PRC 4 build).  Per-node arithmetic follows the
 * reference's expression order.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifndef REAL
#define REAL double
#endif
typedef REAL real;

#ifdef _OPENMP
#include <omp.h>
#endif
#if defined(__x86_64__) || defined(__i386__)
#include <xmmintrin.h>
/* Flush-to-zero / denormals-are-zero during a step, as an x86 host build with
 * nvfortran's default -Mflushz runs: at rest the high-order terms multiply up
 * to six tiny velocities, and subnormal arithmetic on x86 is two orders of
 * magnitude slower.  Set in every OpenMP thread (MXCSR is per thread). */
#define FTZ_ON() _mm_setcsr(_mm_getcsr() | 0x8040)
#else
#define FTZ_ON() ((void)0)
#endif

typedef struct orc_params {
    int lx, ly, lz;
    int pbc_x, pbc_y, pbc_z;
    int lattice;     /* 15, 19 or 27 */
    int highorder;   /* HIGHORDER (LATTICE 27 only) */
    int twocomp;     /* TWOCOMPONENT */
    int densratio;   /* DENSRATIO (implies INTERFACE_INCOMP) */
    int obstacles;   /* INTERNAL_OBSTACLES */
    double visc1, visc2, rho_r, rho_b, sigma, width, tau_diff;
    double fx, fy, fz;
    double wettab_r;
    int phi_correction; /* phi mass correction of every step's input phi (see mass_correction) */
    int smagorinsky;    /* SMAGORINSKI LES relaxation time (see smag_omega) */
    /* open boundaries (openbc = 1, INTERNAL_OBSTACLES): per axis x, y, z and
     * side (low, high) the openbc_type_x/y/z, openbc_press_x/y/z and
     * (openbc_u, openbc_v, openbc_w)_x/y/z values of the input file
     * (vars_module.f90:238-255); see open_face */
    int openbc;
    int obc_type[3][2];
    double obc_press[3][2];
    double obc_vel[3][2][3];
    int bounce_back; /* BOUNCE_BACK: half-way bounce-back in the fused kernel (see fused) */
    /* REPULSIVE_FLUX (see repulsive): switch and the A_rep, cosOppT, q_th of
     * the input file (LBFAST.f90:57-58) */
    int repulsive;
    double a_rep, cos_opp_t, q_th;
} orc_params;

/* ---- lattice tables: vars_module.f90:319-338 (D3Q27), 666-684 (D3Q19), 685-703 (D3Q15) ---- */
static const int ex27[27] = {0, 1,-1, 0, 0, 0, 0, 1,-1, 1,-1, 0, 0, 0, 0, 1,-1,-1, 1, 1,-1, 1,-1,-1, 1, 1,-1};
static const int ey27[27] = {0, 0, 0, 1,-1, 0, 0, 1,-1,-1, 1, 1,-1, 1,-1, 0, 0, 0, 0, 1,-1,-1, 1,-1, 1,-1, 1};
static const int ez27[27] = {0, 0, 0, 0, 0, 1,-1, 0, 0, 0, 0, 1,-1,-1, 1, 1,-1, 1,-1, 1,-1, 1,-1, 1,-1,-1, 1};
static const int opp27[27] = {0, 2, 1, 4, 3, 6, 5, 8, 7,10, 9,12,11,14,13,16,15,18,17,20,19,22,21,24,23,26,25};

typedef struct orc_state {
    orc_params p;
    int nx, ny, nz, NX, NY, NZ;
    long npad;
    int nl;                    /* links incl. rest: 15, 19 or 27 */
    int ex[27], ey[27], ez[27], opp[27];
    real w[27];
    real minv[27][27];         /* minv[r][l] = Minv_mrt(r,l) */
    /* derived parameters, computed in `real` as the reference does */
    real omega, beta, kapp, sharp_c, visc1, visc2, rho_r, rho_b, tau_diff, fx, fy, fz, wettab_r;
    int8_t *isf;
    real *h[2][10];
    real *phi[2];
    real *aux[7];
    real *loc[2];
    real *frc[3];
    real *rep[3];              /* REPULSIVE_FLUX force of the step (locauxfields 6-8) */
    int flip;                  /* index of the buffer that is the input of the next step */
    double phi_sum0;           /* sum of phi over fluid nodes at the first step */
    long step;
    int primed;
    /* copy_print of the last executed step (or of the primed initial state) */
    real *prt_rho, *prt_vel[3], *prt_press;
} orc_state;

static inline long IDX(const orc_state *s, int i, int j, int k)
{
    return ((long)(k + 1) * s->NY + (j + 1)) * s->NX + (i + 1);
}

/* Hermite basis of the D3Q27 Minv_mrt table: r -> axis multiplicities. */
static const int hmul[27][3] = {
    {0,0,0},{1,0,0},{0,1,0},{0,0,1},{2,0,0},{0,2,0},{0,0,2},{1,1,0},{1,0,1},{0,1,1},
    {2,1,0},{2,0,1},{1,2,0},{1,0,2},{0,1,2},{0,2,1},{1,1,1},{2,2,0},{2,0,2},{0,2,2},
    {1,1,2},{1,2,1},{2,1,1},{2,1,2},{2,2,1},{1,2,2},{2,2,2}};

static double herm1(int m, int c)
{
    if (m == 0) return 1.0;
    if (m == 1) return (double)c;
    return (double)(c * c) - 1.0 / 3.0;
}

static void build_tables(orc_state *s)
{
    int l, r;
    if (s->p.lattice == 27) {
        s->nl = 27;
        for (l = 0; l < 27; l++) {
            s->ex[l] = ex27[l]; s->ey[l] = ey27[l]; s->ez[l] = ez27[l]; s->opp[l] = opp27[l];
        }
        for (l = 0; l < 27; l++) {
            int n2 = ex27[l] * ex27[l] + ey27[l] * ey27[l] + ez27[l] * ez27[l];
            s->w[l] = (real)(n2 == 0 ? 8.0 / 27.0 : n2 == 1 ? 2.0 / 27.0 : n2 == 2 ? 1.0 / 54.0 : 1.0 / 216.0);
        }
    } else if (s->p.lattice == 19) {
        /* D3Q19 is the first 19 links of the D3Q27 ordering (vars_module.f90:670-680) */
        s->nl = 19;
        for (l = 0; l < 19; l++) {
            s->ex[l] = ex27[l]; s->ey[l] = ey27[l]; s->ez[l] = ez27[l]; s->opp[l] = opp27[l];
            int n2 = ex27[l] * ex27[l] + ey27[l] * ey27[l] + ez27[l] * ez27[l];
            s->w[l] = (real)(n2 == 0 ? 1.0 / 3.0 : n2 == 1 ? 1.0 / 18.0 : 1.0 / 36.0);
        }
    } else {
        /* D3Q15 (vars_module.f90:685-703): rest, faces and corners, in the
         * reference's order, which is the D3Q27 order of those links; opposite
         * pairs stay adjacent (opp = 0,2,1,4,3,...) */
        static const int l15[15] = {0, 1, 2, 3, 4, 5, 6, 19, 20, 21, 22, 23, 24, 25, 26};
        s->nl = 15;
        for (l = 0; l < 15; l++) {
            int m = l15[l];
            s->ex[l] = ex27[m]; s->ey[l] = ey27[m]; s->ez[l] = ez27[m];
            s->opp[l] = l == 0 ? 0 : (l % 2 ? l + 1 : l - 1);
            int n2 = ex27[m] * ex27[m] + ey27[m] * ey27[m] + ez27[m] * ez27[m];
            s->w[l] = (real)(n2 == 0 ? 2.0 / 9.0 : n2 == 1 ? 1.0 / 9.0 : 1.0 / 72.0);
        }
    }
    /* Minv_mrt(r,l) = w_l H_r(c_l) / <H_r,H_r>_w  (vars_module.f90:360-521, checked
     * element by element against the reference table in the tests) */
    for (r = 0; r < 27; r++) {
        double nrm = 1.0;
        int d;
        for (d = 0; d < 3; d++) nrm *= (hmul[r][d] == 0 ? 1.0 : hmul[r][d] == 1 ? 1.0 / 3.0 : 2.0 / 9.0);
        for (l = 0; l < 27; l++) {
            double wl = (double)((ex27[l] * ex27[l] + ey27[l] * ey27[l] + ez27[l] * ez27[l]) == 0 ? 8.0 / 27.0 :
                                 (ex27[l] * ex27[l] + ey27[l] * ey27[l] + ez27[l] * ez27[l]) == 1 ? 2.0 / 27.0 :
                                 (ex27[l] * ex27[l] + ey27[l] * ey27[l] + ez27[l] * ez27[l]) == 2 ? 1.0 / 54.0 : 1.0 / 216.0);
            double H = herm1(hmul[r][0], ex27[l]) * herm1(hmul[r][1], ey27[l]) * herm1(hmul[r][2], ez27[l]);
            s->minv[r][l] = (real)(wl * H / nrm);
        }
    }
}

/* The link table of a lattice as the oracle builds it: returns the number of
 * links (0 for an unknown lattice) and fills ex, ey, ez, opp, w (27 each). */
int orc_lattice_table(int lattice, int *ex, int *ey, int *ez, int *opp, double *w)
{
    orc_state s;
    int l;
    if (lattice != 15 && lattice != 19 && lattice != 27) return 0;
    memset(&s, 0, sizeof(s));
    s.p.lattice = lattice;
    build_tables(&s);
    for (l = 0; l < s.nl; l++) {
        ex[l] = s.ex[l]; ey[l] = s.ey[l]; ez[l] = s.ez[l]; opp[l] = s.opp[l];
        w[l] = (double)s.w[l];
    }
    return s.nl;
}

void orc_minv_table(double *out /* 27*27, out[r*27+l] */)
{
    orc_state s;
    int r, l;
    memset(&s, 0, sizeof(s));
    s.p.lattice = 27;
    build_tables(&s);
    for (r = 0; r < 27; r++)
        for (l = 0; l < 27; l++) out[r * 27 + l] = (double)s.minv[r][l];
}

static real *zalloc(long n)
{
    real *p = (real *)calloc((size_t)n, sizeof(real));
    return p;
}

orc_state *orc_create(const orc_params *p)
{
    orc_state *s = (orc_state *)calloc(1, sizeof(orc_state));
    int f, b;
    if (!s) return NULL;
    s->p = *p;
    s->nx = p->lx; s->ny = p->ly; s->nz = p->lz;
    s->NX = s->nx + 2; s->NY = s->ny + 2; s->NZ = s->nz + 2;
    s->npad = (long)s->NX * s->NY * s->NZ;
    build_tables(s);
    /* LBFAST.f90:212-219, evaluated in the working precision */
    s->visc1 = (real)p->visc1; s->visc2 = (real)p->visc2;
    s->rho_r = (real)p->rho_r; s->rho_b = (real)p->rho_b;
    s->tau_diff = (real)p->tau_diff;
    s->fx = (real)p->fx; s->fy = (real)p->fy; s->fz = (real)p->fz;
    s->wettab_r = (real)p->wettab_r;
    {
        real tau1 = s->visc1 * (real)3.0 + (real)0.5;
        real sig = (real)p->sigma, wid = (real)p->width;
        s->omega = (real)1.0 / tau1;
        s->beta = (real)12.0 * sig / wid;
        s->kapp = (real)1.5 * sig * wid;
        s->sharp_c = (real)4.0 * s->tau_diff / wid;
    }
    s->isf = (int8_t *)malloc((size_t)s->npad);
    memset(s->isf, 1, (size_t)s->npad);
    for (b = 0; b < 2; b++) {
        for (f = 0; f < 10; f++) s->h[b][f] = zalloc(s->npad);
        s->phi[b] = zalloc(s->npad);
    }
    for (f = 0; f < 7; f++) s->aux[f] = zalloc(s->npad);
    for (f = 0; f < 2; f++) s->loc[f] = zalloc(s->npad);
    for (f = 0; f < 3; f++) s->frc[f] = zalloc(s->npad);
    for (f = 0; f < 3; f++) s->rep[f] = zalloc(s->npad);
    s->prt_rho = zalloc(s->npad);
    s->prt_press = zalloc(s->npad);
    for (f = 0; f < 3; f++) s->prt_vel[f] = zalloc(s->npad);
    s->flip = 0;
    return s;
}

void orc_destroy(orc_state *s)
{
    int f, b;
    if (!s) return;
    free(s->isf);
    for (b = 0; b < 2; b++) {
        for (f = 0; f < 10; f++) free(s->h[b][f]);
        free(s->phi[b]);
    }
    for (f = 0; f < 7; f++) free(s->aux[f]);
    for (f = 0; f < 2; f++) free(s->loc[f]);
    for (f = 0; f < 3; f++) free(s->frc[f]);
    for (f = 0; f < 3; f++) free(s->rep[f]);
    free(s->prt_rho); free(s->prt_press);
    for (f = 0; f < 3; f++) free(s->prt_vel[f]);
    free(s);
}

/* ---- periodic halo copy: mpi_module.f90:646-710 + exchange_*_intpbc ---- */
static void halo_real(const orc_state *s, real *a)
{
    int nx = s->nx, ny = s->ny, nz = s->nz, i, j, k;
    if (s->p.pbc_x)
        for (k = 0; k < nz; k++)
            for (j = 0; j < ny; j++) {
                a[IDX(s, -1, j, k)] = a[IDX(s, nx - 1, j, k)];
                a[IDX(s, nx, j, k)] = a[IDX(s, 0, j, k)];
            }
    if (s->p.pbc_y)
        for (k = 0; k < nz; k++)
            for (i = -1; i <= nx; i++) {
                a[IDX(s, i, -1, k)] = a[IDX(s, i, ny - 1, k)];
                a[IDX(s, i, ny, k)] = a[IDX(s, i, 0, k)];
            }
    if (s->p.pbc_z)
        for (j = -1; j <= ny; j++)
            for (i = -1; i <= nx; i++) {
                a[IDX(s, i, j, -1)] = a[IDX(s, i, j, nz - 1)];
                a[IDX(s, i, j, nz)] = a[IDX(s, i, j, 0)];
            }
}

static void halo_i8(const orc_state *s, int8_t *a)
{
    int nx = s->nx, ny = s->ny, nz = s->nz, i, j, k;
    if (s->p.pbc_x)
        for (k = 0; k < nz; k++)
            for (j = 0; j < ny; j++) {
                a[IDX(s, -1, j, k)] = a[IDX(s, nx - 1, j, k)];
                a[IDX(s, nx, j, k)] = a[IDX(s, 0, j, k)];
            }
    if (s->p.pbc_y)
        for (k = 0; k < nz; k++)
            for (i = -1; i <= nx; i++) {
                a[IDX(s, i, -1, k)] = a[IDX(s, i, ny - 1, k)];
                a[IDX(s, i, ny, k)] = a[IDX(s, i, 0, k)];
            }
    if (s->p.pbc_z)
        for (j = -1; j <= ny; j++)
            for (i = -1; i <= nx; i++) {
                a[IDX(s, i, j, -1)] = a[IDX(s, i, j, nz - 1)];
                a[IDX(s, i, j, nz)] = a[IDX(s, i, j, 0)];
            }
}

/* isfluid of the interior in Fortran order (i fastest), values {1,-1,0} as
 * produced by LBFAST.f90:258-325. */
void orc_set_isfluid(orc_state *s, const int8_t *isf)
{
    int i, j, k;
    memset(s->isf, 1, (size_t)s->npad);
    for (k = 0; k < s->nz; k++)
        for (j = 0; j < s->ny; j++)
            for (i = 0; i < s->nx; i++)
                s->isf[IDX(s, i, j, k)] = isf[((long)k * s->ny + j) * s->nx + i];
    halo_i8(s, s->isf);
}

/* Initial state: h10 = 10 moments (P,u,v,w,Pxx,Pyy,Pzz,Pxy,Pxz,Pyz), each a
 * Fortran-order interior array; phi likewise (ignored for one component).
 * Both buffers receive the same values (init_conditions_module.f90:584-587). */
void orc_set_fields(orc_state *s, const double *h10, const double *phi)
{
    long n = (long)s->nx * s->ny * s->nz;
    int i, j, k, f, b;
    for (b = 0; b < 2; b++) {
        for (f = 0; f < 10; f++) memset(s->h[b][f], 0, sizeof(real) * (size_t)s->npad);
        memset(s->phi[b], 0, sizeof(real) * (size_t)s->npad);
    }
    for (f = 0; f < 7; f++) memset(s->aux[f], 0, sizeof(real) * (size_t)s->npad);
    for (f = 0; f < 2; f++) memset(s->loc[f], 0, sizeof(real) * (size_t)s->npad);
    for (f = 0; f < 3; f++) memset(s->frc[f], 0, sizeof(real) * (size_t)s->npad);
    for (k = 0; k < s->nz; k++)
        for (j = 0; j < s->ny; j++)
            for (i = 0; i < s->nx; i++) {
                long src = ((long)k * s->ny + j) * s->nx + i, dst = IDX(s, i, j, k);
                for (b = 0; b < 2; b++) {
                    for (f = 0; f < 10; f++) s->h[b][f][dst] = (real)h10[f * n + src];
                    if (s->p.twocomp && phi) s->phi[b][dst] = (real)phi[src];
                }
            }
    s->flip = 0;
    s->step = 0;
    s->primed = 0;
}

/* ---------------- kernels ---------------- */

static inline real phi_at(const real *a, long c) { return a[c]; }

/* compute_norm_interface_kernel: lb_cuda_auxfields_module.f90:19-139 */
static void compute_norm(orc_state *s, const real *ph)
{
    const long sx = 1, sy = s->NX, sz = (long)s->NX * s->NY;
    const real p1 = (real)(2.0 / 27.0), p2 = (real)(1.0 / 54.0), p3 = (real)(1.0 / 216.0), p0 = (real)(8.0 / 27.0);
    int k;
#pragma omp parallel for schedule(static)
    for (k = 0; k < s->nz; k++) {
        int i, j;
        for (j = 0; j < s->ny; j++)
            for (i = 0; i < s->nx; i++) {
                long c = IDX(s, i, j, k);
                if (abs(s->isf[c]) != 1) continue;
#define M(a, b, d) ph[c + (a) * sx + (b) * sy + (d) * sz]
                real gx = (real)3.0 * (p1 * (M(1, 0, 0) - M(-1, 0, 0)) +
                                       p2 * ((M(1, 1, 0) - M(-1, -1, 0)) + (M(1, -1, 0) - M(-1, 1, 0)) +
                                             (M(1, 0, 1) - M(-1, 0, -1)) + (M(1, 0, -1) - M(-1, 0, 1))) +
                                       p3 * ((M(1, 1, 1) - M(-1, -1, -1)) + (M(1, -1, -1) - M(-1, 1, 1)) +
                                             (M(1, -1, 1) - M(-1, 1, -1)) + (M(1, 1, -1) - M(-1, -1, 1))));
                real gy = (real)3.0 * (p1 * (M(0, 1, 0) - M(0, -1, 0)) +
                                       p2 * ((M(1, 1, 0) - M(-1, -1, 0)) + (M(-1, 1, 0) - M(1, -1, 0)) +
                                             (M(0, 1, 1) - M(0, -1, -1)) + (M(0, 1, -1) - M(0, -1, 1))) +
                                       p3 * ((M(1, 1, 1) - M(-1, -1, -1)) + (M(-1, 1, -1) - M(1, -1, 1)) +
                                             (M(1, 1, -1) - M(-1, -1, 1)) + (M(-1, 1, 1) - M(1, -1, -1))));
                real gz = (real)3.0 * (p1 * (M(0, 0, 1) - M(0, 0, -1)) +
                                       p2 * ((M(1, 0, 1) - M(-1, 0, -1)) + (M(-1, 0, 1) - M(1, 0, -1)) +
                                             (M(0, 1, 1) - M(0, -1, -1)) + (M(0, -1, 1) - M(0, 1, -1))) +
                                       p3 * ((M(1, 1, 1) - M(-1, -1, -1)) + (M(-1, -1, 1) - M(1, 1, -1)) +
                                             (M(1, -1, 1) - M(-1, 1, -1)) + (M(-1, 1, 1) - M(1, -1, -1))));
                real mg = (real)sqrt(gx * gx + gy * gy + gz * gz);
                real inv = mg + (real)1.0e-9;
                real c0 = M(0, 0, 0);
                s->aux[0][c] = gx / inv;
                s->aux[1][c] = gy / inv;
                s->aux[2][c] = gz / inv;
                s->aux[3][c] = mg;
                s->aux[4][c] = c0 * ((real)1.0 - c0) * (gx / inv);
                s->aux[5][c] = c0 * ((real)1.0 - c0) * (gy / inv);
                s->aux[6][c] = c0 * ((real)1.0 - c0) * (gz / inv);
                s->loc[0][c] = ((real)2.0 * (real)3.0) *
                    (c0 * (p0 - (real)1.0) +
                     (p1 * (M(1, 0, 0) + M(-1, 0, 0) + M(0, 1, 0) + M(0, -1, 0) + M(0, 0, 1) + M(0, 0, -1)) +
                      p2 * ((M(1, 1, 0) + M(-1, -1, 0)) + (M(1, -1, 0) + M(-1, 1, 0)) + (M(1, 0, 1) + M(-1, 0, -1)) +
                            (M(1, 0, -1) + M(-1, 0, 1)) + (M(0, 1, 1) + M(0, -1, -1)) + (M(0, 1, -1) + M(0, -1, 1))) +
                      p3 * ((M(1, 1, 1) + M(-1, -1, -1)) + (M(1, -1, -1) + M(-1, 1, 1)) + (M(1, -1, 1) + M(-1, 1, -1)) +
                            (M(1, 1, -1) + M(-1, -1, 1)))));
#undef M
            }
    }
}

/* compute_div_theta_n_kernel: lb_cuda_auxfields_module.f90:1085-1164 */
static void compute_div_theta(orc_state *s)
{
    const long sx = 1, sy = s->NX, sz = (long)s->NX * s->NY;
    const real p1 = (real)(2.0 / 27.0), p2 = (real)(1.0 / 54.0), p3 = (real)(1.0 / 216.0);
    const real *ax = s->aux[4], *ay = s->aux[5], *az = s->aux[6];
    int k;
#pragma omp parallel for schedule(static)
    for (k = 0; k < s->nz; k++) {
        int i, j;
        for (j = 0; j < s->ny; j++)
            for (i = 0; i < s->nx; i++) {
                long c = IDX(s, i, j, k);
                if (abs(s->isf[c]) != 1) continue;
#define X(a, b, d) ax[c + (a) * sx + (b) * sy + (d) * sz]
#define Y(a, b, d) ay[c + (a) * sx + (b) * sy + (d) * sz]
#define Z(a, b, d) az[c + (a) * sx + (b) * sy + (d) * sz]
                real dx = p1 * (X(1, 0, 0) - X(-1, 0, 0)) +
                          p2 * ((X(1, 1, 0) - X(-1, -1, 0)) + (X(1, -1, 0) - X(-1, 1, 0)) +
                                (X(1, 0, 1) - X(-1, 0, -1)) + (X(1, 0, -1) - X(-1, 0, 1))) +
                          p3 * ((X(1, 1, 1) - X(-1, -1, -1)) + (X(1, -1, -1) - X(-1, 1, 1)) +
                                (X(1, -1, 1) - X(-1, 1, -1)) + (X(1, 1, -1) - X(-1, -1, 1)));
                real dy = p1 * (Y(0, 1, 0) - Y(0, -1, 0)) +
                          p2 * ((Y(1, 1, 0) - Y(-1, -1, 0)) + (Y(-1, 1, 0) - Y(1, -1, 0)) +
                                (Y(0, 1, 1) - Y(0, -1, -1)) + (Y(0, 1, -1) - Y(0, -1, 1))) +
                          p3 * ((Y(1, 1, 1) - Y(-1, -1, -1)) + (Y(-1, 1, -1) - Y(1, -1, 1)) +
                                (Y(1, 1, -1) - Y(-1, -1, 1)) + (Y(-1, 1, 1) - Y(1, -1, -1)));
                real dz = p1 * (Z(0, 0, 1) - Z(0, 0, -1)) +
                          p2 * ((Z(1, 0, 1) - Z(-1, 0, -1)) + (Z(-1, 0, 1) - Z(1, 0, -1)) +
                                (Z(0, 1, 1) - Z(0, -1, -1)) + (Z(0, -1, 1) - Z(0, 1, -1))) +
                          p3 * ((Z(1, 1, 1) - Z(-1, -1, -1)) + (Z(-1, -1, 1) - Z(1, 1, -1)) +
                                (Z(1, -1, 1) - Z(-1, 1, -1)) + (Z(-1, 1, 1) - Z(1, -1, -1)));
                s->loc[1][c] = (dx + dy + dz) * (real)3.0;
#undef X
#undef Y
#undef Z
            }
    }
}

/* PHI_int_boundary_kernel: lb_cuda_boundary_module.f90:218-459.  Runs on the
 * solid nodes of the interior; reads the node's own phi, its neighbours'
 * isfluid, the donor's phi and aux1-4; writes the node's phi. */
static void wetting(orc_state *s, real *ph)
{
    const double eps_norm = 1.0e-14, huge_cot = 1.0e14;
    const double inv_sqrt2 = 0.70710678118654752440, inv_sqrt3 = 0.57735026918962576450;
    const double pi_greek = 3.1415926535897932384626433832795028841971;
    int k;
#pragma omp parallel for schedule(static)
    for (k = 0; k < s->nz; k++) {
        int i, j, l;
        for (j = 0; j < s->ny; j++)
            for (i = 0; i < s->nx; i++) {
                long c = IDX(s, i, j, k);
                if (s->isf[c] != 0) continue;
                real phi_ghost = ph[c];
                real wnx = 0, wny = 0, wnz = 0;
                for (l = 1; l < s->nl; l++) {
                    int d2 = s->ex[l] * s->ex[l] + s->ey[l] * s->ey[l] + s->ez[l] * s->ez[l];
                    if (s->isf[IDX(s, i + s->ex[l], j + s->ey[l], k + s->ez[l])] == 0) continue;
                    real sc = d2 == 1 ? (real)1.0 : d2 == 2 ? (real)0.5 : (real)(1.0 / 3.0);
                    wnx = wnx + sc * (real)(-s->ex[l]);
                    wny = wny + sc * (real)(-s->ey[l]);
                    wnz = wnz + sc * (real)(-s->ez[l]);
                }
                real wn = (real)sqrt(wnx * wnx + wny * wny + wnz * wnz);
                if (wn < (real)eps_norm) continue;
                wnx = wnx / wn; wny = wny / wn; wnz = wnz / wn;
                real best = (real)-1.0e30;
                int di = 0, dj = 0, dk = 0, found = 0;
                real bsx = 0, bsy = 0, bsz = 0;
                for (l = 1; l < s->nl; l++) {
                    int d2 = s->ex[l] * s->ex[l] + s->ey[l] * s->ey[l] + s->ez[l] * s->ez[l];
                    int ni = i + s->ex[l], nj = j + s->ey[l], nk = k + s->ez[l];
                    if (abs(s->isf[IDX(s, ni, nj, nk)]) != 1) continue;
                    real sc = d2 == 1 ? (real)1.0 : d2 == 2 ? (real)inv_sqrt2 : (real)inv_sqrt3;
                    real shx = (real)(-s->ex[l]), shy = (real)(-s->ey[l]), shz = (real)(-s->ez[l]);
                    real score = (shx * wnx + shy * wny + shz * wnz) * sc;
                    if (score > best) {
                        best = score; di = ni; dj = nj; dk = nk; found = 1;
                        bsx = shx; bsy = shy; bsz = shz;
                    }
                }
                /* reference: `if (donor_x==0 .or. donor_y==0 .or. donor_z==0) return` in
                 * 1-based local indices: no donor, or a donor on the low halo layer */
                if (!found || di == -1 || dj == -1 || dk == -1) continue;
                long dc = IDX(s, di, dj, dk);
                real phi_fluid = ph[dc];
                real mg = s->aux[3][dc];
                real gx = s->aux[0][dc] * mg, gy = s->aux[1][dc] * mg, gz = s->aux[2][dc] * mg;
                real gdw = gx * wnx + gy * wny + gz * wnz;
                real tx = gx - gdw * wnx, ty = gy - gdw * wny, tz = gz - gdw * wnz;
                real tmag = (real)sqrt(tx * tx + ty * ty + tz * tz);
                real th = ((real)180.0 - s->wettab_r) * (real)pi_greek / (real)180.0;
                real st = (real)sin(th), ct = (real)cos(th);
                real cot = fabs((double)st) < eps_norm ? (ct >= 0 ? (real)huge_cot : (real)-huge_cot) : ct / st;
                real dn = -tmag * cot;
                real bx = tx + dn * wnx, by = ty + dn * wny, bz = tz + dn * wnz;
                phi_ghost = phi_fluid + (bx * bsx + by * bsy + bz * bsz) * ((real)4.0 * phi_ghost * ((real)1.0 - phi_ghost));
                if (phi_ghost > (real)1.0) phi_ghost = (real)1.0;
                if (phi_ghost < (real)0.0) phi_ghost = (real)0.0;
                ph[c] = phi_ghost;
            }
    }
}

/* index of node (i, j, k) folded into the box on periodic axes; -1 beyond a
 * non-periodic face (the reference's halo layers there: isfluid 1, phi 0,
 * aux 0) */
static long wrap_index(const orc_state *s, int i, int j, int k)
{
    int c[3] = {i, j, k}, d;
    const int n[3] = {s->nx, s->ny, s->nz}, pb[3] = {s->p.pbc_x, s->p.pbc_y, s->p.pbc_z};
    for (d = 0; d < 3; d++)
        if (c[d] < 0 || c[d] >= n[d]) {
            if (!pb[d]) return -1;
            c[d] = ((c[d] % n[d]) + n[d]) % n[d];
        }
    return IDX(s, c[0], c[1], c[2]);
}

/* REPULSIVE_FLUX: thinfilm_scan_mark_kernel and repulsive_flux_normal_kernel
 * (lb_cuda_repulsive_module.f90:19-292), on the step's phi and the normals of
 * compute_norm (aux 1-3).  An interfacial fluid node (q = phi (1 - phi) of
 * the clamped phi >= q_th) looks in the window of +-3 nodes (LBFAST.f90:221)
 * for the nearest fluid node of similar q (within 10 %) whose normal faces its
 * own (n1 . n2 <= cosOppT), ties to the larger facing factor; the pair gives a
 * force along the bisector of the two normals, of strength
 * A_rep / (1 + W^4) qcl face with W = width arcosh(1 / (2 sqrt(qcl))) the
 * film thickness, capped by phi / (1.5 |F|_1). */
static void repulsive(orc_state *s, const real *ph)
{
    const double eps = 1.0e-9, q_th = s->p.q_th;
    int k;
#pragma omp parallel for schedule(static)
    for (k = 0; k < s->nz; k++) {
        int i, j, d;
        for (j = 0; j < s->ny; j++)
            for (i = 0; i < s->nx; i++) {
                long c = IDX(s, i, j, k);
                if (abs(s->isf[c]) != 1) continue;
                for (d = 0; d < 3; d++) s->rep[d][c] = 0;
                /* scan and mark (lb_cuda_repulsive_module.f90:63-150) */
                double qloc = (double)ph[c];
                qloc = qloc < 0 ? 0 : (qloc > 1 ? 1 : qloc);
                qloc = qloc * (1.0 - qloc);
                if (qloc < q_th) continue;
                double nix = s->aux[0][c], niy = s->aux[1][c], niz = s->aux[2][c];
                double best_r2 = 1.0e300, best_face = -1.0;
                int bi = 0, bj = 0, bk = 0, found = 0, di, dj, dk;
                for (di = -3; di <= 3; di++)
                    for (dj = -3; dj <= 3; dj++)
                        for (dk = -3; dk <= 3; dk++) {
                            if (di == 0 && dj == 0 && dk == 0) continue;
                            long nb = wrap_index(s, i + di, j + dj, k + dk);
                            int fnb = nb < 0 ? 1 : s->isf[nb];
                            if (abs(fnb) != 1) continue;
                            double r2 = (double)di * di + (double)dj * dj + (double)dk * dk;
                            if (r2 < 1.0e-12) continue;
                            double qn = nb < 0 ? 0.0 : (double)ph[nb];
                            qn = qn < 0 ? 0 : (qn > 1 ? 1 : qn);
                            qn = qn * (1.0 - qn);
                            if (qn < q_th || fabs(qn - qloc) > 0.1 * (qloc > 1.0e-12 ? qloc : 1.0e-12)) continue;
                            double dotn = nb < 0 ? 0.0 : nix * s->aux[0][nb] + niy * s->aux[1][nb] + niz * s->aux[2][nb];
                            if (dotn > s->p.cos_opp_t) continue;
                            double face = 0.5 * (1.0 - dotn);
                            if (r2 < best_r2 - 1.0e-14) {
                                best_r2 = r2; best_face = face; bi = di; bj = dj; bk = dk; found = 1;
                            } else if (fabs(r2 - best_r2) <= 1.0e-14 && face > best_face) {
                                best_face = face; bi = di; bj = dj; bk = dk; found = 1;
                            }
                        }
                if (!found) continue;
                /* normal repulsive flux (lb_cuda_repulsive_module.f90:194-289) */
                double loc_phi = (double)ph[c];
                double q1 = loc_phi * (1.0 - loc_phi);
                if (q1 <= eps) continue;
                double dx = bi, dy = bj, dz = bk, r = sqrt(dx * dx + dy * dy + dz * dz);
                if (r <= eps) continue;
                dx /= r; dy /= r; dz /= r;
                long nb = wrap_index(s, i + bi, j + bj, k + bk);
                double n2x = nb < 0 ? 0 : s->aux[0][nb], n2y = nb < 0 ? 0 : s->aux[1][nb], n2z = nb < 0 ? 0 : s->aux[2][nb];
                double face = -(nix * n2x + niy * n2y + niz * n2z);
                if (face < 0) face = 0;
                if (face <= eps) continue;
                double nsx = nix - n2x, nsy = niy - n2y, nsz = niz - n2z;
                double nsm = sqrt(nsx * nsx + nsy * nsy + nsz * nsz);
                if (nsm <= eps) {
                    nsx = dx; nsy = dy; nsz = dz;
                } else {
                    nsx /= nsm; nsy /= nsm; nsz /= nsm;
                }
                if (dx * nsx + dy * nsy + dz * nsz < 0) { nsx = -nsx; nsy = -nsy; nsz = -nsz; }
                double phi2 = nb < 0 ? 0.0 : (double)ph[nb];
                double q2 = phi2 * (1.0 - phi2), qpair = 0.5 * (q1 + q2);
                double qcl = qpair > eps ? qpair : eps;
                if (qcl > 0.25 - eps) qcl = 0.25 - eps;
                double arg = 1.0 / (2.0 * sqrt(qcl));
                if (arg <= 1.0) continue;
                double wfilm = s->p.width * log(arg + sqrt(arg * arg - 1.0));
                if (wfilm <= 0) continue;
                double wd = 1.0 / (1.0 + pow(wfilm, 4.0));
                double fx = s->p.a_rep * wd * qcl * face * nsx;
                double fy = s->p.a_rep * wd * qcl * face * nsy;
                double fz = s->p.a_rep * wd * qcl * face * nsz;
                double cap = 1.5 * (fabs(fx) + fabs(fy) + fabs(fz));
                double sc = loc_phi / (cap > 1.0e-9 ? cap : 1.0e-9);
                if (sc > 1.0) sc = 1.0;
                s->rep[0][c] = (real)(fx * sc);
                s->rep[1][c] = (real)(fy * sc);
                s->rep[2][c] = (real)(fz * sc);
            }
    }
}

/* moments_LB_kernel: lb_cuda_moments_module.f90:19-341.  s_ = input buffer
 * (updated in place), o_ = other buffer (velocity u_old). */
static void moments(orc_state *s, real **hs, real **ho, const real *ph)
{
    const int tc = s->p.twocomp, dr = s->p.densratio;
    const real cssq = (real)(1.0 / 3.0);
    int k;
#pragma omp parallel for schedule(static)
    for (k = 0; k < s->nz; k++) {
        int i, j;
        for (j = 0; j < s->ny; j++)
            for (i = 0; i < s->nx; i++) {
                long c = IDX(s, i, j, k);
                if (abs(s->isf[c]) != 1) continue;
                real press = hs[0][c];
                real phi = 0, lap = 0, mask = 0, rhophi, fxv, fyv, fzv;
                real gfx = 0, gfy = 0, gfz = 0, grx = 0, gry = 0, grz = 0;
                real visc = 0, tau = 0;
                if (tc) {
                    phi = ph[c];
                    lap = s->loc[0][c];
                    mask = (real)4.0 * phi * ((real)1.0 - phi);
                }
                if (dr) {
                    rhophi = s->rho_r * phi + ((real)1.0 - phi) * s->rho_b;
                    fxv = rhophi * s->fx; fyv = rhophi * s->fy; fzv = rhophi * s->fz;
                } else {
                    rhophi = (real)1.0;
                    fxv = s->fx; fyv = s->fy; fzv = s->fz;
                }
                if (tc) {
                    real mg = s->aux[3][c];
                    gfx = s->aux[0][c] * mg; gfy = s->aux[1][c] * mg; gfz = s->aux[2][c] * mg;
                    real chem = (real)4.0 * s->beta * phi * (phi - (real)1.0) * (phi - (real)0.5) - s->kapp * lap;
                    fxv = fxv + chem * gfx;
                    fyv = fyv + chem * gfy;
                    fzv = fzv + chem * gfz;
                    if (s->p.repulsive) {
                        /* lb_cuda_moments_module.f90:148-160: rho_phi F_rep, capped at 1e-3 */
                        real t[3];
                        for (int d = 0; d < 3; d++) {
                            t[d] = s->rep[d][c] * rhophi;
                            if (fabs((double)t[d]) > 1.0e-3) t[d] = (real)(t[d] > 0 ? 1.0e-3 : -1.0e-3);
                        }
                        fxv = fxv + t[0] * rhophi;
                        fyv = fyv + t[1] * rhophi;
                        fzv = fzv + t[2] * rhophi;
                    }
                }
                if (dr) {
                    grx = (s->rho_r - s->rho_b) * gfx;
                    gry = (s->rho_r - s->rho_b) * gfy;
                    grz = (s->rho_r - s->rho_b) * gfz;
                    fxv = fxv - mask * press * cssq * grx;
                    fyv = fyv - mask * press * cssq * gry;
                    fzv = fzv - mask * press * cssq * grz;
                }
                real tfx = fxv, tfy = fyv, tfz = fzv;
                real uo = ho[1][c], vo = ho[2][c], wo = ho[3][c];
                if (dr) {
                    real pxx = hs[4][c] - uo * uo, pyy = hs[5][c] - vo * vo, pzz = hs[6][c] - wo * wo;
                    real pxy = hs[7][c] - uo * vo, pxz = hs[8][c] - uo * wo, pyz = hs[9][c] - vo * wo;
                    visc = (s->rho_r * s->visc1 * phi + ((real)1.0 - phi) * s->visc2 * s->rho_b) / rhophi;
                    tau = visc * (real)3.0 + (real)0.5;
                    real cv = visc / (tau * cssq);
                    fxv = fxv - mask * cv * (pxx * grx + pxy * gry + pxz * grz);
                    fyv = fyv - mask * cv * (pyy * gry + pxy * grx + pyz * grz);
                    fzv = fzv - mask * cv * (pzz * grz + pxz * grx + pyz * gry);
                }
                real u = hs[1][c], v = hs[2][c], w = hs[3][c];
                if (dr) {
                    real tmp = -s->sharp_c * s->loc[1][c];
                    u = u + (real)0.5 * fxv / rhophi;
                    v = v + (real)0.5 * fyv / rhophi;
                    w = w + (real)0.5 * fzv / rhophi;
                    real dd = (s->rho_r - s->rho_b) * (s->tau_diff * lap + tmp);
                    real den = (real)1.0 - (real)0.5 * dd / rhophi;
                    u = u / den; v = v / den; w = w / den;
                    tfx = tfx - dd * u; tfy = tfy - dd * v; tfz = tfz - dd * w;
                    fxv = fxv - dd * u; fyv = fyv - dd * v; fzv = fzv - dd * w;
                } else {
                    u = u + (real)0.5 * fxv / rhophi;
                    v = v + (real)0.5 * fyv / rhophi;
                    w = w + (real)0.5 * fzv / rhophi;
                }
                hs[1][c] = u; hs[2][c] = v; hs[3][c] = w;
                real pxx = hs[4][c] + fxv * u / rhophi;
                real pyy = hs[5][c] + fyv * v / rhophi;
                real pzz = hs[6][c] + fzv * w / rhophi;
                real pxy = hs[7][c] + (real)0.5 * (fyv * u + fxv * v) / rhophi;
                real pxz = hs[8][c] + (real)0.5 * (fzv * u + fxv * w) / rhophi;
                real pyz = hs[9][c] + (real)0.5 * (fzv * v + fyv * w) / rhophi;
                hs[4][c] = pxx; hs[5][c] = pyy; hs[6][c] = pzz;
                hs[7][c] = pxy; hs[8][c] = pxz; hs[9][c] = pyz;
                if (dr) {
                    pxx = pxx - u * u; pyy = pyy - v * v; pzz = pzz - w * w;
                    pxy = pxy - u * v; pxz = pxz - u * w; pyz = pyz - v * w;
                    real cv = visc / (tau * cssq);
                    tfx = tfx - mask * cv * (pxx * grx + pxy * gry + pxz * grz);
                    tfy = tfy - mask * cv * (pyy * gry + pxy * grx + pyz * grz);
                    tfz = tfz - mask * cv * (pzz * grz + pxz * grx + pyz * gry);
                }
                s->frc[0][c] = tfx; s->frc[1][c] = tfy; s->frc[2][c] = tfz;
            }
    }
}

/* Post-collision population f*_l at node c: lb_cuda_fused_module.f90:531-713 */
/* SMAGORINSKI (lb_cuda_fused_module.f90:609-616, lb_cuda_boundary_module.f90:150-160):
 * tau = 1/2 + (3 nu + sqrt((3 nu)^2 + 0.053*18 sqrt(2 Q) / rho_phi)) / 6 with Q the
 * squared Frobenius norm of the non-equilibrium stress; 0.053*18 is a
 * single-precision product in the reference. */
static real smag_omega(real visc, real pxx, real pyy, real pzz, real pxy, real pxz, real pyz, real invrho)
{
    const real QQ = pxx * pxx + pyy * pyy + pzz * pzz + (real)2.0 * (pxy * pxy + pxz * pxz + pyz * pyz);
    const real c = (real)(double)(0.053f * 18.0f);
    real tau = (real)0.5 + ((real)1.0 / (real)6.0) *
                               ((real)3.0 * visc + (real)sqrt(((real)3.0 * visc) * ((real)3.0 * visc) +
                                                              c * (real)sqrt((real)2.0 * QQ) * invrho));
    return (real)1.0 / tau;
}

static void collide_node(const orc_state *s, real **hin, const real *ph, long c, real *fout)
{
    const int tc = s->p.twocomp, dr = s->p.densratio;
    const int ho = s->p.highorder && s->p.lattice == 27;
    const real cssq = (real)(1.0 / 3.0), invcssq = (real)3.0, HALF = (real)0.5, ONE = (real)1.0;
    real phi = 0, inv = ONE;
    int l;
    if (tc) phi = ph[c];
    if (dr) inv = (real)1.0 / (s->rho_r * phi + (ONE - phi) * s->rho_b);
    real fx = s->frc[0][c] * inv, fy = s->frc[1][c] * inv, fz = s->frc[2][c] * inv;
    real press = hin[0][c], u = hin[1][c], v = hin[2][c], w = hin[3][c];
    real pxx = hin[4][c], pyy = hin[5][c], pzz = hin[6][c], pxy = hin[7][c], pxz = hin[8][c], pyz = hin[9][c];
    if (s->p.obstacles && s->isf[c] == 0) {
        fx = fy = fz = 0; press = u = v = w = 0; pxx = pyy = pzz = pxy = pxz = pyz = 0;
    }
    pxx = pxx - u * u; pyy = pyy - v * v; pzz = pzz - w * w;
    pxy = pxy - u * v; pxz = pxz - u * w; pyz = pyz - v * w;
    real om, visc = s->visc1;
    if (tc) {
        visc = (s->rho_r * s->visc1 * phi + (ONE - phi) * s->visc2 * s->rho_b) * inv;
        om = visc * invcssq + (real)0.5;
        om = (real)1.0 / om;
    } else {
        om = s->omega;
    }
    if (s->p.smagorinsky) om = smag_omega(visc, pxx, pyy, pzz, pxy, pxz, pyz, inv);
    const real (*Mi)[27] = s->minv;
    real uu = HALF * (u * u + v * v + w * w) * invcssq;
    real feq = s->w[0] * (press - uu);
    real fneq = s->w[0] * (HALF * invcssq) * (-pxx - pyy - pzz);
    if (ho) {
        feq = feq + Mi[17][0] * u * u * v * v + Mi[18][0] * u * u * w * w + Mi[19][0] * v * v * w * w +
              Mi[26][0] * u * u * v * v * w * w;
        fneq = fneq + Mi[17][0] * (pyy * u * u + (real)2.0 * v * ((real)3.0 * pxy * u + pxx * v)) +
               Mi[18][0] * (pzz * u * u + (real)2.0 * w * ((real)3.0 * pxz * u + pxx * w)) +
               Mi[19][0] * (pzz * v * v + (real)2.0 * w * ((real)3.0 * pyz * v + pyy * w)) +
               Mi[26][0] * (pzz * u * u * v * v +
                            w * ((real)6.0 * u * v * (pyz * u + pxz * v) + (real)3.0 * pyy * u * u * w +
                                 (real)2.0 * v * ((real)7.0 * pxy * u + (real)2.0 * pxx * v) * w));
    }
    real fd = s->w[0] * (-u * fx - v * fy - w * fz) * invcssq;
    fout[0] = feq + (ONE - om) * fneq + HALF * fd;
    for (l = 1; l < s->nl; l++) {
        real dex = (real)s->ex[l], dey = (real)s->ey[l], dez = (real)s->ez[l];
        real ud = (u * dex + v * dey + w * dez) * invcssq;
        feq = s->w[l] * (press + (ud + (real)0.5 * ud * ud - uu));
        fneq = s->w[l] * (HALF / (cssq * cssq)) *
               ((dex * dex - cssq) * pxx + (dey * dey - cssq) * pyy + (dez * dez - cssq) * pzz +
                (real)2.0 * (dex * dey) * pxy + (real)2.0 * (dex * dez) * pxz + (real)2.0 * (dey * dez) * pyz);
        if (ho) {
            feq = feq + Mi[10][l] * u * u * v + Mi[11][l] * u * u * w + Mi[12][l] * u * v * v +
                  Mi[13][l] * u * w * w + Mi[14][l] * v * w * w + Mi[15][l] * v * v * w + Mi[16][l] * u * v * w +
                  Mi[17][l] * u * u * v * v + Mi[18][l] * u * u * w * w + Mi[19][l] * v * v * w * w +
                  Mi[20][l] * u * v * w * w + Mi[21][l] * u * v * v * w + Mi[22][l] * u * u * v * w +
                  Mi[23][l] * u * u * v * w * w + Mi[24][l] * u * u * v * v * w + Mi[25][l] * u * v * v * w * w +
                  Mi[26][l] * u * u * v * v * w * w;
            fneq = fneq + Mi[10][l] * ((real)2.0 * pxy * u + pxx * v) + Mi[11][l] * ((real)2.0 * pxz * u + pxx * w) +
                   Mi[12][l] * (pyy * u + (real)2.0 * pxy * v) + Mi[13][l] * (pzz * u + (real)2.0 * pxz * w) +
                   Mi[14][l] * (pzz * v + (real)2.0 * pyz * w) + Mi[15][l] * ((real)2.0 * pyz * v + pyy * w) +
                   Mi[16][l] * (pyz * u + pxz * v + pxy * w) +
                   Mi[17][l] * (pyy * u * u + (real)2.0 * v * ((real)3.0 * pxy * u + pxx * v)) +
                   Mi[18][l] * (pzz * u * u + (real)2.0 * w * ((real)3.0 * pxz * u + pxx * w)) +
                   Mi[19][l] * (pzz * v * v + (real)2.0 * w * ((real)3.0 * pyz * v + pyy * w)) +
                   Mi[20][l] * (pzz * u * v + w * ((real)3.0 * pyz * u + (real)3.0 * pxz * v + (real)2.0 * pxy * w)) +
                   Mi[21][l] * ((real)2.0 * pyz * u * v + pxz * v * v + (real)2.0 * pyy * u * w + (real)4.0 * pxy * v * w) +
                   Mi[22][l] * (pyz * u * u + (real)2.0 * pxz * u * v + (real)4.0 * pxy * u * w + (real)2.0 * pxx * v * w) +
                   Mi[23][l] * (pzz * u * u * v +
                                (real)3.0 * w * (pyz * u * u + (real)2.0 * pxz * u * v + (real)2.0 * pxy * u * w + pxx * v * w)) +
                   Mi[24][l] * ((real)2.0 * u * v * (pyz * u + pxz * v) + (real)2.0 * pyy * u * u * w +
                                v * ((real)10.0 * pxy * u + (real)3.0 * pxx * v) * w) +
                   Mi[25][l] * (pzz * u * v * v +
                                (real)3.0 * w * ((real)2.0 * pyz * u * v + pxz * v * v + pyy * u * w + (real)2.0 * pxy * v * w)) +
                   Mi[26][l] * (pzz * u * u * v * v +
                                w * ((real)6.0 * u * v * (pyz * u + pxz * v) + (real)3.0 * pyy * u * u * w +
                                     (real)2.0 * v * ((real)7.0 * pxy * u + (real)2.0 * pxx * v) * w));
        }
        fd = s->w[l] * (((dex - u) + ud * dex) * fx + ((dey - v) + ud * dey) * fy + ((dez - w) + ud * dez) * fz) * invcssq;
        fout[l] = feq + (ONE - om) * fneq + HALF * fd;
    }
}

/* fused_LB_kernel: every interior node x receives f*_l(x - c_l), summed in
 * link order into the ten output moments (lb_cuda_fused_module.f90:637-748).
 * BOUNCE_BACK (fused_LB_kernel_bb, lb_cuda_fused_module.f90:364-380): a link
 * whose upstream node x - c_l is solid (isfluid = 0) brings instead the
 * node's own post-collision population of the opposite link -- the solid
 * node sends back what it received from x, in the same step (half-way
 * bounce-back); solid nodes push nothing (zeroed moments). */
static void fused(orc_state *s, real **hin, real **hout, const real *ph)
{
    const real cssq = (real)(1.0 / 3.0);
    const int NXY = s->NX * s->NY;
    const int nl = s->nl;
    const int bb = s->p.obstacles && s->p.bounce_back;
    real *fst = (real *)malloc(sizeof(real) * (size_t)s->npad * (size_t)nl);
    int k;
    /* post-collision populations on the interior and its halo ring */
#pragma omp parallel for schedule(static)
    for (k = -1; k <= s->nz; k++) {
        int i, j;
        real fo[27];
        for (j = -1; j <= s->ny; j++)
            for (i = -1; i <= s->nx; i++) {
                long c = IDX(s, i, j, k);
                int l;
                collide_node(s, hin, ph, c, fo);
                for (l = 0; l < nl; l++) fst[(size_t)c * nl + l] = fo[l];
            }
    }
#pragma omp parallel for schedule(static)
    for (k = 0; k < s->nz; k++) {
        int i, j, l;
        for (j = 0; j < s->ny; j++)
            for (i = 0; i < s->nx; i++) {
                long c = IDX(s, i, j, k);
                real f0 = fst[(size_t)c * nl + 0];
                real op = f0, ou = 0, ov = 0, ow = 0;
                real oxx = f0 * (-cssq), oyy = f0 * (-cssq), ozz = f0 * (-cssq), oxy = 0, oxz = 0, oyz = 0;
                for (l = 1; l < nl; l++) {
                    long src = c - s->ex[l] - (long)s->ey[l] * s->NX - (long)s->ez[l] * NXY;
                    real f = fst[(size_t)src * nl + l];
                    if (bb && s->isf[src] == 0) f = fst[(size_t)c * nl + s->opp[l]];
                    real dex = (real)s->ex[l], dey = (real)s->ey[l], dez = (real)s->ez[l];
                    op = op + f;
                    ou = ou + f * dex; ov = ov + f * dey; ow = ow + f * dez;
                    oxx = oxx + f * (dex * dex - cssq);
                    oyy = oyy + f * (dey * dey - cssq);
                    ozz = ozz + f * (dez * dez - cssq);
                    oxy = oxy + f * dex * dey;
                    oxz = oxz + f * dex * dez;
                    oyz = oyz + f * dey * dez;
                }
                hout[0][c] = op; hout[1][c] = ou; hout[2][c] = ov; hout[3][c] = ow;
                hout[4][c] = oxx; hout[5][c] = oyy; hout[6][c] = ozz;
                hout[7][c] = oxy; hout[8][c] = oxz; hout[9][c] = oyz;
            }
    }
    free(fst);
}

/* update_phifields_kernel: lb_cuda_update_phi_module.f90:19-104 */
static void update_phi(orc_state *s, real **hs, const real *pin, real *pout)
{
    int k;
#pragma omp parallel for schedule(static)
    for (k = 0; k < s->nz; k++) {
        int i, j;
        for (j = 0; j < s->ny; j++)
            for (i = 0; i < s->nx; i++) {
                long c = IDX(s, i, j, k);
                if (abs(s->isf[c]) != 1) continue;
                real tmp = -s->sharp_c * s->loc[1][c];
                real mg = s->aux[3][c];
                real gx = s->aux[0][c] * mg, gy = s->aux[1][c] * mg, gz = s->aux[2][c] * mg;
                real phi = pin[c], lap = s->loc[0][c];
                real u = hs[1][c], v = hs[2][c], w = hs[3][c];
                pout[c] = phi - u * (real)0.5 * gx - v * (real)0.5 * gy - w * (real)0.5 * gz + s->tau_diff * lap + tmp;
            }
    }
}

/* LB_int_boundary_kernel: lb_cuda_boundary_module.f90:19-216 */
static void obstacle_bb(orc_state *s, real **hin, real **hout, const real *ph)
{
    const int tc = s->p.twocomp, dr = s->p.densratio;
    const real cssq = (real)(1.0 / 3.0), ONE = (real)1.0, HALF = (real)0.5;
    int k;
#pragma omp parallel for schedule(static)
    for (k = 0; k < s->nz; k++) {
        int i, j, l;
        for (j = 0; j < s->ny; j++)
            for (i = 0; i < s->nx; i++) {
                long c = IDX(s, i, j, k);
                if (s->isf[c] != -1) continue;
                real phi = 0, rhophi = ONE;
                if (tc) phi = ph[c];
                if (dr) rhophi = s->rho_r * phi + (ONE - phi) * s->rho_b;
                real press = hin[0][c], u = hin[1][c], v = hin[2][c], w = hin[3][c];
                real pxx = hin[4][c] - u * u, pyy = hin[5][c] - v * v, pzz = hin[6][c] - w * w;
                real pxy = hin[7][c] - u * v, pxz = hin[8][c] - u * w, pyz = hin[9][c] - v * w;
                real o[10];
                for (l = 0; l < 10; l++) o[l] = hout[l][c];
                real om, visc = s->visc1;
                if (tc) {
                    visc = (s->rho_r * s->visc1 * phi + (ONE - phi) * s->visc2 * s->rho_b) / rhophi;
                    om = visc * (real)3.0 + (real)0.5;
                    om = (real)1.0 / om;
                } else {
                    om = s->omega;
                }
                if (s->p.smagorinsky) om = smag_omega(visc, pxx, pyy, pzz, pxy, pxz, pyz, (real)1.0 / rhophi);
                for (l = 1; l < s->nl; l++) {
                    int lo = s->opp[l];
                    if (s->isf[IDX(s, i + s->ex[lo], j + s->ey[lo], k + s->ez[lo])] != 0) continue;
                    real dex = (real)s->ex[l], dey = (real)s->ey[l], dez = (real)s->ez[l];
                    real feq = s->w[l] * press;
                    real fneq = s->w[l] * (HALF / (cssq * cssq)) *
                                ((dex * dex - cssq) * pxx + (dey * dey - cssq) * pyy + (dez * dez - cssq) * pzz +
                                 (real)2.0 * (dex * dey) * pxy + (real)2.0 * (dex * dez) * pxz + (real)2.0 * (dey * dez) * pyz);
                    real fp = feq + (ONE - om) * fneq;
                    o[0] = o[0] + fp;
                    o[1] = o[1] + fp * dex; o[2] = o[2] + fp * dey; o[3] = o[3] + fp * dez;
                    o[4] = o[4] + fp * (dex * dex - cssq);
                    o[5] = o[5] + fp * (dey * dey - cssq);
                    o[6] = o[6] + fp * (dez * dez - cssq);
                    o[7] = o[7] + fp * dex * dey;
                    o[8] = o[8] + fp * dex * dez;
                    o[9] = o[9] + fp * dey * dez;
                }
                for (l = 0; l < 10; l++) hout[l][c] = o[l];
            }
    }
}

/* Open face (axis 0/1/2 = x/y/z, side 0 = low, 1 = high) of
 * bcs_mesoscopic_hfields, boundary_cds_module.f90:57-1311, run after
 * LB_int_boundary on the moments B of the step.  Nodes: isfluid = -1 on the
 * plane next to the wall (reference gi = 2 or lx-1), the two tangential
 * indices strictly inside (1, l) of the reference's 1-based range.  For every
 * link l whose upstream node x - c_l is a wall (isfluid = 0) the population
 * w_l P + (1 - omega) fneq(Pi') is taken out of B with the weights c_a c_b,
 * and the population of the face's state is added with c_a c_b - cs^2 delta
 * (HIGHORDER: with the Minv_mrt rows 10-26 of the face velocity), where
 * Pi' = Pi - cs^2 P - u u from the node's moments after the force half-step
 * (A), and omega is the molecular relaxation rate of the node's phi.  Face
 * types (openbc_type): 2 zero gradient (the node's P and u), 1 pressure
 * (openbc_press, the node's u), other velocity (the node's P, openbc_u/v/w).
 * The removal does not invert the bounce-back (other Pi, other weights):
 * both are kept as the reference writes them. */
static void open_face(orc_state *s, real **hin, real **hout, const real *ph, int axis, int side)
{
    const int tc = s->p.twocomp, dr = s->p.densratio, ho = s->p.highorder && s->p.lattice == 27;
    const real cssq = (real)(1.0 / 3.0), invcssq = (real)3.0, ONE = (real)1.0, HALF = (real)0.5, TWO = (real)2.0;
    const real THREE = (real)3.0, FOUR = (real)4.0, SIX = (real)6.0, SEVEN = (real)7.0, TEN = (real)10.0;
    const int n[3] = {s->nx, s->ny, s->nz};
    const int a1 = axis == 0 ? 1 : 0, a2 = axis == 2 ? 1 : 2;  /* tangential axes */
    const int plane = side ? n[axis] - 2 : 1;
    const int type = s->p.obc_type[axis][side];
    int t2;
#pragma omp parallel for schedule(static)
    for (t2 = 1; t2 <= n[a2] - 2; t2++) {
        int t1, l, r;
        for (t1 = 1; t1 <= n[a1] - 2; t1++) {
            int x[3];
            x[axis] = plane; x[a1] = t1; x[a2] = t2;
            const int i = x[0], j = x[1], k = x[2];
            long c = IDX(s, i, j, k);
            if (s->isf[c] != -1) continue;
            real press = hin[0][c], u = hin[1][c], v = hin[2][c], w = hin[3][c];
            real pxx = hin[4][c], pyy = hin[5][c], pzz = hin[6][c];
            real pxy = hin[7][c], pxz = hin[8][c], pyz = hin[9][c];
            real o[10];
            for (l = 0; l < 10; l++) o[l] = hout[l][c];
            real presstmp = press, utmp = u, vtmp = v, wtmp = w;
            if (type == 1) {
                presstmp = (real)s->p.obc_press[axis][side];
            } else if (type != 2) {
                utmp = (real)s->p.obc_vel[axis][side][0];
                vtmp = (real)s->p.obc_vel[axis][side][1];
                wtmp = (real)s->p.obc_vel[axis][side][2];
            }
            pxx = pxx - cssq * press - u * u;
            pyy = pyy - cssq * press - v * v;
            pzz = pzz - cssq * press - w * w;
            pxy = pxy - u * v;
            pxz = pxz - u * w;
            pyz = pyz - v * w;
            real om = s->omega;
            if (tc) {
                real phi = ph[c], rhophi = ONE;
                if (dr) rhophi = s->rho_r * phi + (ONE - phi) * s->rho_b;
                real visc = (s->rho_r * s->visc1 * phi + (ONE - phi) * s->visc2 * s->rho_b) / rhophi;
                om = ONE / (visc * invcssq + HALF);
            }
            real uu = HALF * (utmp * utmp + vtmp * vtmp + wtmp * wtmp) * invcssq;
            /* HIGHORDER terms of the face population (rows 10..26): equilibrium
             * monomials and non-equilibrium projections */
            real meq[27], mneq[27];
            if (ho) {
                const real U = utmp, V = vtmp, W = wtmp;
                meq[10] = U * U * V; meq[11] = U * U * W; meq[12] = U * V * V; meq[13] = U * W * W;
                meq[14] = V * W * W; meq[15] = V * V * W; meq[16] = U * V * W;
                meq[17] = U * U * V * V; meq[18] = U * U * W * W; meq[19] = V * V * W * W;
                meq[20] = U * V * W * W; meq[21] = U * V * V * W; meq[22] = U * U * V * W;
                meq[23] = U * U * V * W * W; meq[24] = U * U * V * V * W; meq[25] = U * V * V * W * W;
                meq[26] = U * U * V * V * W * W;
                mneq[10] = TWO * pxy * U + pxx * V;
                mneq[11] = TWO * pxz * U + pxx * W;
                mneq[12] = pyy * U + TWO * pxy * V;
                mneq[13] = pzz * U + TWO * pxz * W;
                mneq[14] = pzz * V + TWO * pyz * W;
                mneq[15] = TWO * pyz * V + pyy * W;
                mneq[16] = pyz * U + pxz * V + pxy * W;
                mneq[17] = pyy * U * U + TWO * V * (THREE * pxy * U + pxx * V);
                mneq[18] = pzz * U * U + TWO * W * (THREE * pxz * U + pxx * W);
                mneq[19] = pzz * V * V + TWO * W * (THREE * pyz * V + pyy * W);
                mneq[20] = pzz * U * V + W * (THREE * pyz * U + THREE * pxz * V + TWO * pxy * W);
                mneq[21] = TWO * pyz * U * V + pxz * V * V + TWO * pyy * U * W + FOUR * pxy * V * W;
                mneq[22] = pyz * U * U + TWO * pxz * U * V + FOUR * pxy * U * W + TWO * pxx * V * W;
                mneq[23] = pzz * U * U * V + THREE * W * (pyz * U * U + TWO * pxz * U * V + TWO * pxy * U * W + pxx * V * W);
                mneq[24] = TWO * U * V * (pyz * U + pxz * V) + TWO * pyy * U * U * W + V * (TEN * pxy * U + THREE * pxx * V) * W;
                mneq[25] = pzz * U * V * V + THREE * W * (TWO * pyz * U * V + pxz * V * V + pyy * U * W + TWO * pxy * V * W);
                mneq[26] = pzz * U * U * V * V +
                           W * (SIX * U * V * (pyz * U + pxz * V) + THREE * pyy * U * U * W + TWO * V * (SEVEN * pxy * U + TWO * pxx * V) * W);
            }
            for (l = 1; l < s->nl; l++) {
                int lo = s->opp[l];
                if (s->isf[IDX(s, i + s->ex[lo], j + s->ey[lo], k + s->ez[lo])] != 0) continue;
                real dex = (real)s->ex[l], dey = (real)s->ey[l], dez = (real)s->ez[l];
                real feq = s->w[l] * press;
                real fneq = s->w[l] * (HALF / (cssq * cssq)) *
                            ((dex * dex - cssq) * pxx + (dey * dey - cssq) * pyy + (dez * dez - cssq) * pzz +
                             TWO * (dex * dey) * pxy + TWO * (dex * dez) * pxz + TWO * (dey * dez) * pyz);
                real fp = feq + (ONE - om) * fneq;
                o[0] = o[0] - fp;
                o[1] = o[1] - fp * dex; o[2] = o[2] - fp * dey; o[3] = o[3] - fp * dez;
                o[4] = o[4] - fp * dex * dex; o[5] = o[5] - fp * dey * dey; o[6] = o[6] - fp * dez * dez;
                o[7] = o[7] - fp * dex * dey; o[8] = o[8] - fp * dex * dez; o[9] = o[9] - fp * dey * dez;
                real udotc = (utmp * dex + vtmp * dey + wtmp * dez) * invcssq;
                feq = s->w[l] * (presstmp + udotc + HALF * udotc * udotc - uu);
                if (ho)
                    for (r = 10; r < 27; r++) {
                        feq = feq + s->minv[r][l] * meq[r];
                        fneq = fneq + s->minv[r][l] * mneq[r];
                    }
                fp = feq + (ONE - om) * fneq;
                o[0] = o[0] + fp;
                o[1] = o[1] + fp * dex; o[2] = o[2] + fp * dey; o[3] = o[3] + fp * dez;
                o[4] = o[4] + fp * (dex * dex - cssq);
                o[5] = o[5] + fp * (dey * dey - cssq);
                o[6] = o[6] + fp * (dez * dez - cssq);
                o[7] = o[7] + fp * dex * dey; o[8] = o[8] + fp * dex * dez; o[9] = o[9] + fp * dey * dez;
            }
            for (l = 0; l < 10; l++) hout[l][c] = o[l];
        }
    }
}

/* the open faces in the reference's order: x low, x high, y low, ..., on
 * the non-periodic axes */
static void open_bc(orc_state *s, real **hin, real **hout, const real *ph)
{
    const int pbc[3] = {s->p.pbc_x, s->p.pbc_y, s->p.pbc_z};
    int axis, side;
    for (axis = 0; axis < 3; axis++)
        if (!pbc[axis])
            for (side = 0; side < 2; side++) open_face(s, hin, hout, ph, axis, side);
}

/* Open boundaries, phase field (bcs_mesoscopic_phifields after
 * PHI_int_boundary, boundary_cds_module.f90:1351-1663): on each open face the
 * wall nodes (reference gi = 1 or lx), tangential indices strictly inside
 * (1, l), take the phi of their neighbour on the plane next to them. */
static void open_phi_copy(orc_state *s, real *ph)
{
    const int pbc[3] = {s->p.pbc_x, s->p.pbc_y, s->p.pbc_z};
    const int n[3] = {s->nx, s->ny, s->nz};
    int axis, side, t1, t2;
    for (axis = 0; axis < 3; axis++) {
        if (pbc[axis]) continue;
        const int a1 = axis == 0 ? 1 : 0, a2 = axis == 2 ? 1 : 2;
        for (side = 0; side < 2; side++)
            for (t2 = 1; t2 <= n[a2] - 2; t2++)
                for (t1 = 1; t1 <= n[a1] - 2; t1++) {
                    int x[3], y[3];
                    x[axis] = side ? n[axis] - 1 : 0; x[a1] = t1; x[a2] = t2;
                    y[axis] = side ? n[axis] - 2 : 1; y[a1] = t1; y[a2] = t2;
                    ph[IDX(s, x[0], x[1], x[2])] = ph[IDX(s, y[0], y[1], y[2])];
                }
    }
}

/* Phi carried through the open faces in one step (BCPHIFLUX,
 * boundary_cds_module.f90:1667-1861): over the isfluid = -1 nodes of the
 * planes next to the walls (no tangential limits), + u_n phi on low faces and
 * - u_n phi on high faces, u_n the moment velocity normal to the face, in
 * FP64. */
static double phi_flux(const orc_state *s, real **h, const real *ph)
{
    const int pbc[3] = {s->p.pbc_x, s->p.pbc_y, s->p.pbc_z};
    const int n[3] = {s->nx, s->ny, s->nz};
    double flux = 0.0;
    int axis, side, t1, t2;
    for (axis = 0; axis < 3; axis++) {
        if (pbc[axis]) continue;
        const int a1 = axis == 0 ? 1 : 0, a2 = axis == 2 ? 1 : 2;
        for (side = 0; side < 2; side++)
            for (t2 = 0; t2 < n[a2]; t2++)
                for (t1 = 0; t1 < n[a1]; t1++) {
                    int x[3];
                    x[axis] = side ? n[axis] - 2 : 1; x[a1] = t1; x[a2] = t2;
                    long c = IDX(s, x[0], x[1], x[2]);
                    if (s->isf[c] != -1) continue;
                    double q = (double)h[1 + axis][c] * (double)ph[c];
                    flux += side ? -q : q;
                }
    }
    return flux;
}

/* copy_print: print_module.f90:638-776 (stepskip = 1) */
static void copy_print(orc_state *s, real **hs, const real *ph)
{
    long c;
    for (c = 0; c < s->npad; c++) {
        if (s->p.twocomp) {
            if (s->p.densratio)
                s->prt_rho[c] = s->rho_r * ph[c] + ((real)1.0 - ph[c]) * s->rho_b;
            else
                s->prt_rho[c] = ph[c];
        } else {
            s->prt_rho[c] = hs[0][c];
        }
        s->prt_press[c] = hs[0][c];
        s->prt_vel[0][c] = hs[1][c];
        s->prt_vel[1][c] = hs[2][c];
        s->prt_vel[2][c] = hs[3][c];
    }
}

static void exchange_h(orc_state *s, real **h)
{
    int f;
    for (f = 0; f < 10; f++) halo_real(s, h[f]);
}

/* Integrator preamble: integrator_module.f90:186-248 */
/* Sum of phi over fluid nodes (|isfluid| = 1) in FP64 and the number of
 * interface nodes 0.5 < phi < 0.9: phi_sum_count_kernel,
 * lb_cuda_boundary_module.f90:459-506 (the initial sum as
 * init_conditions_module.f90:468-490). */
static double phi_sum_count(const orc_state *s, const real *ph, long *cnt)
{
    double sum = 0.0;
    long c = 0;
    int i, j, k;
    for (k = 0; k < s->nz; k++)
        for (j = 0; j < s->ny; j++)
            for (i = 0; i < s->nx; i++) {
                long n = IDX(s, i, j, k);
                int f = s->isf[n];
                double v;
                if (f != 1 && f != -1) continue;
                v = (double)ph[n];
                sum += v;
                if (v > 0.5 && v < 0.9) c++;
            }
    if (cnt) *cnt = c;
    return sum;
}

/* phi mass correction (boundary_cds_module.f90:1864-1885 with
 * apply_lagrangian_phi_kernel, lb_cuda_boundary_module.f90:509-563): the
 * lost mass dphi = sum0 - sum is spread over the interface nodes,
 * corr = dphi / count added to every fluid node with 0.5 < phi < 0.9.  The
 * reference applies it only with open boundaries, where the target is
 * sum0 + flux, flux the phi carried through the open faces (phi_flux) by the
 * step's input moments; with periodic and wall boundaries it is zero.  It
 * runs inside bcs_mesoscopic_phifields on the step's INPUT phi, after
 * compute_norm has read it and before div theta, the moments, the fused
 * kernel and update_phi (integrator_module.f90:297, 315, 371): the
 * gradient, normal and Laplacian of the step see the uncorrected phi, the
 * rest the corrected one.  Only interior nodes are written (the kernel's
 * grid covers the interior tiles), so the periodic halo copy of phi keeps
 * the uncorrected values until the next exchange -- which the fused
 * kernel's halo ring reads. */
static void mass_correction(orc_state *s, real *ph, double flux)
{
    long cnt = 0;
    double sum = phi_sum_count(s, ph, &cnt), corr;
    int i, j, k;
    if (cnt == 0) return;
    corr = (s->phi_sum0 + flux - sum) / (double)cnt;
    for (k = 0; k < s->nz; k++)
        for (j = 0; j < s->ny; j++)
            for (i = 0; i < s->nx; i++) {
                long n = IDX(s, i, j, k);
                int f = s->isf[n];
                double v;
                if (f != 1 && f != -1) continue;
                v = (double)ph[n];
                if (v > 0.5 && v < 0.9) ph[n] = (real)(v + corr);
            }
}

static void prime(orc_state *s)
{
    real **A = s->h[s->flip];
    if (s->p.twocomp) s->phi_sum0 = phi_sum_count(s, s->phi[s->flip], NULL);
    if (s->p.twocomp && s->p.obstacles) {
        wetting(s, s->phi[s->flip]);
        if (s->p.openbc) {
            open_phi_copy(s, s->phi[s->flip]);
            /* the pre-loop bcs_mesoscopic_phifields corrects once with the
             * flux of the initial state (integrator_module.f90:179-182) */
            if (s->p.phi_correction) mass_correction(s, s->phi[s->flip], phi_flux(s, A, s->phi[s->flip]));
        }
    }
    copy_print(s, A, s->phi[s->flip]);
    if (s->p.twocomp) halo_real(s, s->phi[s->flip]);
    exchange_h(s, A);
    s->primed = 1;
}

/* One time step: integrator_module.f90:270-544. */
static void one_step(orc_state *s)
{
    int in = s->flip, out = 1 - s->flip, f;
    real **A = s->h[in], **B = s->h[out];
    real *pA = s->phi[in], *pB = s->phi[out];
    if (s->p.twocomp) {
        compute_norm(s, pA);
        for (f = 0; f < 7; f++) halo_real(s, s->aux[f]);
        if (s->p.obstacles) {
            wetting(s, pA);
            if (s->p.openbc) open_phi_copy(s, pA);
        }
        /* bcs_mesoscopic_phifields: the mass correction of the input phi
         * (integrator_module.f90:297), no halo exchange after it */
        if (s->p.phi_correction)
            mass_correction(s, pA, s->p.obstacles && s->p.openbc ? phi_flux(s, A, pA) : 0.0);
        compute_div_theta(s);
        if (s->p.repulsive) repulsive(s, pA);
    }
    moments(s, A, B, pA);
    exchange_h(s, A);
    for (f = 0; f < 3; f++) halo_real(s, s->frc[f]);
    copy_print(s, A, pA);
    fused(s, A, B, pA);
    if (s->p.twocomp) update_phi(s, A, pA, pB);
    if (s->p.obstacles) {
        /* bcs_mesoscopic_hfields: LB_int_boundary only without BOUNCE_BACK
         * (boundary_cds_module.f90:50-56), then the open faces */
        if (!s->p.bounce_back) obstacle_bb(s, A, B, pA);
        if (s->p.openbc) open_bc(s, A, B, pA);
    }
    if (s->p.twocomp) halo_real(s, pB);
    s->flip = out;
    s->step++;
}

void orc_step(orc_state *s, int nsteps)
{
    int n;
    unsigned int saved = 0;
#if defined(__x86_64__) || defined(__i386__)
    saved = _mm_getcsr();
#endif
#pragma omp parallel
    FTZ_ON();
    FTZ_ON();
    if (!s->primed) prime(s);
    for (n = 0; n < nsteps; n++) one_step(s);
#if defined(__x86_64__) || defined(__i386__)
    _mm_setcsr(saved);
#pragma omp parallel
    _mm_setcsr(saved);
#else
    (void)saved;
#endif
}

void orc_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* The state a next step would start from: moments (10 x N), phi (N), and the
 * velocity u_old the next step's DENSRATIO force reads (3 x N). */
void orc_get_fields(orc_state *s, double *h10, double *phi, double *uold)
{
    long n = (long)s->nx * s->ny * s->nz;
    int i, j, k, f;
    if (!s->primed) prime(s);
    for (k = 0; k < s->nz; k++)
        for (j = 0; j < s->ny; j++)
            for (i = 0; i < s->nx; i++) {
                long dst = ((long)k * s->ny + j) * s->nx + i, src = IDX(s, i, j, k);
                if (h10)
                    for (f = 0; f < 10; f++) h10[f * n + dst] = (double)s->h[s->flip][f][src];
                if (phi) phi[dst] = (double)s->phi[s->flip][src];
                if (uold)
                    for (f = 0; f < 3; f++) uold[f * n + dst] = (double)s->h[1 - s->flip][1 + f][src];
            }
}

/* phi of both buffers (solid-node ghost values differ between them). */
void orc_get_phi_buffers(orc_state *s, double *phi_in, double *phi_other)
{
    int i, j, k;
    if (!s->primed) prime(s);
    for (k = 0; k < s->nz; k++)
        for (j = 0; j < s->ny; j++)
            for (i = 0; i < s->nx; i++) {
                long dst = ((long)k * s->ny + j) * s->nx + i, src = IDX(s, i, j, k);
                if (phi_in) phi_in[dst] = (double)s->phi[s->flip][src];
                if (phi_other) phi_other[dst] = (double)s->phi[1 - s->flip][src];
            }
}

/* copy_print output of the last step (rho, vel as 3 x N, press). */
void orc_get_print(orc_state *s, double *rho, double *vel, double *press)
{
    long n = (long)s->nx * s->ny * s->nz;
    int i, j, k;
    if (!s->primed) prime(s);
    for (k = 0; k < s->nz; k++)
        for (j = 0; j < s->ny; j++)
            for (i = 0; i < s->nx; i++) {
                long dst = ((long)k * s->ny + j) * s->nx + i, src = IDX(s, i, j, k);
                if (rho) rho[dst] = (double)s->prt_rho[src];
                if (press) press[dst] = (double)s->prt_press[src];
                if (vel) {
                    vel[dst] = (double)s->prt_vel[0][src];
                    vel[n + dst] = (double)s->prt_vel[1][src];
                    vel[2 * n + dst] = (double)s->prt_vel[2][src];
                }
            }
}

long orc_get_step(orc_state *s) { return s->step; }
int orc_real_size(void) { return (int)sizeof(real); }
