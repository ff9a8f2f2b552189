/*
 * lbfast_gpu.h -- C ABI of the B200 implementation of the LBFAST time step.
 *
 * The reference drives its GPU kernels through the Fortran module
 * lb_cuda_driver (lb_cuda_driver_module.f90), called by the integrator
 * (integrator_module.f90:39-46) on device-resident tiled arrays that the
 * Fortran side owns.  This header replaces that module with a flat C
 * interface a Fortran driver binds through iso_c_binding (bind(C)), in the
 * style of the reference's only existing C binding (nvml_wrapper.c:6-33,
 * nvml_interface_module.f90:6-20): integer status returns, value arguments
 * for scalars, plain pointers for arrays.  The library owns the device
 * fields; the caller exchanges host arrays in Fortran order (i fastest).
 *
 * Every function returns LBF_OK (0) or a negative LBF_E* code; the message
 * of the last failure on the calling thread is returned by lbf_last_error.
 * No exception crosses this boundary.
 */
#ifndef LBFAST_GPU_H
#define LBFAST_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LBF_ABI_VERSION 1

enum {
    LBF_OK = 0,
    LBF_E_ARG = -1,      /* invalid argument */
    LBF_E_CUDA = -2,     /* CUDA runtime error */
    LBF_E_NOMEM = -3,    /* device or host allocation failed */
    LBF_E_STATE = -4,    /* call out of order (e.g. step before set_fields) */
    LBF_E_UNSUPPORTED = -5,
    LBF_E_IO = -6,       /* file could not be read or written */
    LBF_E_NUMERIC = -7   /* non-finite value detected */
};

/* storage of the moment fields in HBM */
enum { LBF_STORE_F32 = 0, LBF_STORE_F16 = 1, LBF_STORE_BF16 = 2, LBF_STORE_F64 = 3 };
/* element type of host arrays */
enum { LBF_F32 = 0, LBF_F64 = 1 };

/*
 * Run parameters.  Mirrors the reference's compile-time macros (defines.h:1-74:
 * LATTICE, HIGHORDER, TWOCOMPONENT, DENSRATIO -> INTERFACE_INCOMP,
 * INTERNAL_OBSTACLES) and the `simulation` / `fluid` namelists
 * (LBFAST.f90:32-60).  Derived quantities (tau, omega, beta, kappa, sharp_c)
 * are computed inside with the formulas of LBFAST.f90:212-219.
 */
typedef struct lbf_params {
    int lx, ly, lz;          /* box (one GPU: nx = lx etc.) */
    int pbc_x, pbc_y, pbc_z; /* 1 = periodic */
    int lattice;             /* 15, 19 or 27 */
    int highorder;           /* HIGHORDER, LATTICE 27 only */
    int twocomponent;        /* TWOCOMPONENT */
    int densratio;           /* DENSRATIO (requires twocomponent) */
    int obstacles;           /* INTERNAL_OBSTACLES */
    int storage;             /* LBF_STORE_* */
    double visc1, visc2;     /* kinematic viscosities */
    double rho_r, rho_b;     /* densities of the phi=1 and phi=0 fluids */
    double sigma, width;     /* surface tension, interface width */
    double tau_diff;         /* phase-field diffusivity */
    double fx, fy, fz;       /* body force */
    double wettab_r;         /* contact angle in degrees (obstacles, two components); the reference
                                applies it only with WETTABILITY and otherwise uses 90
                                (lb_cuda_boundary_module.f90:264,275) */
    int printphi;            /* PRINTPHI: `rho` output holds phi */
    int zseg;                /* planes per z segment of the kernel (one CTA per tile and segment); < 0 =
                                split columns: per column one CTA for planes [0, -zseg) and one for the
                                rest (for boxes whose columns fill less than one wave of SMs); 0 = a
                                persistent schedule: one CTA per resident slot, each advancing an equal
                                contiguous share of the box's columns x planes */
    int tile_y;              /* rows of the kernel's 32-wide tile: 8 or 16 (FP64: 8 only).  0 = 16 rows (8 in
                                FP64) and, when zseg = 0, the schedule autotuned at the first lbf_step: each
                                candidate (persistent, z segments of several lengths, split columns) is timed on the box
                                itself, the fastest is kept and remembered for boxes of the same shape and
                                class.  The schedule does not change the results; the tile height may in
                                the last bit (separate compilations). */
    int phi_correction;      /* two components: after every step restore the FP64 sum of phi over fluid
                                nodes to its value at the first step by adding (sum0 - sum) / count to
                                the count interface nodes with 0.5 < phi < 0.9 (the reference's
                                BCPHIFLUX Lagrange correction, boundary_cds_module.f90:1864-1885, which it
                                applies with open boundaries only); 0 = off (the reference default) */
    int smagorinsky;         /* SMAGORINSKI: LES relaxation time from the non-equilibrium stress
                                (lb_cuda_fused_module.f90:609-616, lb_cuda_boundary_module.f90:150-160) */
    int openbc;              /* openbc = 1 (requires obstacles): open faces on every non-periodic axis, as
                                bcs_mesoscopic_hfields / _phifields do (boundary_cds_module.f90:57-1663).
                                At the isfluid = -1 nodes of the plane next to each wall (tangential indices
                                1 .. l-2) the wall links' bounce-back populations are replaced by those of
                                the face's state; the wall nodes of the face take the phi of their
                                neighbour; with phi_correction the mass target moves by the phi carried
                                through the faces (BCPHIFLUX) */
    int openbc_type[3][2];   /* per axis (x, y, z) and side (low, high), openbc_type_x/y/z: 2 zero gradient
                                (the node's own P and u), 1 pressure (openbc_press, the node's u), any other
                                value velocity (the node's P, openbc_vel) */
    double openbc_press[3][2];   /* pressure moment P of a pressure face (openbc_press_x/y/z) */
    double openbc_vel[3][2][3];  /* (u, v, w) of a velocity face (openbc_u/v/w_x/y/z) */
    int bounce_back;         /* BOUNCE_BACK (requires obstacles): half-way bounce-back -- a link whose upstream
                                node is solid brings the node's own post-collision population of the opposite
                                link (fused_LB_kernel_bb, lb_cuda_fused_module.f90:20-424) -- instead of the
                                moment-space correction of LB_int_boundary */
    int repulsive_flux;      /* REPULSIVE_FLUX (requires twocomponent): before each step every interfacial node
                                pairs with the nearest facing interface within 3 nodes and gets a film
                                repulsion force, added (capped at 1e-3) in the moments prologue
                                (lb_cuda_repulsive_module.f90:19-292, lb_cuda_moments_module.f90:148-160) */
    double a_rep, cos_opp_t, q_th;  /* A_rep, cosOppT, q_th of the &fluid namelist: strength, facing threshold
                                       of n1 . n2, interface threshold of phi (1 - phi) */
} lbf_params;

typedef struct lbf_handle lbf_handle;

/* Library version string; never fails. */
const char* lbf_version(void);

/* Message of the last failed call on this thread (truncated to n bytes). */
int lbf_last_error(char* buf, size_t n);

/* Replaces setup_cuda + allocate_struct (lb_cuda_driver_module.f90:44-168,
 * allocate_module.f90:10-71): validates the parameters and allocates the
 * device state on the current device. */
int lbf_create(const lbf_params* p, lbf_handle** out);

/* Frees the device state (the reference frees at program end). */
int lbf_destroy(lbf_handle* h);

/* Optional CUDA stream (cudaStream_t) for all later work of this handle. */
int lbf_set_stream(lbf_handle* h, void* cuda_stream);

/* isfluid as produced by LBFAST.f90:258-325 (values 1, -1, 0; int8, lx*ly*lz,
 * Fortran order).  Required when obstacles = 1; otherwise all nodes are fluid. */
int lbf_set_isfluid(lbf_handle* h, const int8_t* isfluid);

/* Initial state, replacing the host->device mirror of hfields_flip /
 * phifields_flip after initial_conditions_all (init_conditions_module.f90:15-589).
 * mom10: 10 consecutive fields (P,u,v,w,Pxx,Pyy,Pzz,Pxy,Pxz,Pyz), each lx*ly*lz
 * in Fortran order; phi: lx*ly*lz (two components; may be NULL otherwise).
 * Both time levels receive these values, as `hfields_flop=hfields_flip`
 * (init_conditions_module.f90:584-587).  dtype: LBF_F32 or LBF_F64. */
int lbf_set_fields(lbf_handle* h, const void* mom10, const void* phi, int dtype);

/* Advances nsteps time steps: the body of the integrator loop
 * (integrator_module.f90:270-825).  The first call after lbf_set_fields also
 * performs the integrator's pre-loop wetting (integrator_module.f90:186-190).
 * Asynchronous with respect to the host; errors of earlier launches surface
 * here or at the next synchronising call. */
int lbf_step(lbf_handle* h, int nsteps);

/* Waits for the handle's stream and reports any device-side failure. */
int lbf_sync(lbf_handle* h);

/* Number of steps done since lbf_set_fields. */
int lbf_get_step(lbf_handle* h, long long* step);
/* The kernel tile height and z segment (0: persistent schedule, < 0: columns
 * split at plane -zseg) in use, after the autotuner if it ran. */
int lbf_get_tuning(lbf_handle* h, int* tile_y, int* zseg);

/* State a next step starts from: moments (10 x N), phi (N) and the velocity
 * after the force half-step of the last step (3 x N, the u_old of the next
 * DENSRATIO force).  Any pointer may be NULL.  dtype: LBF_F32 or LBF_F64. */
int lbf_get_fields(lbf_handle* h, void* mom10, void* phi, void* uold, int dtype);

/* copy_print (print_module.f90:638-776, stepskip = 1) of the last step:
 * rho (phi with printphi, rho_phi for two components with density ratio,
 * phi for two components without, P for one component), vel (3 x N,
 * interleaved per node as the reference's velprint(1:3,i,j,k)), press (P).
 * float32, Fortran order.  Any pointer may be NULL. */
int lbf_get_print_fields(lbf_handle* h, float* rho, float* vel, float* press);

/* Global sums in FP64 over fluid nodes (|isfluid| = 1): sum of phi, of P
 * (mass) and of u, v, w (momentum), computed on the device.
 * Counterpart of the reference's phi_sum_count_kernel
 * (lb_cuda_boundary_module.f90:461-515) and sum_world_float
 * (mpi_module.f90:7491-7560) on one rank.  out[5] = {phi, P, u, v, w}.
 * Returns LBF_E_NUMERIC (with the sums written) when a sum is not finite:
 * the check a driver calls every few steps to stop a run that blew up. */
int lbf_reduce(lbf_handle* h, double out[5]);

/* ---- z slabs: one box split over several handles / GPUs ----
 * Replaces the reference's MPI decomposition of the box and its halo
 * exchange (mpi_module.f90:2203-3650: exchange_hfields/phifields/auxfields/
 * forces_sendrecv, packed per direction at :2991-3210) for a split along z of
 * a box periodic in z.  lbf_create_slab makes a handle on planes [z0, z1) of
 * the box in `global` (at least 3 planes) with 3 halo planes on each side;
 * its fields (lbf_set_isfluid, lbf_set_fields, lbf_get_fields) are the
 * slab's box of z1 - z0 + 6 planes, halo planes included.  lbf_step advances
 * the slab's own planes from the current halo planes.  Between steps the
 * halos are refilled: lbf_slabs_exchange copies them between the slabs of
 * one process (a periodic ring, slabs[i] above slabs[i-1]; peer copies when
 * the slabs are on different GPUs), or the caller copies the regions of
 * lbf_slab_region across processes (NCCL send/recv): for side 0 (low z) / 1
 * (high z) and recv 0 / 1, the device address and byte count of the 3 planes
 * of field `field` (0 .. lbf_slab_nregions - 1) of the current time level
 * that a neighbour receives / that this slab receives; a side-1 send region
 * goes to the side-0 receive region of the slab above.  Call the exchange
 * also once after the first lbf_step(h, 0), which applies the pre-loop
 * wetting.  Every node's arithmetic is the single box's: the slabs together
 * give its bits.  Not for phi_correction, repulsive_flux or openbc (box-wide
 * sums and windows) -> LBF_E_UNSUPPORTED; lbf_reduce of a slab too. */
int lbf_create_slab(const lbf_params* global, int z0, int z1, lbf_handle** h);
int lbf_slab_nregions(lbf_handle* h, int* n);
int lbf_slab_region(lbf_handle* h, int side, int recv, int field, void** ptr, size_t* bytes);
int lbf_slabs_exchange(lbf_handle* const* slabs, int n);
/* nsteps steps of the slabs of one process (on one GPU or several) with the
 * halo exchange of each step overlapped with the planes that do not read the
 * halos (4 planes from each face inward), as the reference's ASYNCMPI split
 * does (integrator_module.f90:278-368): per slab the inner planes run while
 * the halos of the step's input are copied on a second stream, then the
 * planes next to the halos.  Primes fresh slabs and exchanges once first;
 * ends with the halos of the new time level filled. */
int lbf_slabs_step(lbf_handle* const* slabs, int n, int nsteps);

/* ---- full-state checkpoint ----
 * No counterpart in the reference, whose restart (lbf_write_restart_raw) is
 * one time level in float32 and so resumes a run only approximately.  The
 * checkpoint holds every stored field of both time levels in the storage
 * precision, the wetting ghost values not yet written, the phi
 * mass-correction sums, the storage scales, the step count and the
 * time-level index; a run resumed from it continues bit for bit.
 * lbf_read_checkpoint needs a handle created with the same parameters (and,
 * with obstacles, the same isfluid set first); it returns LBF_E_ARG for a
 * checkpoint of another box, storage or configuration. */
int lbf_write_checkpoint(lbf_handle* h, const char* path);
int lbf_read_checkpoint(lbf_handle* h, const char* path);

/* ---- allocation-free reduction ----
 * No counterpart in the reference.  For callers that cannot let a library
 * allocate device memory while they run: a Fortran integrator whose device
 * arrays belong to OpenACC data regions and reach the library only as device
 * pointers, a host application that hands out all device memory from its
 * own pool, a solver held to a fixed device memory budget (an allocation
 * inside a call could fail or push it over).  Computes the same FP64 sums as lbf_reduce -- phi, P, u, v,
 * w over nodes with isfluid = 1 or -1 -- over caller-owned device arrays:
 * mom10 (float, 10 x lx*ly*lz, only the first four fields are read), phi
 * (float, may be NULL), isfluid (int8, may be NULL = all fluid).  out is a
 * host array of 5 doubles.  It calls no cudaMalloc/cudaFree: its scratch is a
 * file-scope __device__ array of LBF_NOALLOC_MAX_PLANES + 1 rows of five
 * doubles (328 KB held on every GPU that loads the library until process
 * exit); boxes with lz > LBF_NOALLOC_MAX_PLANES are rejected with LBF_E_ARG.
 * mom10, phi and isfluid must be device (or managed) memory of the current
 * device: anything else -- a host address passed without `host_data
 * use_device` -- is rejected with LBF_E_ARG before any launch.  Every call
 * looks up the array's device address with the current device; the first
 * call on a device also loads the kernels there, so make it before any
 * stream capture.  Calls share the array: calls that overlap on the GPU
 * race.  Runs on the legacy default stream, which does not wait for
 * non-blocking streams or OpenACC async queues: the caller synchronises the
 * stream or queue that produced the fields first (`!$acc wait`).  Returns
 * after the totals reached `out`; LBF_E_NUMERIC (sums written) when a sum is
 * not finite, as lbf_reduce does. */
#define LBF_NOALLOC_MAX_PLANES 8192
int lbf_reduce_noalloc(const float* mom10, const float* phi, const int8_t* isfluid, int lx, int ly, int lz,
                       double out[5]);

/* ---- host-side set-up helpers (the driver's part of LBFAST.f90) ---- */

/* LBFAST.f90:258-325: from raw isfluid (1 fluid / 0 solid, as read from
 * isfluid.raw) build the marked array: walls at non-periodic faces when
 * obstacles = 1, then fluid nodes with a non-fluid neighbour become -1. */
int lbf_mark_isfluid(int lx, int ly, int lz, int pbc_x, int pbc_y, int pbc_z, int lattice, int obstacles,
                     const int8_t* raw, int8_t* out);

/* Solid-node phi seeding of init_conditions_module.f90:492-541 (in place). */
int lbf_seed_solid_phi(int lx, int ly, int lz, int lattice, const int8_t* isfluid, double* phi);

/* Taylor-Green initial moments (init_conditions_module.f90:298-314), double,
 * mom10 as in lbf_set_fields. */
int lbf_ic_taylor_green(int lx, int ly, int lz, double u0, double* mom10);

/* Droplet at rest with the Laplace pressure inside (default DOBENCHMARK
 * branch, init_conditions_module.f90:394-426): phi and mom10 on fluid nodes. */
int lbf_ic_droplet(int lx, int ly, int lz, const double center[3], double radius, double width, double sigma,
                   double rho_r, double rho_b, int densratio, const int8_t* isfluid, double* mom10, double* phi);

/* LAMBTEST initial droplet (init_conditions_module.f90:355-393): as
 * lbf_ic_droplet with the x distance halved (an ellipsoid twice as long in x). */
int lbf_ic_lamb(int lx, int ly, int lz, const double center[3], double radius, double width, double sigma,
                double rho_r, double rho_b, int densratio, const int8_t* isfluid, double* mom10, double* phi);

/* Run controls of the `simulation` and `fluid` namelists that are not
 * lbf_params (LBFAST.f90:32-60), with the DOBENCHMARK defaults of
 * LBFAST.f90:159-191. */
typedef struct lbf_run {
    int nsteps, stamp, stamp2D, stamp_term, stepskip;
    int lreadisfluid, lreadinit, lprint, lvtk, lraw, lrestart, lwriterestart;
    int openbc, nplanes, every_time_check;
    int iprobe, jprobe, kprobe;
    double time_limit;
    double uwall, radius, width, center[3];
} lbf_run;

/* Reads the `simulation` and `fluid` namelists of a reference input file
 * (LBFAST.f90:193-232) into p (physics) and run (controls); p->lx..wettab_r
 * and run are first set to the DOBENCHMARK defaults.  The compile-time macro
 * fields of p (lattice, highorder, twocomponent, densratio, obstacles,
 * storage, printphi) are left as the caller set them; openbc and the
 * openbc_* arrays (whole-array or element assignments) go to both p and run.
 * Unknown keys and malformed values are errors. */
int lbf_read_namelists(const char* path, lbf_params* p, lbf_run* run);

/* The reference's restart file <dir>/restart.raw (write_restart_serial_2c /
 * _1c and their readers, print_module.f90:1030-1677): one time level in
 * float32, the ten moments in the reference's file order (P, u, v, w, Pxx,
 * Pxy, Pxz, Pyy, Pyz, Pzz), phi when phi != NULL (two components), then iframe
 * and iframe2D (int32).  mom10 is in this header's order (P, u, v, w, Pxx, Pyy,
 * Pzz, Pxy, Pxz, Pyz), Fortran order.  The reader checks the file size. */
int lbf_write_restart_raw(const char* dir, int lx, int ly, int lz, const float* mom10, const float* phi, int iframe,
                          int iframe2D);
int lbf_read_restart_raw(const char* dir, int lx, int ly, int lz, float* mom10, float* phi, int* iframe,
                         int* iframe2D);

/* VTK ImageData writer of print_vtk_sync (print_module.f90:22-244, 2789-2814):
 * <dir>/out_rho_NNNNNN.vti, out_vel_... (3 components), and out_press_... when
 * press is not NULL, byte for byte in the reference's layout (Float32 data). */
int lbf_write_vtk(const char* dir, int iframe, int lx, int ly, int lz, const float* rho, const float* vel,
                  const float* press);
/* The same files in the reference's PRINTHALF layout (print_module.f90:110-121,
 * mpi_module.f90:3737-3842): the values rounded to IEEE binary16 (round to
 * nearest even), declared DataArray type="UnsignedShort". */
int lbf_write_vtk_half(const char* dir, int iframe, int lx, int ly, int lz, const float* rho, const float* vel,
                       const float* press);

/* raw + XDMF writer of print_raw_sync (print_module.f90:2007-2180): writes
 * <dir>/out_rho_NNNNNN.raw/.xdmf, out_vel_..., and out_press_... when press
 * is not NULL. */
int lbf_write_raw_xdmf(const char* dir, int iframe, int lx, int ly, int lz, const float* rho, const float* vel,
                       const float* press);
/* The same files in the reference's PRINTHALF layout (print_module.f90:2053-2164):
 * binary16 bit patterns (round to nearest even), XDMF NumberType="UInt"
 * Precision="2". */
int lbf_write_raw_xdmf_half(const char* dir, int iframe, int lx, int ly, int lz, const float* rho, const float* vel,
                            const float* press);

/* ---------------------------------------------------------------------------
 * Batched solve server (no counterpart in the reference, which runs one box
 * per process).  Independent solves of uneven box sizes are submitted as they
 * arrive; a solve is admitted when its resident device bytes fit the memory
 * budget (first in, first out), its fields stay in device memory until it
 * finishes, and every time step of all resident solves of one kernel class
 * (lattice, HIGHORDER, TWOCOMPONENT, storage) is ONE kernel launch over a
 * work list of (solve, tile column, z range) items, replayed as a captured CUDA
 * graph of `chunk` steps.  Solves that arrive while others run are admitted
 * at the next chunk boundary.  A solve's result does not depend on what else
 * is resident.  Each call must come from one host thread at a time.
 * ------------------------------------------------------------------------- */
typedef struct lbf_server lbf_server;

typedef struct lbf_server_config {
    long long mem_budget; /* device bytes resident solves may hold; <= 0: 80% of the free memory */
    int max_active;       /* resident solves at most; <= 0: no limit */
    int chunk;            /* steps per graph replay (even; <= 0: 32) */
    int use_graph;        /* 1: replay captured CUDA graphs; 0: launch every step */
} lbf_server_config;

enum { LBF_SOLVE_QUEUED = 0, LBF_SOLVE_ACTIVE = 1, LBF_SOLVE_DONE = 2, LBF_SOLVE_FAILED = 3, LBF_SOLVE_CANCELLED = 4 };

typedef struct lbf_solve_info {
    int state;            /* LBF_SOLVE_* */
    long long steps_done;
    long long nsteps;
    long long device_bytes;
    /* CLOCK_MONOTONIC seconds (Python: time.monotonic()); 0 while not reached */
    double t_submit, t_admit, t_done;
} lbf_solve_info;

int lbf_server_create(const lbf_server_config* cfg, lbf_server** out);
/* waits for the device, frees every resident solve and record */
int lbf_server_destroy(lbf_server* s);
/* Queues one solve of nsteps steps of the box p describes (p->obstacles: isfluid
 * as for lbf_set_isfluid, else NULL) from the fields mom10/phi of lbf_set_fields
 * in dtype; the inputs are copied, the caller may free them on return.  A solve
 * whose resident bytes exceed the budget is rejected with LBF_E_NOMEM. */
int lbf_server_submit(lbf_server* s, const lbf_params* p, const int8_t* isfluid, const void* mom10, const void* phi,
                      int dtype, long long nsteps, long long* id);
/* Admits queued solves that fit, advances the resident ones by up to
 * max_chunks chunks (each ends with a device synchronisation), and retires
 * finished solves (their fields are copied to host memory and their device
 * memory is released, which may admit more).  Returns after max_chunks chunks
 * or when nothing is resident; *active and *queued (either may be NULL) give
 * the counts on return. */
int lbf_server_run(lbf_server* s, int max_chunks, int* active, int* queued);
int lbf_server_poll(lbf_server* s, long long id, lbf_solve_info* info);
/* Copies a finished solve's mom10 and phi (either may be NULL) in the dtype it
 * was submitted with and forgets it; LBF_E_STATE until it is done. */
int lbf_server_fetch(lbf_server* s, long long id, void* mom10, void* phi);
/* Drops a queued or resident solve; its device memory is released at once. */
int lbf_server_cancel(lbf_server* s, long long id);
/* Device bytes a solve of these parameters holds while resident. */
long long lbf_server_solve_bytes(const lbf_params* p);

#ifdef __cplusplus
}
#endif

#endif /* LBFAST_GPU_H */
