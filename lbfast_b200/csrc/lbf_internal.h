// lbf_internal.h -- declarations shared by the translation units of the
// library (not part of the C ABI).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#include "../../include/lbfast_gpu.h"

namespace lbf {

constexpr int NSCALE_H = 14;

// Storage-agnostic arguments of one fused step launch.
struct StepArgs {
    int nx, ny, nz, pbx, pby, pbz;
    int densratio, obstacles, write_u, zseg, smag;
    int zlo, zhi;           // the planes advanced (a slab: its interior planes)
    double omega, visc1, visc2, rho_r, rho_b, beta, kapp, sharp_c, tau_diff, fx, fy, fz;
    double scale[NSCALE_H];
    const void* min;
    void* mout;
    const void* uin;
    void* uout;
    const void* pin;
    void* pout;
    const float* pres_in;   // P, u, v, w with 16-bit storage (4 x N)
    float* pres_out;
    const int8_t* isf;
    int* err;
    const void* rep;        // REPULSIVE_FLUX force of the step (3 x N, arithmetic type), or nullptr
    const double* mass;     // phi mass correction: sums of the step's input phi (see launch_mass), or nullptr
};

using StepLauncher = cudaError_t (*)(const StepArgs&, cudaStream_t);

// Step launcher of one kernel class (lattice 19/27, HIGHORDER, TWOCOMPONENT)
// for a storage type and tile height (8 or 16 rows); nullptr if not built.
StepLauncher step_launcher(int storage, int lat, int ho, int tc, int obs, int tile_y);
// kernel class argument `tc` of a run: 0 one component, 1 two components,
// 2 two components with REPULSIVE_FLUX (its own compilation of the step)
inline int kernel_tc(const lbf_params& p) { return p.twocomponent ? (p.repulsive_flux ? 2 : 1) : 0; }
// kernel class argument `obs`: the compilation with the obstacle code, which
// also carries the phi mass correction of the step's input phi
inline int kernel_obs(const lbf_params& p) { return (p.obstacles || p.phi_correction) ? 1 : 0; }
bool tile_available(int storage, int tile_y);

// Batched step of many boxes of one kernel class and tile height: fill writes
// the device-format parameters of one box (params_bytes bytes) from its
// StepArgs; launch runs one CTA per work item (int4: box, first and end
// column-plane of the box, column index = tile y * tiles in x + tile x, plane
// fastest); resident gives the CTAs of the batched kernel one SM holds.
struct BatchOps {
    size_t params_bytes;
    int tile_y;
    void (*fill)(const StepArgs&, void*);
    cudaError_t (*launch)(const void* d_boxes, const int4* d_work, int nwork, cudaStream_t st);
    int (*resident)();
};
// resident CTA slots of the current GPU (SMs x CTAs per SM), and the CTAs of a
// persistent launch over W column-planes (no share shorter than 8 planes)
int resident_slots(int resident_per_sm);
int persistent_grid(long long W, int resident_per_sm);
BatchOps batch_ops(int storage, int lat, int ho, int tc, int obs, int tile_y);
// CTA tile width of the step kernel in nodes (the height is 8 or 16)
constexpr int STEP_TILE_X = 32;

// wetting tables (solid nodes whose ghost phi the reference updates)
struct WetArgs {
    int n;                    // entries
    int nx, ny, nz, pbx, pby, pbz;
    const long long* s_idx;   // solid node
    const int* donor;         // 3 x n wrapped donor coordinates
    const int* flag;          // WET_*
    const double* wn;         // 3 x n unit wall normal
    const int* shift;         // 3 x n link shift -c of the donor link
    double cot_theta;
    const void* pin;          // phi read (ghost before update, donor phi, donor stencil)
    void* wout;               // new ghost values (n)
    void* scatter_dst;        // phi buffer receiving scatter_src (or nullptr)
    const void* scatter_src;  // ghost values of the previous step
    int prime;                // integrator pre-loop call: aux = 0 and halos = 0
};
enum { WET_NORMAL = 0, WET_OUTSIDE = 1, WET_HIGHWRAP = 2, WET_OPENCOPY = 3 };

cudaError_t launch_wetting(int storage, const WetArgs& a, cudaStream_t st);
cudaError_t launch_wet_apply(int storage, int n, const long long* s_idx, const void* src, void* dst, cudaStream_t st);

// host array <-> device field conversions
cudaError_t launch_convert_in(int storage, bool is_phi, const void* src, int src_dtype, void* dst, long long n,
                              double scale, cudaStream_t st);
cudaError_t launch_convert_out(int storage, bool is_phi, const void* src, void* dst, int dst_dtype, long long n,
                               double inv_scale, cudaStream_t st);

// copy_print extraction
struct PrintArgs {
    long long N;
    int mode;            // 0: P, 1: phi, 2: rho_phi
    double rho_r, rho_b;
    const void* P;       // moment field 0 (float array with 16-bit storage)
    const void* vel;     // 3 consecutive velocity fields (storage type)
    const float* vel32;  // or, when not null, 3 consecutive FP32 velocity fields
    const void* phi;
    double sP, su[3];    // inverse scales
    float* rho;
    float* vel_out;      // interleaved 3 x N
    float* press;
    const double* mass;  // phi mass correction of the printed step's input phi, or nullptr
    const int8_t* isf;   // isfluid with obstacles, else nullptr (all fluid)
};
cudaError_t launch_print(int storage, const PrintArgs& a, cudaStream_t st);

// FP64 reductions over fluid nodes: out[5] = {sum phi, sum P, sum u, sum v, sum w}
// (16-bit storage: P, u, v, w from pres)
cudaError_t launch_reduce(int storage, long long N, const void* mom, const float* pres, const void* phi,
                          const int8_t* isf, const double* inv_scale, double* d_out, cudaStream_t st);

// 16-bit upload, on the 10 host fields staged in device memory (f32 or f64,
// src_dtype): the largest finite |u|, |v|, |w| and |Pi - u u| as float bits
// in d_max[0..1], and component c (0..5) of Pi - u u converted to the storage
// type with a scale
cudaError_t launch_upload_maxabs(int src_dtype, long long N, const void* staged10, unsigned* d_max, cudaStream_t st);
cudaError_t launch_upload_pin(int storage, int src_dtype, long long N, const void* staged10, int c, void* dst,
                              double scale, cudaStream_t st);
// 16-bit download: component c of Pi = (Pi - u u) + u u from the stored
// fields (mom: the six 16-bit Pi - u u fields, inv_scale per moment field;
// vel32: the FP32 u, v, w) into dst (dst_dtype)
cudaError_t launch_download_pi(int storage, int dst_dtype, long long N, const void* mom, const float* vel32,
                               const double* inv_scale, int c, void* dst, cudaStream_t st);

// phi mass correction, d_mass = {sum, count, sum0, flux}.  MASS_INITIAL
// stores the FP64 sum of phi over fluid nodes in d_mass[2]; MASS_SUM puts the
// sum and the count of 0.5 < phi < 0.9 in d_mass[0..1] (the kernels of the
// step then correct those nodes' values where they read them, see mass_corr);
// MASS_APPLY also adds (d_mass[2] + d_mass[3] - sum) / count to those nodes in
// memory (the pre-loop correction).  d_mass[3] is the open-face flux of the
// state (0 without open faces).  No host synchronisation (graph-capturable).
enum MassMode { MASS_INITIAL = 0, MASS_SUM = 1, MASS_APPLY = 2 };
cudaError_t launch_mass(int storage, MassMode mode, long long N, void* phi, const int8_t* isf, double* d_mass,
                        cudaStream_t st);

// Wall passes after a step, on the step's output moments, at isfluid = -1
// nodes; each recomputes its nodes' moments after the force half-step from the
// step's input buffers, which the step leaves intact (lbf_walls.cu).
//  * open face (axis 0/1/2, side 0 low / 1 high): replaces the bounce-back
//    populations of the wall links by those of the face's state
//    (boundary_cds_module.f90:57-1311); one launch per face, in the
//    reference's order x low, x high, y low, ..., z high.
//  * BOUNCE_BACK (lb_cuda_fused_module.f90:20-424): replaces the step's
//    moment-space bounce-back of the wall links by the half-way bounce-back
//    of the node's own post-collision populations, over the nodes of `nodes`.
struct BoundaryArgs {
    int nx, ny, nz, pbx, pby, pbz;
    int axis, side, type;       // type: 2 zero gradient, 1 pressure, other velocity
    double press, vel[3];
    int lattice, highorder, tc, dr;
    double omega, visc1, visc2, rho_r, rho_b, beta, kapp, sharp_c, tau_diff, fx, fy, fz;
    int smag;                   // SMAGORINSKI relaxation in the collision
    const void* rep;            // REPULSIVE_FLUX force of the step (3 x N, arithmetic type), or nullptr
    const long long* nodes;     // BOUNCE_BACK: the isfluid = -1 nodes
    long long nnodes;
    const int8_t* isf;
    const void* min;            // the step's input moments
    const float* pres_in;       // the step's input P, u, v, w (16-bit storage, 4 x N)
    const void* uin;            // the step's input u_old (DENSRATIO)
    const void* phi;            // the step's input phi (two components)
    void* mom;                  // the step's output moments
    float* pres;                // the step's output P, u, v, w (16-bit storage, 4 x N)
    double scale[NSCALE_H];
    const double* mass;         // phi mass correction of the step's input phi (see launch_mass), or nullptr
};
cudaError_t launch_open_face(int storage, const BoundaryArgs& a, cudaStream_t st);
cudaError_t launch_bounce_back(int storage, const BoundaryArgs& a, cudaStream_t st);

// phi carried through the open faces by a state (BCPHIFLUX,
// boundary_cds_module.f90:1667-1861): sum over the isfluid = -1 nodes of the
// planes next to the walls of +-u_n phi, into d_flux (set, not added)
cudaError_t launch_phi_flux(int storage, int nx, int ny, int nz, int open, const void* mom, const float* pres,
                            const void* phi, const int8_t* isf, const double* inv_scale, double* d_flux,
                            cudaStream_t st);

// REPULSIVE_FLUX before a step (lbf_repulsive.cu): the film-repulsion force
// of every node from the step's input phi into `force`
struct RepulsiveArgs {
    int nx, ny, nz, pbx, pby, pbz;
    double width, a_rep, cos_opp_t, q_th;
    const int8_t* isf;          // nullptr without obstacles
    const void* phi;            // the step's input phi
    double* nrm;                // 3 x N normals (work array)
    void* force;                // 3 x N force, arithmetic type of the storage
    const double* mass;         // phi mass correction of the step's input phi (see launch_mass), or nullptr
};
cudaError_t launch_repulsive(int storage, const RepulsiveArgs& a, cudaStream_t st);

size_t storage_bytes(int storage);

// sets the message returned by lbf_last_error on the calling thread
void record_error(const char* msg);
size_t phi_bytes(int storage);

}  // namespace lbf
