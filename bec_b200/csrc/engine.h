// engine.h -- internal interfaces between the C-ABI host code (bec_api.cpp)
// and the kernel files (plain_fp64.cu, batched_fp32.cu, reduce.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "../../include/bec.h"

// ----------------------------------------------------------------------------
// FP64 per-group geometry and physics, passed by value to the plain kernels.
struct GeomD {
    int nx, ny, nz, lx, ly, lz, cells;
    double dkx, dky, dkz;
    double xmax, ymax, zmax, dx, dy, dz, lambda;
    double g11, g12, g22, l111, l12, l22, detuning;
    double dt_evo, dt_steady, dV;
    double Va, Vb;
    int itmax, noise;
    uint64_t seed;
};

// FP32 per-group parameters of the batched path (device array, one per group).
struct GroupParamsF {
    float dkx, dky, dkz;
    float xmax, ymax, zmax, dx, dy, dz, inv_lambda2;
    float g11, g12, g22, l111, l12, l22, detuning;
    float dt;                 // dt_evo, natural units
    float noise_amp;          // sqrt(dt / (2 dV))
    float c1, c2, c3;         // loss-noise amplitudes 3 sqrt(l111/6), sqrt(l12/2), sqrt(l22)
    float init_a, init_b;     // Va / sqrt(dV), Vb / sqrt(dV)
    int itmax, noise;
    uint32_t seed_lo, seed_hi;
    // kinetic phase per unit index squared in turns, 0.5 dk^2 dt_evo / (2 pi) per axis (ky term 0 in
    // 2D): the angle 0.5 k^2 dt reaches several radians at the largest k, so it is formed in FP64 from
    // exact integer indices, k = dk * i, and only its sine and cosine are rounded to FP32
    double kin_x, kin_y, kin_z;
};

// Geometry of one grid class of the batched path (all trajectories sharing nx, ny, nz).
struct ClassGeom {
    int nx, ny, nz, lx, ly, lz, cells;
    int n_traj;
};

// ----------------------------------------------------------------------------
// plain_fp64.cu (one trajectory at a time; a, b point at that trajectory)
void plain_kick(double2 *a, double2 *b, const GeomD &g, double scale, int apply_scale, cudaStream_t s);
void plain_fft3d(double2 *data, const GeomD &g, const double2 *tw_x, const double2 *tw_y,
                 const double2 *tw_z, int inv, cudaStream_t s);
void plain_nl(double2 *a, double2 *b, const GeomD &g, uint32_t traj, uint32_t step, cudaStream_t s);
void plain_scale(double2 *a, int n, double scale, cudaStream_t s);
void plain_pulse(double2 *a, double2 *b, int n, double2 m11, double2 m12, double2 m21, double2 m22,
                 cudaStream_t s);
void plain_init(double2 *a, double2 *b, const double2 *gs, const double2 *noise_a, const double2 *noise_b,
                const GeomD &g, uint32_t traj, cudaStream_t s);
// per-z sums (|a|^2, |b|^2, Re, Im conj(a) b) of x-space arrays into out[nz][4], accumulating
void plain_axial_sums(const double2 *a, const double2 *b, const GeomD &g, double *out, cudaStream_t s);
// ground state
void plain_gs_tf(double2 *a, const GeomD &g, double mu, cudaStream_t s);
void plain_gs_kick(double2 *a, const GeomD &g, cudaStream_t s);
void plain_gs_nl(double2 *a, const GeomD &g, cudaStream_t s);
// sums of |a|^2 into out[0] (device scalar, Neumaier); tmp has >= 2*1024 doubles
void plain_norm(const double2 *a, int n, double *out, double *tmp, cudaStream_t s);
// a *= sqrt(N / (sum * dV)) with sum read from device memory
void plain_renorm(double2 *a, int n, const double *sum, double N, double dV, cudaStream_t s);
// x-space sums: out[0] = sum n V, out[1] = sum n^2, out[2] = sum n
void plain_gs_xsums(const double2 *a, const GeomD &g, double *out, double *tmp, cudaStream_t s);
// out[0] = sum |a - prev|^2, out[1] = sum |a|^2
void plain_diff2(const double2 *a, const double2 *prev, int n, double *out, double *tmp, cudaStream_t s);
// k-space sum of |ak|^2 k^2/2 into out[0]
void plain_gs_ksum(const double2 *ak, const GeomD &g, double *out, double *tmp, cudaStream_t s);
// reference energy integrand sum (wigner_kernel.cu:232-258) into out[0]
void plain_gs_ref_energy(const double2 *ax, const double2 *ak, const GeomD &g, double *out, double *tmp,
                         cudaStream_t s);
// h = (V + g11 n - mu) psi + hk (hk = FORWARD(psik k^2/2)); out[0] = sum |h|^2
void plain_gs_residual(const double2 *ax, const double2 *hk, const GeomD &g, double mu, double *out,
                       double *tmp, cudaStream_t s);
// hk = ak * k^2/2
void plain_mul_k2(const double2 *ak, double2 *hk, const GeomD &g, cudaStream_t s);

// ----------------------------------------------------------------------------
// batched_fp32.cu
struct ZPassArgs {
    float pre;            // kick fraction before the observation (0 or 0.5)
    float post;           // kick fraction after it (0 or 0.5)
    float scale;          // applied after the inverse z transform (1 / cells)
    float out_scale;      // applied before the forward z transform: 1 when a plane pass
                          // follows, nx*ny when the pass ends a step (see batched_fp32.cu)
    int has_m1;           // 1: apply matrix m1 before the observation
    float2 m1[4];         // row-major 2x2 (m11, m12, m21, m22)
    int observe;          // 1: write per-z partial moments
    int has_m2;           // 1: apply matrix m2 after the observation
    float2 m2[4];
};

// x-space initial state of ne consecutive trajectories of one group (GS + vacuum noise);
// noise == NULL draws from Philox, else [traj][a|b][cell] float2
void fp32_init_group(float4 *state, int cells, int ne, const GroupParamsF &gp, const double2 *gs,
                     const float2 *noise, cudaStream_t s);
// k_init for n_traj consecutive trajectories of a class from many ensembles: tgroup / tlocal of the run,
// gs_ptrs[group] the ensemble's device ground state, in the element type of host_type (BEC_HOST_*)
void fp32_init_batched(float4 *state, int cells, int n_traj, const int *tgroup, const int *tlocal,
                       const GroupParamsF *gp, const void *const *gs_ptrs, int host_type, cudaStream_t s);
// x-space -> stored representation (inverse transform over x and y)
void fp32_prep(float4 *state, const ClassGeom &c, const float2 *tw_x, const float2 *tw_y, cudaStream_t s);
// stored representation -> x-space (forward transform over x and y)
void fp32_unprep(float4 *state, const ClassGeom &c, const float2 *tw_x, const float2 *tw_y, cudaStream_t s);
void fp32_zpass(float4 *state, const ClassGeom &c, const GroupParamsF *gp, const int *tgroup,
                const float2 *tw_z, const ZPassArgs &z, double *obs_partial, cudaStream_t s);
void fp32_ppass(float4 *state, const ClassGeom &c, const GroupParamsF *gp, const int *tgroup,
                const int *tlocal, const float2 *tw_x, const float2 *tw_y, const uint32_t *d_step, cudaStream_t s);
// the plane passes read the Philox step index from a device scalar, so a captured step graph can replay:
// an eagerly launched step writes it (fp32_put_step); a step advances it at its end (fp32_inc_step, or the
// last CTA of a plane launch given inc_done, or of the fused step kernel)
void fp32_put_step(uint32_t *d_step, uint32_t v, cudaStream_t s);
void fp32_inc_step(uint32_t *d_step, cudaStream_t s);
int fp32_zpass_tiles(const ClassGeom &c);   // tiles per trajectory of the z pass (obs_partial layout)
// obs_partial[traj][tile][z][4] -> traj_axial[traj][z][4] * traj_scale[traj] (1 if NULL),
// traj_tot[traj][4] = sum over z; traj_axial may be NULL
void obs_reduce(const double *obs_partial, int n_traj, int tiles, int nz, const double *traj_scale,
                double *traj_axial, double *traj_tot, cudaStream_t s);
// group sums: for g: out[g][4] = sum_{t in group} traj_tot[t]; trajectories of a group are contiguous
// FP64 sums (|a|^2, |b|^2, conj(a) b) of every trajectory's stored state in `blocks` ranges each, times scale,
// into part[traj][block][4] (k_obs_reduce's layout with `blocks` tiles and nz = 1)
void fp32_state_sums(const float4 *state, int cells, int n_traj, int blocks, double scale, double *part,
                     cudaStream_t s);
void group_reduce(const double *traj_tot, const int *group_first, const int *group_count, int n_groups,
                  double *out, cudaStream_t s);

// gs_passes.cu: batched FP32 imaginary-time ground states (one trajectory per group)
struct GsParamsF {
    double N;                 // target norm
    double parseval;          // cells * dV: N' = parseval * sum |psi_k|^2
    float dt_steady;          // natural units
    float mu;                 // Thomas-Fermi chemical potential (start profile)
};
bool gs_batched_supported(const ClassGeom &c);
void gs_init(float2 *state, const ClassGeom &c, const GroupParamsF *gp, const GsParamsF *gs, const int *tgroup,
             const float2 *warm, cudaStream_t s);
void gs_prep(float2 *state, const ClassGeom &c, const GroupParamsF *gp, const GsParamsF *gs, const int *tgroup,
             cudaStream_t s);
// active (device, c.n_traj entries, may be NULL = 0 .. n_traj-1): the class-local trajectories this launch
// processes, so converged trajectories can leave the batch
void gs_plane_step(float2 *state, const ClassGeom &c, const GroupParamsF *gp, const GsParamsF *gs, const int *tgroup,
                   const double *norm_in, double *norm_clear, cudaStream_t s, const int *active = nullptr);
// FFT_xy of the stored state times in_scale * sqrt(N / N'): x-space rows to out, sums (n V, n^2, n,
// |u - previous out|^2) to xsums[4 traj ..]
void gs_output(float2 *state, const ClassGeom &c, const GroupParamsF *gp, const GsParamsF *gs, const int *tgroup,
               const double *norm_in, float2 *out, double *xsums, float in_scale, cudaStream_t s,
               const int *active = nullptr);
// kick exp(-dt frac1 k^2/2) * scale [measure] then exp(-dt frac2 k^2/2) * out_scale
void gs_pencil(float2 *state, const ClassGeom &c, const GroupParamsF *gp, const GsParamsF *gs, const int *tgroup,
               const float2 *tw_full, float frac1, float frac2, float scale, float out_scale, double *norm,
               double *ekin, cudaStream_t s, const int *active = nullptr);

void gs_to_double(const float2 *in, double2 *out, size_t n, cudaStream_t s);

// warmstart.cu: the 64-term correction over Thomas-Fermi (one grid per call), from the
// built-in analytic basis or from a table of basis rows installed for that grid
struct WsTable {
    int nx = 0, ny = 0, nz = 0, nb = 0;
    float *d_basis = nullptr;          // nb x cells, grid index order
    std::vector<double> gram;          // 64 x 64 Gram matrix (the identity beyond nb)
};
int warmstart_basis_size();
cudaError_t warmstart_table_init(WsTable &t, const float *host_basis, cudaStream_t s);
cudaError_t warmstart_project(const float2 *psi, int n, const bec_derived *d, const WsTable *tab, double *coef_out,
                              float *profile_out, cudaStream_t s);
cudaError_t warmstart_synth(const double *coef, int n, const bec_derived *d, const WsTable *tab, float2 *psi_out,
                            cudaStream_t s);

// render.cu: projections after the reference's second pi/2 and the colour ramp
void render_project(const float4 *x, const ClassGeom &c, float in_scale, float sub, float *xy_a, float *xy_b,
                    float *zy_a, float *zy_b, cudaStream_t s);
void render_colour(const float *level, int n, float max_level, float4 *rgba, cudaStream_t s);

// launch counter (kernels this library enqueued since the counter was reset)
extern thread_local long long g_launches;
// Sets the kernel's dynamic shared memory limit to `bytes` on the current device, once per (kernel, device);
// safe from several host threads (a process may drive several GPUs).
cudaError_t ensure_smem_limit(const void *kernel, int bytes);

// fused_passes.cu: register-resident passes (square planes 8/16/32; nz = 64/128/256)
bool fp32_fast_plane_supported(const ClassGeom &c);
bool fp32_fast_pencil_supported(const ClassGeom &c);
// occupancy: 0 = 16 warps per SM, no spill; 1 = 20 warps per SM at 96 registers (an autotuner choice)
void fp32_plane_fast(float4 *state, const ClassGeom &c, const GroupParamsF *gp, const int *tgroup, const int *tlocal,
                     uint32_t *d_step, int occupancy, int *inc_done, cudaStream_t s);
// CTAs of that launch; inc_done != NULL: its last CTA also advances *d_step (inc_done: a zero int counter)
int fp32_plane_fast_ctas(const ClassGeom &c);
// tw_full: nz entries W_nz^e; frac: kick in units of dt; scale: 1/cells times out_scale;
// m: optional pulse matrix (row-major, 4 entries) or NULL; obs: when not NULL the pass
// ends a step and writes per-z partial moments [traj][tile][z][4] (tiles = fp32_fast_pencil_tiles)
// kin: the class's kinetic phase table for frac (fp32_kin_tables), or NULL to evaluate the phases in place
void fp32_pencil_fast(float4 *state, const ClassGeom &c, const GroupParamsF *gp, const int *tgroup,
                      const float2 *tw_full, float frac, float scale, const float2 *m, double *obs,
                      float out_scale, const float2 *kin, cudaStream_t s);
// kinetic phase factors of a class for kick fraction frac: per class-local trajectory t, tab[t * (nz + nx ny) + i]
// = e^{+i kz_i^2/2 dt frac} for i < nz, then e^{+i (kx^2 + ky^2)/2 dt frac} per pencil (y * nx + x)
void fp32_kin_tables(float2 *tab, const ClassGeom &c, const GroupParamsF *gp, const int *tgroup, float frac,
                     cudaStream_t s);
// onchip_step.cu: a steady step (full kick, no pulse, no observation) of an 8x8x64 class with each trajectory's
// state in shared memory, one launch instead of its pencil and plane launches; kin_full: the class's full-kick
// kinetic table; inc_done as fp32_plane_fast
bool fp32_onchip_supported(const ClassGeom &c);
void fp32_onchip_step(float4 *state, const ClassGeom &c, const GroupParamsF *gp, const int *tgroup, const int *tlocal,
                      const float2 *tw_full, const float2 *kin_full, uint32_t *d_step, int *inc_done, cudaStream_t s);
// pencil_tma.cu: the non-observing pencil pass as a persistent kernel with TMA tile loads and stores
// (bit-identical to fp32_pencil_fast); d_err: set to 1 when a wait gave up; d_never: a zero int
bool fp32_pencil_tma_supported(const ClassGeom &c);
cudaError_t fp32_pencil_tma(float4 *state, const ClassGeom &c, const float2 *tw_full, float frac, float scale,
                            const float2 *m, const float2 *kin, int *d_err, const int *d_never, cudaStream_t s);
int fp32_fast_pencil_tiles(const ClassGeom &c);

// step_kernel.cu: one launch per split step for the classes of the register passes. Items of the work
// list are int4 (kind | class << 4, class-local trajectory, item index within the trajectory, counter
// index of the trajectory).
struct StepClassDev {
    float4 *state;
    const int *tgroup, *tlocal;
    const float2 *tw;         // W_nz^e, e < nz
    const float2 *kin[2];     // kinetic phase tables for kick fractions 0.5 and 1 (fp32_kin_tables)
    int nx, ny, nz, lx, cells, tiles, n_traj;
    int pencil_items;         // pencil items per trajectory (filled by step_plan_build)
};
struct StepLaunch {
    const StepClassDev *cls;
    const GroupParamsF *gp;
    const int4 *items;
    int n_items;
    int *queue, *finished, *err, *done;
    int n_counters;
    uint32_t *d_step;
    int wait, inc_step;
    int stall;                // added to every plane item's dependency count (fault injection in tests)
    unsigned long long wait_limit_ns;
};
constexpr int kStepCandidates = 5;     // two-phase, then interleaved at 0.5, 1, 2, 4 waves
struct StepPlan {
    bool ready = false;
    int candidate = -1;
    bool two_phase = false;
    int grid = 0, n_items = 0, n_pencil = 0, n_plane = 0, n_counters = 0;
    int4 *d_items = nullptr;
    StepClassDev *d_cls = nullptr;
    int *d_counters = nullptr;          // queue, finished, error flag, pad, then one per trajectory
    int stall = 0;                      // BEC_STEP_INJECT_STALL: plane items wait for a count never reached
    unsigned long long wait_limit_ns = 2000000000ull;   // BEC_STEP_WAIT_LIMIT_MS
};
bool step_class_supported(const ClassGeom &c);
const char *step_plan_name(int candidate);
// builds (or rebuilds, reusing the buffers) the work list of candidate `candidate` for the classes geoms
// (cls: their device descriptors; traj_offset: first counter index of each)
cudaError_t step_plan_build(StepPlan &P, const std::vector<ClassGeom> &geoms, const std::vector<StepClassDev> &cls,
                            const std::vector<int> &traj_offset, int candidate, cudaStream_t s);
void step_plan_free(StepPlan &P);
// one split step (kick fraction frac of dt, optional pulse matrix m) of every class in the plan; the
// last CTA advances *d_step
void step_launch(const StepPlan &P, const GroupParamsF *gp, uint32_t *d_step, float frac, const float2 *m,
                 cudaStream_t s);
// *err = 1 if a dependency wait of a launch since the plan was built gave up (synchronises s)
cudaError_t step_read_error(const StepPlan &P, int *err, cudaStream_t s);
// per-process cache of the autotuned candidate for a class mix on this device (-1: per-pass launches)
bool step_plan_cached(const std::vector<ClassGeom> &geoms, int *candidate);
void step_plan_remember(const std::vector<ClassGeom> &geoms, int candidate);
