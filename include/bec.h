/*
 * bec.h -- C ABI of the B200 split-step Gross-Pitaevskii / truncated-Wigner engine.
 *
 * Plain C types only: pointers, sizes, doubles. No CUDA or C++ types cross this
 * boundary, so any FFI (ctypes, cgo, JNI, N-API) can bind it.
 *
 * The reference reaches its hot path through free C functions declared in
 * programs/bec_wigner_3d.cuda/wigner.cpp:32-40 (initConstants,
 * calculateSteadyState, initEvolution, calculateEvolution, initWaveVectors,
 * releaseWaveVectors) that read a process-global __constant__ parameter block
 * and texture (wigner_kernel.cu:8-12) and abort the process on any error
 * (cutilSafeCall). This ABI keeps the same operations and parameter surface
 * (defines.h:25-54) but
 *   - holds all state in an explicit context (one per host thread),
 *   - returns a status code instead of aborting,
 *   - lets the caller own every host array and the context own device memory.
 *
 * Complex arrays on the host are interleaved doubles (re, im), x fastest:
 * index = ((z * nvy + y) * nvx + x)  (wigner_kernel.cu:29-34, :101-106).
 */
#ifndef BEC_H
#define BEC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BEC_ABI_VERSION 3

typedef enum bec_status {
    BEC_OK = 0,
    BEC_ERR_INVALID_ARG = 1,      /* bad pointer, size or parameter value */
    BEC_ERR_UNSUPPORTED_GRID = 2, /* grid not a supported power-of-two shape */
    BEC_ERR_CUDA = 3,             /* a CUDA runtime call failed; see bec_last_error */
    BEC_ERR_OUT_OF_MEMORY = 4,    /* device allocation failed (or would pass BEC_DEVICE_BYTES_LIMIT) */
    BEC_ERR_STATE = 5,            /* call out of order (e.g. evolve before init) */
    BEC_ERR_NUMERICAL = 6,        /* NaN/Inf or norm blow-up detected in a reduction */
    BEC_ERR_NO_DEVICE = 7,        /* no CUDA device visible */
    BEC_ERR_UNIMPLEMENTED = 8
} bec_status;

/* Execution paths. */
enum {
    /* One trajectory at a time, one kernel per operation, FP64 throughout:
     * structured like the reference's propagate() (wigner.cu:178-199). */
    BEC_PATH_FP64_PLAIN = 0,
    /* All trajectories of all groups in fused FP32 passes with FP64
     * compensated reductions; the product path. */
    BEC_PATH_FP32_BATCHED = 1
};

/*
 * Model parameters of one ensemble ("group"), real units.
 * Mirrors ModelParameters (programs/bec_wigner_3d.cuda/defines.h:25-54) with
 * three differences: the loss rates are SI (m^6/s for gamma111, m^3/s for
 * gamma12/gamma22; the reference takes cm units and divides by 1e12 / 1e6 in
 * wigner.cpp:141-143), nvy == 1 selects a 2D x-z slice, and the loss-noise
 * switch and RNG seed are explicit.
 */
typedef struct bec_params {
    double a11, a12, a22;          /* scattering lengths, Bohr radii */
    double m;                      /* particle mass, kg */
    double fx, fy, fz;             /* trap frequencies, Hz (fy only renormalises 2D) */
    double N;                      /* atom number */
    double detuning;               /* Hz */
    double gamma111;               /* three-body loss, m^6/s */
    double gamma12, gamma22;       /* two-body losses, m^3/s */
    double Va, Vb;                 /* vacuum-noise weights (0 = none, 1 = full) */
    int32_t nvx, nvy, nvz;         /* grid points; powers of two; nvy == 1 => 2D */
    int32_t itmax;                 /* midpoint iterations of the nonlinear step */
    double dt_steady;              /* imaginary-time step, s */
    double t_equilib;              /* equilibration time before the first pi/2, s */
    double dt_evo;                 /* real-time step, s */
    int32_t ne;                    /* trajectories in this ensemble */
    int32_t loss_noise;            /* 1: add the Wigner loss-noise terms */
    uint64_t seed;                 /* Philox key for this ensemble */
} bec_params;

/*
 * Derived parameters in natural units (l_rho = sqrt(hbar/(m w_x)), t_rho = 1/w_x).
 * Mirrors CalculationParameters (defines.h:57-112) as filled by
 * fillDerivedParameters (wigner.cpp:119-176), in FP64, including the
 * reference's dk = pi / xmax (wigner.cpp:167-169).
 */
typedef struct bec_derived {
    double N;
    double g11, g12, g22;          /* couplings (2D: divided by sqrt(2 pi) l_y) */
    double mu;                     /* Thomas-Fermi chemical potential */
    double Va, Vb, V;              /* V = (Va + Vb) / 2 */
    double lambda;                 /* fx / fz */
    double l_rho, t_rho;           /* natural length (m) and time (s) */
    double detuning;               /* natural units */
    double l111, l12, l22;         /* loss rates, natural units */
    double xmax, ymax, zmax;       /* box half-widths */
    double dx, dy, dz;             /* space steps (dy = 1 in 2D) */
    double dkx, dky, dkz;          /* k steps */
    double dV;                     /* cell volume dx*dy*dz (dx*dz in 2D) */
    double dt_steady, t_equilib, dt_evo;
    int32_t nvx, nvy, nvz;
    int32_t cells;
    int32_t itmax;
    int32_t ne;
    int32_t dims;                  /* 2 or 3 */
    int32_t n_equil_steps;         /* steps taken by the equilibration loop (wigner.cu:222) */
} bec_derived;

/* Ground-state stopping rules. */
enum {
    BEC_GS_FIXED_STEPS = 0,  /* exactly max_steps imaginary-time steps */
    BEC_GS_MU = 1,           /* stop when |d mu| / mu < tol between checks */
    BEC_GS_REFERENCE_E = 2,  /* the reference's |dE/E| < 1e-6 test on its energy integral (wigner.cu:148-156) */
    BEC_GS_MU_RESIDUAL = 3   /* MU's test and, at the same check, the fixed-point residual
                              *   || psi_n - psi_{n-c} || / (c dt mu || psi_n ||) < res_tol
                              * of the imaginary-time map (c = check_every, dt and mu in the
                              * scaled units of bec_derived): mu alone passes through an extremum
                              * on its way from Thomas-Fermi, where |d mu| is small long before
                              * the state has stopped changing */
};

typedef struct bec_gs_opts {
    int32_t mode;            /* BEC_GS_* */
    int32_t max_steps;       /* step cap (the exact count for FIXED_STEPS) */
    int32_t check_every;     /* steps between convergence checks (MU mode) */
    int32_t warm_per_group;  /* bec_ground_state_batch: 1 = warm_start holds one start per listed group, back to back */
    double tol;              /* relative tolerance for MU mode (REFERENCE_E uses 1e-6) */
    const double *warm_start;/* optional x-space start (interleaved complex, cells); NULL = Thomas-Fermi */
    double res_tol;          /* MU_RESIDUAL: bound on the fixed-point residual (<= 0: 10 tol) */
} bec_gs_opts;

typedef struct bec_gs_report {
    int32_t steps;           /* imaginary-time steps taken */
    int32_t converged;       /* 1 if the stopping rule was met before max_steps */
    double mu;               /* chemical potential (Parseval kinetic + potential + 2x interaction) / N */
    double energy;           /* energy per particle */
    double N;                /* norm after the last renormalisation */
    double residual;         /* || H psi - mu psi || / || psi || */
    double seconds;          /* device time of the loop */
    double step_residual;    /* MU / MU_RESIDUAL: the fixed-point residual at the last check (0 before two checks) */
} bec_gs_report;

/*
 * Per-sample FP64 moments of one ensemble, summed over its trajectories
 * (compensated summation on the device):
 *   na = sum |a|^2 dV,  nb = sum |b|^2 dV,  s = sum conj(a) b dV.
 * All of the reference's observables are closed-form functions of these:
 * see bec_observables().
 */
typedef struct bec_moments {
    double t;                /* physical time since the first pi/2 pulse, s */
    double na, nb;
    double s_re, s_im;
} bec_moments;

/* Observables derived from moments (no device work). */
typedef struct bec_obs {
    double t;
    double N1, N2;           /* per-trajectory populations, Wigner term V/(2 dV) subtracted (wigner_kernel.cu:283-286) */
    double Ntotal;           /* the reference's printed population after its second pi/2 (wigner.cu:363-369) */
    double visibility;       /* 2 |<psi1|psi2>| / (N1 + N2)  (report.tex:855-860) */
    double visibility_scan;  /* max over alpha = 0, 0.5, ... < 2 pi of |N1-N2|/(N1+N2) (wigner.cu:267-277) */
    double phase;            /* arg <psi1|psi2>, reference sign convention */
} bec_obs;

/* Run schedule for bec_run. Time zero is the state at call time. */
typedef struct bec_schedule {
    int32_t n_steps;         /* real-time steps to take */
    int32_t sample_every;    /* record moments after every k-th step (0: only after the last) */
    int32_t pi_pulse_step;   /* apply a pi pulse after this step count (-1: none) */
    int32_t axial;           /* 1: also record axial (z) projections per sample */
} bec_schedule;

typedef struct bec_ctx bec_ctx;

/* ---- parameters ------------------------------------------------------- */

/* fillDerivedParameters (wigner.cpp:119-176), FP64, SI loss rates. */
bec_status bec_derive_params(const bec_params *p, bec_derived *out);

/* ---- context ---------------------------------------------------------- */

/* Creates a context holding n_groups ensembles on the current CUDA device.
 * If the environment sets BEC_DEVICE_BYTES_LIMIT (bytes), the context's own device buffers may
 * not exceed it: creation then fails with BEC_ERR_OUT_OF_MEMORY before the device is asked,
 * which exercises the out-of-memory paths without filling a GPU.
 * Replaces initConstants + initWaveVectors + EvolutionState::init
 * (wigner_kernel.cu:395-399, :25-55; defines.h:157-184). */
bec_status bec_create(const bec_params *groups, int32_t n_groups, int32_t path, bec_ctx **out);
void bec_destroy(bec_ctx *ctx);                         /* releaseWaveVectors + EvolutionState::release */
const char *bec_last_error(const bec_ctx *ctx);         /* message of the last failing call ("" if none) */
int32_t bec_abi_version(void);
bec_status bec_group_info(const bec_ctx *ctx, int32_t group, bec_derived *out);
int64_t bec_total_trajectories(const bec_ctx *ctx);

/* ---- ground state ----------------------------------------------------- */

/* calculateSteadyState (wigner.cu:84-175) for one group's parameters:
 * imaginary-time split-step from Thomas-Fermi (or a warm start), renormalised
 * to N after every step. psi_out receives the x-space ground state
 * (interleaved complex, cells). */
bec_status bec_ground_state(bec_ctx *ctx, int32_t group, const bec_gs_opts *opts,
                            double *psi_out, bec_gs_report *report);

/* Ground states for several groups at once (batched), one stopping rule. */
bec_status bec_ground_state_batch(bec_ctx *ctx, int32_t n, const int32_t *groups,
                                  const bec_gs_opts *opts, double *const *psi_out,
                                  bec_gs_report *reports);

/* Ground states of n groups that share one grid, run batched in FP32 on the device
 * (FIXED_STEPS, MU or MU_RESIDUAL rules, batched path only), exchanging only coefficients
 * of the 64-term correction over Thomas-Fermi with the host (bec_warmstart_basis_size):
 *   coef_in     (n x 64, may be NULL): warm starts psi = A max(f_TF + sum c_k B_k, 0),
 *               synthesised on the device (NULL = Thomas-Fermi);
 *   coef_out    (n x 64, may be NULL): least-squares projection of each result;
 *   profile_out (n x cells floats, may be NULL): each result's scaled correction
 *               |psi| / A - f_TF on the grid (the data a basis is learned from);
 *   reports     (n, may be NULL): steps, convergence, mu, energy, residual (FP64 on the device);
 *               seconds covers the warm-start synthesis and the loop.
 * B_k is the basis installed for the grid by bec_warmstart_set_basis, else the analytic
 * one; the basis and scaling are documented in bec_b200/csrc/warmstart.cu. */
bec_status bec_ground_state_coeffs(bec_ctx *ctx, int32_t n, const int32_t *groups, const bec_gs_opts *opts,
                                   const double *coef_in, double *coef_out, float *profile_out,
                                   bec_gs_report *reports);
int32_t bec_warmstart_basis_size(void);

/* Installs nb (1..64) basis rows of nvx*nvy*nvz floats (grid index order, scaled units as
 * profile_out) for that grid in this context; coefficients k >= nb are then zero. nb = 0 or
 * basis = NULL removes it (back to the analytic basis). BEC_ERR_INVALID_ARG when the rows are
 * linearly dependent. */
bec_status bec_warmstart_set_basis(bec_ctx *ctx, int32_t nvx, int32_t nvy, int32_t nvz, int32_t nb,
                                   const float *basis);

/* ---- evolution -------------------------------------------------------- */

/* initializeEnsembles (wigner_kernel.cu:295-317) for one group:
 *   a = psi_gs + Va * eta_a / sqrt(dV),  b = Vb * eta_b / sqrt(dV),
 * eta complex normal with <|eta|^2> = 1/2. noise == NULL draws eta from
 * Philox4x32-10 keyed by (seed, trajectory); otherwise noise holds
 * ne * 2 * cells interleaved complex values laid out [traj][a|b][cell]. Returns once psi_gs and
 * noise have been copied to the device (the caller may reuse them); the kernels run on. */
bec_status bec_init_group(bec_ctx *ctx, int32_t group, const double *psi_gs, const double *noise);

/* Host element types of bec_init_groups' ground states. BEC_HOST_R32 is real FP32 (imaginary part
 * zero): an imaginary-time ground state from Thomas-Fermi is real, every factor the loop applies
 * being real, so a quarter of the complex128 bytes carries it exactly to the FP32 path. */
enum { BEC_HOST_C128 = 0, BEC_HOST_C64 = 1, BEC_HOST_R32 = 2 };

/* bec_init_group (noise == NULL) for n distinct groups at once: the same initial states bit for
 * bit. psi_gs[i] is the x-space ground state of groups[i]. It holds cells values, interleaved
 * complex128 (BEC_HOST_C128) or complex64 (BEC_HOST_C64), or real FP32 (BEC_HOST_R32). The batched
 * FP32 path rounds a ground state to FP32 on the device either way, so complex64 halves the
 * host-to-device copy, and real FP32 halves it again for a real ground state, without changing
 * any result. The batched path copies the ground states (consecutive groups whose host
 * arrays lie back to back in memory in one transfer), then launches one
 * initialisation kernel and one preparation pass per run of consecutive trajectories of a grid
 * class, not one pair per group. The plain path initialises group by group. BEC_ERR_INVALID_ARG
 * for an index out of range, a repeated group, a NULL pointer or an unknown host_type. Returns once the
 * ground states have been copied to the device (the caller may reuse the arrays); the kernels run on.
 * Extends initEvolution (wigner.cu:202-218) and initializeEnsembles
 * (wigner_kernel.cu:295-317), which the reference calls once per ensemble. */
bec_status bec_init_groups(bec_ctx *ctx, int32_t n, const int32_t *groups, const void *const *psi_gs,
                           int32_t host_type);

/* Advances every trajectory by n real-time split steps (propagate, wigner.cu:178-199). */
bec_status bec_evolve(bec_ctx *ctx, int32_t n_steps);

/* Instantaneous Rabi rotation of every trajectory (report.tex rotation matrix):
 *   a' = cos(theta/2) a - i e^{-i phi} sin(theta/2) b
 *   b' = -i e^{i phi} sin(theta/2) a + cos(theta/2) b.
 * theta = pi/2, phi = 0 is applyHalfPiPulse (wigner_kernel.cu:320-329);
 * theta = pi, phi = 0 is applyPiPulse (:332-341). */
bec_status bec_pulse(bec_ctx *ctx, double theta, double phi);

/* A Rabi pulse of finite duration (the report's coupled equations, report.tex:305-330,
 * which the reference only approximates by instantaneous rotations): the state
 * evolves for round(duration / dt_evo) split steps with the coupling
 * (Omega / 2)(e^{-i phi} |1><2| + h.c.) on, Omega = 2 pi rabi_hz, the detuning
 * staying in the nonlinear step as in the reference. Each step is Strang-split
 * as R(Omega dt / 2) . step . R(Omega dt / 2) with R the rotation of bec_pulse.
 * Every group must share dt_evo. */
bec_status bec_pulse_finite(bec_ctx *ctx, double rabi_hz, double duration_s, double phi);

/* The reference's initEvolution (wigner.cu:202-227) after bec_init_group for every
 * group: the equilibration steps (t = 0; t <= t_equilib; t += dt_evo), then the
 * first pi/2 pulse. Resets the time origin to zero. */
bec_status bec_start_evolution(bec_ctx *ctx);

/* Moments of every group at the current time; out has n_groups entries. */
bec_status bec_moments_now(bec_ctx *ctx, bec_moments *out);

/* Axial profiles of one group at the current time: for each z,
 * out[4*z + 0..3] = (sum_xy |a|^2 dV, sum_xy |b|^2 dV, Re, Im of sum_xy conj(a) b dV),
 * summed over the group's trajectories. out has 4 * nvz doubles. */
bec_status bec_axial_now(bec_ctx *ctx, int32_t group, double *out);

/* Per-trajectory moments at the current time: n_traj entries, trajectories
 * ordered by group then index. */
bec_status bec_traj_moments_now(bec_ctx *ctx, bec_moments *out);

/* Headless version of the reference's state drawing (drawState, wigner.cu:413-430 with
 * the projections of :384-410 and the colour ramp of spectre.cu:34-46): densities of both
 * components after a pi/2 pulse about alpha = 0, Wigner term subtracted, summed over the
 * group's trajectories and projected on xy (sum over z) and zy (sum over x), then mapped to
 * RGBA floats with max levels 3 N ne nvz / (cells dV) (xy) and 3 N ne nvx / (cells dV) (zy).
 * xy_*: nvy x nvx pixels, zy_*: nvy x nvz pixels, 4 floats each; levels_* (may be NULL) get
 * the projected densities. Batched path only. */
bec_status bec_render_projections(bec_ctx *ctx, int32_t group, float *xy_a, float *xy_b, float *zy_a,
                                  float *zy_b, float *levels_xy, float *levels_zy);

/* Runs a schedule. samples receives n_samples * n_groups moments
 * (sample-major), n_samples = n_steps / sample_every (or 1). When
 * schedule->axial is set, axial receives n_samples * sum_g(4 * nvz_g) doubles
 * (sample-major, groups in order); otherwise it may be NULL. */
bec_status bec_run(bec_ctx *ctx, const bec_schedule *schedule, bec_moments *samples, double *axial);

/* Observables of one group from its moments (pure host arithmetic). */
bec_status bec_observables(const bec_ctx *ctx, int32_t group, const bec_moments *m, bec_obs *out);

/* Rotated populations after a final pi/2 pulse about axis angle alpha (halfPiRotate,
 * wigner_kernel.cu:344-360) for n_alpha angles: out[2*j], out[2*j+1] = N1(alpha_j), N2(alpha_j),
 * per trajectory, Wigner term subtracted. */
bec_status bec_phase_scan(const bec_ctx *ctx, int32_t group, const bec_moments *m,
                          int32_t n_alpha, const double *alpha, double *out);

/* ---- state I/O (checkpoint / parity) ---------------------------------- */

/* x-space state of one trajectory of one group: a then b, each cells
 * interleaved complex (2 * cells complex values). */
bec_status bec_get_state(bec_ctx *ctx, int32_t group, int32_t traj, double *ab_out);
bec_status bec_set_state(bec_ctx *ctx, int32_t group, int32_t traj, const double *ab_in);
/* Steps taken since initialisation: the step counter of the Philox loss-noise draws. */
int64_t bec_step_index(const bec_ctx *ctx);
/* Steps taken since bec_start_evolution (moments report t = this count times dt_evo). */
int64_t bec_evolution_steps(const bec_ctx *ctx);
/* Sets both counters, e.g. after bec_set_state in a fresh context resuming a saved run, so
 * that its loss noise continues the saved run's Philox stream (step <= 2^32 - 1). The
 * reference has no counterpart: its noise came from the host rand() seeded by the time
 * (wigner.cu:210). */
bec_status bec_set_step_index(bec_ctx *ctx, int64_t step, int64_t evo_steps);

/*
 * Checkpoints: the stored device representation of every trajectory, bit for bit, with the
 * step counters and any pending half kick or pulse of the batched path, so that a context
 * created with the same groups and path resumes the run bit-identically
 * (bec_checkpoint_load, then bec_evolve / bec_run). No counterpart in the reference, which
 * keeps its ground state in host memory and has its state dumps commented out
 * (wigner.cpp:335-362). bytes must be at least bec_checkpoint_bytes(ctx); the load checks
 * grids, trajectory counts, seeds and path against the context (BEC_ERR_INVALID_ARG).
 */
int64_t bec_checkpoint_bytes(const bec_ctx *ctx);
bec_status bec_checkpoint_save(bec_ctx *ctx, void *buf, int64_t bytes);
bec_status bec_checkpoint_load(bec_ctx *ctx, const void *buf, int64_t bytes);

/* Batched path: steady steps (no pulse or sample due) replay CUDA graphs captured once per context
 * (8 steps and 1 step; set BEC_CUDA_GRAPHS=0 in the environment before bec_create to launch them one by
 * one instead). Returns the number of step graphs captured and in use (0 or 2). */
int32_t bec_step_graphs(const bec_ctx *ctx);

/* Batched path: the schedule of a split step, written to out as a JSON object (len bytes at most,
 * NUL included). Every grid class can run a step as two launches (its pencil and plane passes);
 * the classes whose planes are 8x8, 16x16 or 32x32 and whose nvz is 64, 128 or 256 can instead
 * run it together as ONE launch of a persistent kernel walking a work list of pencil-pass and
 * plane-pass items (a trajectory's plane items wait on its pencil items). Before the context's
 * first step an autotuner times the candidates on a copy of the state -- per-pass launches with
 * the plane passes at 16 or at 20 warps per SM, each with the register pencil kernel or with every
 * class's pencil pass on the faster of the register kernel and a persistent TMA kernel (timed per
 * class: "pencil_kernels" in the JSON), and the work list run in two phases or interleaving each
 * trajectory's plane items 0.5 to 4 waves of the grid after its pencil items -- and keeps the
 * fastest for this class mix and device (cached per process). BEC_STEP_PLAN in the environment
 * forces one (unfused, unfused-20, unfused-tma and unfused-20-tma with every class on the TMA
 * pencil kernel, unfused-onchip with every 8x8x64 class's steady steps as one launch holding each
 * trajectory in shared memory, or 0..4 for the work lists), BEC_AUTOTUNE=0 takes the per-pass launches
 * untimed; every schedule computes the same bits. The reference has one fixed schedule of eight
 * launches per ensemble and step (wigner.cu:178-199) with cuFFT plans built by batchfftPlan3d
 * (batchfft.cu:22-100). */
bec_status bec_step_plan(bec_ctx *ctx, char *out, int32_t len);

/* Runs n_steps steady real-time steps (they advance the run like bec_evolve) with CUDA events on
 * the engine's stream around each launch of the fused step kernel (both launches of a two-phase
 * plan) and reports the mean device time of one step's fused launch and the cells it covers
 * (trajectories x cells over the fused classes). BEC_ERR_STATE when no class is fused. */
bec_status bec_profile_fused_step(bec_ctx *ctx, int32_t n_steps, double *ms_per_step, int64_t *cells);

/* ---- timing ----------------------------------------------------------- */

/* Device time of the last bec_evolve / bec_run call, milliseconds (CUDA events). */
double bec_last_device_ms(const bec_ctx *ctx);
/* Number of this library's kernel launches issued by the last bec_evolve / bec_run. */
int64_t bec_last_launch_count(const bec_ctx *ctx);

/* Runs n_steps real-time steps with CUDA events on the engine's stream around
 * every launch and reports, per grid class c (batched path; on the plain path
 * every group is a class): dims[3c..3c+2] = (nvx, nvy, nvz), traj[c] = its
 * trajectory count, ms[2c] / ms[2c+1] = mean device time of one z-pass /
 * plane-pass launch (plain path: ms[2c] = one trajectory-step, ms[2c+1] = 0).
 * At most max_classes classes are written; *n_classes receives the count.
 * No counterpart in the reference, which times with gettimeofday around whole
 * steps (wigner.cpp:365-369). */
bec_status bec_profile_steps(bec_ctx *ctx, int32_t n_steps, int32_t max_classes, int32_t *dims,
                             int64_t *traj, double *ms, int32_t *n_classes);

/* ---- warm-start network ------------------------------------------------ */

/*
 * A multilayer perceptron Y = act(X W^T + b) per layer (tanh on hidden layers,
 * identity on the last), trained and evaluated on the GPU with tensor-core
 * GEMMs on split BF16 operands (x = hi + lo, about 16 significant bits)
 * accumulating in FP32. No counterpart in the reference: it
 * predicts the coefficients of a correction to the Thomas-Fermi profile that
 * seeds bec_ground_state_batch (warm_start), which alone decides convergence.
 * widths has n_layers + 1 entries (inputs, hidden..., outputs). Host parameter
 * layout: for each layer W [out x in] row-major, then b [out].
 */
typedef struct bec_mlp bec_mlp;
bec_status bec_mlp_create(const int32_t *widths, int32_t n_layers, uint64_t seed, bec_mlp **out);
void bec_mlp_destroy(bec_mlp *m);
int64_t bec_mlp_param_count(const bec_mlp *m);
bec_status bec_mlp_get_params(bec_mlp *m, float *params);
bec_status bec_mlp_set_params(bec_mlp *m, const float *params);
/* x: batch x inputs, y: batch x outputs (host, FP32) */
bec_status bec_mlp_forward(bec_mlp *m, const float *x, int32_t batch, float *y);
/* loss = mean over the batch and outputs of (y - target)^2 and its gradient (host layout) */
bec_status bec_mlp_gradients(bec_mlp *m, const float *x, const float *target, int32_t batch, float *loss,
                             float *grads);
/* Learning-rate schedules of bec_mlp_train */
enum {
    BEC_LR_CONSTANT = 0,     /* lr at every step */
    BEC_LR_COSINE = 1        /* lr (1 + cos(pi step / steps)) / 2 */
};
/* Adam (beta 0.9, 0.999) on seeded minibatches of n samples; loss_history[step] (may be NULL) */
bec_status bec_mlp_train(bec_mlp *m, const float *x, const float *target, int32_t n, int32_t batch, int32_t steps,
                         float lr, int32_t schedule, uint64_t seed, float *loss_history);

/* ---- moments without device allocation -------------------------------- */

/* Largest ne * cells accepted by bec_moments_device_noalloc. */
#define BEC_NOALLOC_MAX_ELEMENTS 1073741824

/*
 * FP64 moments (na, nb, Re s, Im s), as in bec_moments, of ne x-space
 * trajectories that already live in the caller's device memory:
 *   d_psi: ne * 2 * cells interleaved complex doubles laid out [traj][a|b][cell];
 *   d_out: 4 doubles of device memory receiving sum |a|^2 dV, sum |b|^2 dV and
 *          the real and imaginary parts of sum conj(a) b dV over all trajectories;
 *   stream: a cudaStream_t of the current device, or NULL for the default
 *          stream. The call only enqueues work: synchronise the stream before
 *          reading d_out.
 * No counterpart in the reference. It exists for callers that cannot let a
 * library call cudaMalloc: hosts whose device memory all comes from their own
 * pool, and loops that must never block on an allocation (cudaMalloc and
 * cudaFree synchronise the device and can fail mid-run). It allocates nothing:
 * the reduction's partial sums live in a fixed 64 KiB array that is part of the
 * library image (every GPU that loads the library holds it until the process
 * exits). Every call looks up that array's device address in the current
 * context (no allocation); the first call on a device also loads the library's
 * device code there, so make one call on each device before capturing any
 * stream. All calls share
 * the array: calls that overlap on the GPU (different streams, or several host
 * threads) race and must be serialised by the caller; each call rewrites every
 * partial sum it reads, so nothing carries over from the previous call.
 * Returns BEC_ERR_INVALID_ARG for null pointers, non-positive sizes or dV, and
 * for ne * cells above BEC_NOALLOC_MAX_ELEMENTS.
 */
bec_status bec_moments_device_noalloc(const double *d_psi, int32_t cells, int32_t ne, double dV,
                                      double *d_out, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* BEC_H */
