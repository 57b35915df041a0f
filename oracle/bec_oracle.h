/*
 * bec_oracle.h -- CPU FP64 oracle for the split-step GPE / truncated-Wigner path.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker: the parity tests,
 * the smoke check and the CPU-baseline leg of the benchmark call it; the
 * product library never links or loads it.
 *
 * It restates, in plain C99 and double precision, the algorithm of
 * programs/bec_wigner_3d.cuda (wigner.cpp, wigner.cu, wigner_kernel.cu) with
 * its own radix-2 FFT in place of cuFFT, following the reference line by line
 * (citations in bec_oracle.c). Terms the reference does not implement
 * (Wigner loss noise, the 2D transverse renormalisation, the mu stopping
 * rule) are defined here and in the product the same way.
 */
#ifndef BEC_ORACLE_H
#define BEC_ORACLE_H

#include "../include/bec.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_ens oracle_ens;

/* parameters */
int oracle_derive(const bec_params *p, bec_derived *out);

/* primitives exposed for known-answer tests */
void oracle_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
void oracle_normals4(uint64_t seed, uint32_t traj, uint32_t step, uint32_t cell, uint32_t tag, double out[4]);
/* the six loss-noise normals of (seed, traj, step, cell): one Philox draw cut into 21-bit fields */
void oracle_loss_normals6(uint64_t seed, uint32_t traj, uint32_t step, uint32_t cell, double out[6]);
int oracle_fft3d(double *data, int nx, int ny, int nz, int sign);   /* unnormalised, sign -1 forward, +1 inverse */
void oracle_k2_table(const bec_derived *d, double *k2half);          /* (kx^2+ky^2+kz^2)/2 per cell */
void oracle_potential_table(const bec_derived *d, double *v);        /* V per cell */

/* ground state (calculateSteadyState) */
int oracle_ground_state(const bec_params *p, const bec_gs_opts *opts, double *psi_out, bec_gs_report *rep);
/* mu, energy per particle and residual of an x-space single-component state */
int oracle_gs_measures(const bec_params *p, const double *psi, double *mu, double *energy, double *residual, double *N);

/* ensembles */
oracle_ens *oracle_create(const bec_params *p);
void oracle_free(oracle_ens *e);
int oracle_init(oracle_ens *e, const double *psi_gs, const double *noise);
int oracle_evolve(oracle_ens *e, int n_steps, int threads);
int oracle_pulse(oracle_ens *e, double theta, double phi);
int oracle_round_fp32(oracle_ens *e);
int oracle_start_evolution(oracle_ens *e, int threads);
int oracle_moments(oracle_ens *e, bec_moments *out);
int oracle_traj_moments(oracle_ens *e, bec_moments *out);
int oracle_axial(oracle_ens *e, double *out);
int oracle_get_state(oracle_ens *e, int traj, double *ab);
int oracle_set_state(oracle_ens *e, int traj, const double *ab);
long long oracle_step_index(const oracle_ens *e);
double oracle_time(const oracle_ens *e);

/* literal restatements of the reference's measurement kernels */
int oracle_ref_rotated_sums(oracle_ens *e, double alpha, double *na, double *nb);
int oracle_ref_visibility(oracle_ens *e, double *vis);
int oracle_ref_axial_ratio(oracle_ens *e, double *out);

#ifdef __cplusplus
}
#endif

#endif
