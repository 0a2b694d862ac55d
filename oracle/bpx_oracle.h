/*
 * bpx_oracle.h -- CPU oracle for the bedpostx per-voxel path.  TEST INFRASTRUCTURE ONLY.
 *
 * An FP64 restatement of what xfibres_gpu computes per voxel (LM initial fits, Rician tau,
 * MCMC burn-in and recording, sample finishing).  Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline arm of bench.py may load it, and only as the checker / the timed CPU baseline.
 * The product (libbpx.so) never calls it.
 *
 * Parity pinning: the reference ships no tests, fixtures or golden vectors and its CPU xfibres
 * needs FSL libraries that are absent.  Its CUDA kernels, however, build from their own sources
 * (oracle/Makefile, target ref -> oracle/_ref/librefgpu.so), and tests/test_gpu_refpin.py checks
 * this oracle against them on the same inputs: the LM models' cost, gradient and Hessian
 * (cf_/grad_/hess_PVM_*), the LM fits, the MCMC's initial likelihood and prior energies
 * (init_Fibres_Multifibres_kernel) and the posterior means of its chains (runmcmc_kernel).
 * Analytic known-answer checks (noiseless LM recovery, finite-difference Jacobians, the
 * Philox-4x32-10 published known-answer vectors, logI0 against its series) pin the rest.
 *
 * Random numbers: the oracle and the GPU share one counter-based generator, Philox-4x32-10
 * (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC11), keyed by
 * the 64-bit seed and countered by (iteration, proposal slot, voxel id), so both draw the same
 * numbers for the same proposal and short chains can be compared step by step.
 */
#ifndef BPX_ORACLE_H
#define BPX_ORACLE_H

#include <stdint.h>

#include "../include/bpx.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Proposal slots of one MCMC iteration (fixed, whatever the options). */
#define ORC_SLOT_F0 0
#define ORC_SLOT_TAU 1
#define ORC_SLOT_D 2
#define ORC_SLOT_DSTD 3
#define ORC_SLOT_R 4
#define ORC_SLOT_S0 5
#define ORC_SLOT_TH(k) (6 + 3 * (k))
#define ORC_SLOT_PH(k) (7 + 3 * (k))
#define ORC_SLOT_F(k) (8 + 3 * (k))

void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
/* normal draw and log of the acceptance uniform of one proposal slot */
void orc_rng_slot(uint64_t seed, uint64_t vox, uint32_t iter, uint32_t slot, double* normal,
                  double* log_u);
double orc_logI0(double x);

/* DTI::linfit + calc_tensor_parameters (diffmodels.cc:17-46,239-266).
 * out[16] = s0, md, fa, l1, l2, l3, v1[3], v2[3], v3[3], sse. */
int orc_dti(int ndir, const float* y, const float* bvecs, const float* bvals, double* out);

/* remove_NonPositive_entries on every voxel, in place (CUDA/xfibres_gpu.cu:350-367). */
void orc_prepare_data(int nvox, int ndir, float* data);

/* fit() + calculate_tau.  params [nvox][nparams_fit], tau [nvox] (may be NULL unless rician),
 * status [nvox] (may be NULL).  With opts->gradnonlin, bvecs/bvals are per voxel. */
int orc_fit(const bpx_options* opts, int nvox, int ndir, const float* data, const float* bvecs,
            const float* bvals, double* params, double* tau, uint32_t* status, int nthreads);

/* Start parameters of one LM model (before the fit): kind 0 PVM_single, 1 PVM_single_c. */
int orc_lm_start(int kind, int nfib, int f0, int ndir, const float* y, const float* bvecs,
                 const float* bvals, double* p);
/* orc_lm_start for every voxel of data [nvox][ndir]; p [nvox][np] */
int orc_lm_starts(int kind, int nfib, int f0, int nvox, int ndir, const float* data, const float* bvecs,
                  const float* bvals, double* p, int nthreads);
/* One LM model fit from given start parameters, returning finalised parameters.
 * kind 0 single, 1 single_c, 2 multi (start = finalised PVM_single params), with
 * gamma_ball_only 0 (model 2) or 2 (model 3).  Returns the number of LM iterations. */
int orc_lm_fit(int kind, int nfib, int f0, int gamma_ball_only, double R, int ndir,
               const float* y, const float* bvecs, const float* bvals, const double* start,
               double* final_params);
/* cost, gradient and Gauss-Newton Hessian of one model at raw (unfinalised) parameters */
double orc_lm_eval(int kind, int nfib, int f0, int gamma_ball_only, double R, int ndir,
                   const float* y, const float* bvecs, const float* bvals, const double* p,
                   double* grad, double* hess);

/* MCMC burn-in + recording.  records [BPX_NREC(nfib)][nsamples][nvox]. */
int orc_mcmc(const bpx_options* opts, int nvox, int ndir, const float* data, const float* bvecs,
             const float* bvals, const double* params, const double* tau, uint64_t voxel_offset,
             double* records, int nthreads);

/* Sample finishing.  th/ph/f [nfib][nsamples][nvox]; means [nvox]; mean_f [nfib][nvox];
 * dyads [nfib][3][nvox].  Any output may be NULL. */
int orc_finish(const bpx_options* opts, int nvox, const double* records, double* th, double* ph,
               double* f, double* mean_d, double* mean_dstd, double* mean_R, double* mean_f0,
               double* mean_tau, double* mean_S0, double* mean_f, double* dyads);

/* Likelihood and prior energies of given states [nvox][BPX_NSTATE]. */
int orc_energy(const bpx_options* opts, int nvox, int ndir, const float* data, const float* bvecs,
               const float* bvals, const double* states, double* lik, double* prior);

/* probtrackx simple mode on bedpostx samples (track_oracle.c): adds each kept streamline's
 * distinct voxels to paths [nz][ny][nx] and the kept streamlines to *waytotal. */
int orc_probtrack(const bpx_track_options* o, const bpx_track_volume* v, int nseeds, const float* seeds,
                  int32_t* paths, int64_t* waytotal);
/* the uniforms of one tracking step, and the single-precision sine/cosine both paths use */
void orc_track_uniforms(uint64_t seed, uint64_t pid, int half, uint32_t step, float u[8]);
void orc_track_uniforms_euler(uint64_t seed, uint64_t pid, int half, uint32_t step, float u[8]);
void orc_sincos_fast(float x, float* sn, float* cs);

#ifdef __cplusplus
}
#endif
#endif
