/*
 * bpx.h -- C-ABI of the B200 bedpostx per-voxel path (libbpx.so).
 *
 * The library replaces the GPU half of FSL FDT's xfibres_gpu:
 *   - the host entry  void xfibres_gpu(Matrix datam, Matrix bvecs, Matrix bvals,
 *       Matrix gradm, int idpart, int idSubpart, float seed, string subjdir)
 *     (CUDA/xfibres_gpu.h:15-23, implemented in CUDA/xfibres_gpu.cu:29-146),
 *   - the kernel-level entries of libbedpostx_cuda.so
 *     (CUDA/fit_gpu_kernels.h:9-102, CUDA/runmcmc_kernels.cu:26,193,507),
 *   - the host sample finishing (CUDA/xfibres_gpu.cu:659-738, CUDA/samples.cu:134-347).
 *
 * Plain pointers and sizes only.  Every function returns a bpx_status; nothing calls exit().
 * Functions named *_dev take DEVICE pointers and a cudaStream_t passed as void*; they are
 * asynchronous with respect to the host unless stated.  bpx_xfibres_host takes HOST pointers
 * and is synchronous.  Options are passed explicitly (the reference reads a process-wide
 * xfibresOptions singleton).  Concurrency: the stage entries that take all their buffers from
 * the caller (bpx_mcmc_*, bpx_finish_dev, bpx_postproc_dev, bpx_prepare_data_dev,
 * bpx_gemm_bf16_dev) may run concurrently on different streams.  The entries that use workspace
 * memory (bpx_fit_dev, bpx_xfibres_dev/_host, bpx_xfibres_learned_*, bpx_mlp_forward_dev,
 * bpx_mlp_train_step_dev) take it from the handle bound to the calling host thread
 * (bpx_handle_bind), or, with none bound, from a per-device workspace shared by every unbound
 * caller on the device: unbound calls must be issued on one stream, or each made to wait for the
 * previous such call's work.  Calls bound to different handles may run concurrently, from
 * different threads and on different streams.  A bpx_batch owns its buffers; different batches may
 * run concurrently.
 *
 * Array layouts (row-major, C order):
 *   data      [nvox][ndir]                 (voxel-major; CUDA/xfibres_gpu.cu:390-399)
 *   bvecs     [3][ndir], bvals [ndir]      (or [nvox][3][ndir], [nvox][ndir] with gradnonlin;
 *                                           CUDA/xfibres_gpu.cu:411-446)
 *   params    [nvox][bpx_nparams_fit()]    LM output, layout
 *             [S0, d, (d_std,) (f,th,ph)*nfib, (f0)]   (CUDA/PVM_multi.cu:549-566)
 *   records   [BPX_NREC(nfib)][nsamples][nvox]   one row per recorded parameter, in the
 *             order d, f0, tau, d_std, R, S0, then th_k, ph_k, f_k for k = 0..nfib-1
 *             (the records of CUDA/runmcmc_kernels.cu:1326-1339, transposed so that every
 *             row has the [nsamples][nvox] layout of the part files)
 *   samples   th/ph/f [nfib][nsamples][nvox]: the th{k}samples/ph{k}samples/f{k}samples
 *             part files of Samples::save (CUDA/samples.cu:262-347), fibres sorted by
 *             decreasing sum of f over samples.
 */
#ifndef BPX_H
#define BPX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BPX_ABI_VERSION 1
#define BPX_MAX_FIBRES 3
/* number of recorded parameters: d, f0, tau, d_std, R, S0 + (th, ph, f) per fibre */
#define BPX_NREC(nfib) (6 + 3 * (nfib))

typedef enum bpx_status {
  BPX_OK = 0,
  BPX_ERR_INVALID_ARG = 1, /* a size, pointer or option is out of range */
  BPX_ERR_CUDA = 2,        /* a CUDA runtime call failed; see bpx_last_error() */
  BPX_ERR_NO_DEVICE = 3,   /* no CUDA device, or the device is not sm_100 */
  BPX_ERR_UNSUPPORTED = 4, /* option combination not built (e.g. ndir too large) */
  BPX_ERR_IO = 5,          /* part-file read/write failed */
  BPX_ERR_BAD_DATA = 6     /* non-finite input data */
} bpx_status;

/* Per-voxel status bits written by the pipeline (bpx_outputs.status). */
#define BPX_VOX_NONFINITE_DATA 1u  /* data held NaN/Inf: voxel skipped, outputs zero */
#define BPX_VOX_F0_REFIT 2u        /* the f0 plausibility rule re-fitted this voxel without f0 */
#define BPX_VOX_NONFINITE_ENERGY 4u /* the chain met a non-finite energy */
#define BPX_VOX_LM_ITERATION_CAP 8u /* the LM fit that gave the start stopped at its 200-iteration cap,
                                       not at the cost tolerance */

/*
 * The xfibresOptions fields that act on the per-voxel path (xfibresoptions.h:104-149).
 * Booleans are 0/1.  bpx_options_default() gives the xfibres defaults.
 */
typedef struct bpx_options {
  int32_t model;               /* --model 1|2|3                       (default 1) */
  int32_t nfibres;             /* --nf 1..3                           (default 1) */
  float fudge;                 /* --fudge ARD weight                  (default 1) */
  int32_t njumps;              /* --nj                                (default 1250) */
  int32_t nburn;               /* --bi                                (default 1000) */
  int32_t sampleevery;         /* --se                                (default 25) */
  int32_t updateproposalevery; /* --upe                               (default 40) */
  int32_t no_ard;              /* --noard */
  int32_t all_ard;             /* --allard */
  int32_t nonlin;              /* --nonlinear: model 1 fitted with PVM_single */
  int32_t cnonlin;             /* --cnonlinear: model 1 fitted with PVM_single_c (the GPU default) */
  int32_t rician;              /* --rician */
  int32_t f0;                  /* --f0 */
  int32_t ardf0;               /* --ardf0 */
  float R_prior_mean;          /* --Rmean                             (default 0.13) */
  float R_prior_std;           /* --Rstd                              (default 0.03) */
  float R_prior_fudge;         /* --Rfudge                            (default 0) */
  int32_t gradnonlin;          /* --gradnonlin given: per-voxel b-matrix */
  uint64_t seed;               /* --seed                              (default 8665904) */
  int32_t mcmc_tpv;            /* MCMC launch layout: lanes per voxel (0 = automatic) */
  int32_t mcmc_mpl;            /* MCMC launch layout: measurements per lane (0 = automatic) */
  int32_t reserved[6];         /* zero */
} bpx_options;

/* One volume (a part or subpart of xfibres_gpu). */
typedef struct bpx_volume {
  int32_t nvox;          /* voxels (may be 0) */
  int32_t ndir;          /* measurements per voxel, 1..BPX max (bpx_max_ndir()) */
  const float* data;     /* [nvox][ndir] */
  const float* bvecs;    /* [3][ndir], unit vectors; [nvox][3][ndir] with gradnonlin */
  const float* bvals;    /* [ndir]; [nvox][ndir] with gradnonlin */
  const float* grad;     /* host entry only: [nvox][9] gradient-nonlinearity tensors or NULL */
  uint64_t voxel_offset; /* global index of voxel 0: keys the counter-based RNG, so a voxel's
                            chain does not depend on how the volume is split */
} bpx_volume;

/* Outputs of the full pipeline.  Any pointer may be NULL to skip that output. */
typedef struct bpx_outputs {
  float* th;        /* [nfib][nsamples][nvox]  merged_th{k}samples */
  float* ph;        /* [nfib][nsamples][nvox]  merged_ph{k}samples */
  float* f;         /* [nfib][nsamples][nvox]  merged_f{k}samples  */
  float* mean_d;    /* [nvox] mean_dsamples */
  float* mean_dstd; /* [nvox] mean_d_stdsamples (model >= 2) */
  float* mean_R;    /* [nvox] mean_Rsamples (model 3) */
  float* mean_f0;   /* [nvox] mean_f0samples (--f0) */
  float* mean_tau;  /* [nvox] mean_tausamples (--rician) */
  float* mean_S0;   /* [nvox] mean_S0samples */
  float* mean_f;    /* [nfib][nvox] mean_f{k}samples */
  float* dyads;     /* [nfib][3][nvox] principal eigenvector of the mean dyadic tensor */
  uint32_t* status; /* [nvox] BPX_VOX_* bits */
} bpx_outputs;

/* ---- library facts ---- */
int32_t bpx_abi_version(void);
void bpx_options_default(bpx_options* opts);
/* LM parameter count: 2+3*nf (+1 model>=2) (+1 f0)  (CUDA/xfibres_gpu.cu:190-193) */
int32_t bpx_nparams_fit(const bpx_options* opts);
int32_t bpx_nsamples(const bpx_options* opts); /* njumps / sampleevery */
int32_t bpx_max_ndir(void);
/* Message of the last failing call on this host thread ("" if none). */
const char* bpx_last_error(void);

/* ---- stage entry points (device pointers, asynchronous on `stream`) ---- */

/*
 * Initial fits, replacing fit() (CUDA/xfibres_gpu.cu:173-348) and calculate_tau
 * (CUDA/diffmodels.cu:259-347): DTI start values, LM fit of PVM_single / PVM_single_c /
 * PVM_multi, the f0 plausibility re-fit with mix_params, and tau = 1/var(residuals) when
 * opts->rician.  params: [nvox][bpx_nparams_fit]; tau: [nvox] (may be NULL unless rician);
 * status: [nvox] or NULL.  Under --rician the data must already have had non-positive
 * entries replaced (bpx_prepare_data_dev).
 */
bpx_status bpx_fit_dev(const bpx_options* opts, const bpx_volume* vol, float* params, float* tau,
                       uint32_t* status, void* stream);

/*
 * remove_NonPositive_entries for every voxel (CUDA/xfibres_gpu.cu:350-367): non-positive
 * samples of a voxel with a positive maximum are replaced by its smallest positive sample.
 * In place on data [nvox][ndir].
 */
bpx_status bpx_prepare_data_dev(int32_t nvox, int32_t ndir, float* data, void* stream);

/*
 * MCMC: init_Fibres_Multifibres_kernel + runmcmc_kernel burn-in and recording
 * (CUDA/runmcmc.cu:27-316).  records: [BPX_NREC(nfib)][nsamples][nvox].
 * tau may be NULL unless rician.  status may be NULL.
 */
bpx_status bpx_mcmc_dev(const bpx_options* opts, const bpx_volume* vol, const float* params,
                        const float* tau, float* records, uint32_t* status, void* stream);

/*
 * Sample finishing: Samples::record/finish_voxel/save (CUDA/samples.cu:134-347).
 * Sorts fibres by sum of f, writes th/ph/f sample arrays, means and dyads.
 */
bpx_status bpx_finish_dev(const bpx_options* opts, int32_t nvox, const float* records,
                          bpx_outputs* out, void* stream);

/*
 * Whole pipeline on device buffers: prepare (rician) -> fit -> mcmc -> finish, for one volume.
 * `data` is modified in place under --rician.  Workspace comes from a per-device cache
 * owned by the library (grown on demand, freed by bpx_release_workspace) and shared by every
 * workspace-using call on the device: see Concurrency above.
 */
bpx_status bpx_xfibres_dev(const bpx_options* opts, const bpx_volume* vol, bpx_outputs* out,
                           void* stream);

/*
 * Drop-in for xfibres_gpu() with HOST buffers: copies data/bvecs/bvals (and grad under
 * gradnonlin) to the current device, corrects the b-matrix per voxel when vol->grad is given
 * (correct_bvals_bvecs, CUDA/xfibres_gpu.cu:151-170), runs the pipeline and copies the
 * outputs back into host buffers.  Synchronous.  The volume goes through in sub-volumes of 65536
 * voxels (or BPX_HOST_CHUNK from the environment) on two alternating device buffer sets, the
 * copies of one overlapping the computation of the next (pinned host buffers let them run
 * asynchronously); the outputs equal those of one pass over the whole volume, bit for bit, and
 * the device memory held is that of two sub-volumes.
 */
bpx_status bpx_xfibres_host(const bpx_options* opts, const bpx_volume* vol, bpx_outputs* host_out);

/*
 * Energies of given chain states, for checking the FP32 likelihood against an FP64 evaluation
 * (compute_likelihood + compute_prior, CUDA/runmcmc_kernels.cu:140-191).
 * states: [nvox][BPX_NSTATE] = S0, d, d_std, R, tau, f0, (th, ph, f) * 3.
 * lik, prior: [nvox] outputs (either may be NULL).
 */
#define BPX_NSTATE 15
bpx_status bpx_energy_dev(const bpx_options* opts, const bpx_volume* vol, const float* states,
                          float* lik, float* prior, void* stream);

/*
 * Gradient-nonlinearity correction on the device (correct_bvals_bvecs, CUDA/xfibres_gpu.cu:151-170):
 * for every voxel and every b>0 measurement, g' = (I+L) g / |(I+L) g| and b' = |(I+L) g|^2 b, with
 * L the voxel's 3x3 coil tensor stored column-major in grad [nvox][9].
 * bvecs [3][ndir], bvals [ndir] in; bvecs_out [nvox][3][ndir], bvals_out [nvox][ndir] out.
 */
bpx_status bpx_gradnonlin_dev(int32_t nvox, int32_t ndir, const float* grad, const float* bvecs,
                              const float* bvals, float* bvecs_out, float* bvals_out, void* stream);

/* MCMC launch layouts compiled into the library: writes up to `max` (tpv, mpl) pairs and returns
 * how many exist. */
int32_t bpx_mcmc_layouts(int32_t* tpv, int32_t* mpl, int32_t max);

/*
 * Measures the current device's MUFU (ex2.approx) and FP32 FMA issue rates with two
 * throughput-bound microkernels (synchronous, ~20 ms).  Results in operations per second,
 * one operation = one lane-instruction.  These are the denominators of the MCMC roofline.
 */
bpx_status bpx_measure_pipes(double* mufu_ops_per_s, double* fma_ops_per_s);

/*
 * Allocation-free variant of bpx_xfibres_dev.  No counterpart in the reference: xfibres_gpu
 * allocates its working memory (thrust vectors) on every call.
 *
 * Some callers cannot call cudaMalloc once they are running: frameworks that reserve the device
 * memory up front for their own pool (a later cudaMalloc fails or fragments that pool), and
 * latency-sensitive services for which cudaMalloc's implicit device synchronisation would stall
 * every other stream.  This entry performs the whole pipeline (--rician data clean-up, fits, MCMC,
 * finishing) with its intermediates (fit parameters, tau, MCMC records, status) in a file-scope
 * __device__ array of BPX_NOALLOC_SCRATCH_BYTES (40 MiB), which every GPU that loads the library
 * keeps until the process exits.  It calls no cudaMalloc, cudaFree or allocating library routine.
 *
 * Size limit: the intermediates take 4*(P + 2 + (6+3*nfib)*nsamples) + 132 bytes per voxel (the
 * last 132 hold the fit stages' FP64 parameters), each block rounded up to 256 bytes
 * (P = bpx_nparams_fit); larger volumes are rejected with BPX_ERR_UNSUPPORTED and a message giving
 * the maximum voxel count for the options.  At the whole-brain options (model 2, 3 fibres, f0,
 * rician, 50 samples) that is 13,100 voxels, more than one 12,800-voxel subpart of xfibres_gpu.
 *
 * The first call on a device resolves the array's device address (cudaGetSymbolAddress, with that
 * device current); that is also when the CUDA runtime loads the array's module and takes its device
 * memory.  Make that first call at start-up -- a call with vol->nvox == 0 does it and nothing else --
 * before reserving a memory pool and before any stream capture.  The address is resolved again in a
 * new context (after cudaDeviceReset).  Arguments are checked before anything runs, as by
 * bpx_xfibres_dev; a rejected call leaves `data` untouched.  All calls share the one array
 * and it keeps the last call's contents; every element a call reads it has written first, so no
 * clearing is needed, but calls that overlap on the GPU (different streams, or threads) race on
 * the array and must be serialised by the caller.  Inputs and outputs are caller-owned device
 * buffers as for bpx_xfibres_dev; `data` is modified in place under --rician.
 */
#define BPX_NOALLOC_SCRATCH_BYTES (40u * 1024u * 1024u)
bpx_status bpx_xfibres_noalloc_dev(const bpx_options* opts, const bpx_volume* vol, bpx_outputs* out,
                                   void* stream);

/*
 * MCMC with per-voxel proposal widths (no counterpart in the reference).  As bpx_mcmc_dev, plus:
 *   props_in   [6+3*nfib][nvox] starting proposal widths in slot order f0, tau, d, d_std, R, S0,
 *              (th, ph, f) per fibre; NULL = initialise_props (CUDA/runmcmc_kernels.cu:430-460).
 *   props_out  [6+3*nfib][nvox] widths after the last iteration, or NULL.
 *   freeze_props  0: adapt every updateproposalevery iterations (the reference's behaviour);
 *              1: never adapt (the chain keeps the starting widths); 2: adapt during the burn-in
 *              only, then record with the widths frozen.  A random-walk chain with fixed widths
 *              has the same target distribution.
 */
bpx_status bpx_mcmc_ex_dev(const bpx_options* opts, const bpx_volume* vol, const float* params,
                           const float* tau, const float* props_in, float* props_out,
                           int32_t freeze_props, float* records, uint32_t* status, void* stream);

/*
 * A stretch of the chain, for checkpoint and resume (no counterpart in the reference, which
 * restarts a part from its first iteration): iterations [it_begin, it_end) of the chain of
 * opts->nburn + opts->njumps iterations.
 *   state_in   [6+3*nfib][nvox] chain state at it_begin in the record rows (d, f0, tau, d_std, R,
 *              S0, then th, ph, f per fibre); NULL = start from params/tau as bpx_mcmc_ex_dev
 *              (required when it_begin > 0; params and tau are then not read).
 *   props_in   widths as for bpx_mcmc_ex_dev; acc_in [6+3*nfib][nvox] acceptances since the last
 *              width update (NULL = zeros).
 *   records    [6+3*nfib][nsamples][nvox]: the samples recorded in the stretch are written at
 *              their positions in the whole chain; the others are left as they are.
 *   state_out, props_out, acc_out  the state, widths and acceptance counts at it_end (each may be
 *              NULL).
 * The RNG is keyed by the iteration and every signal, likelihood and prior is recomputed from
 * the state, so consecutive stretches, each passed the previous one's state_out, props_out and
 * acc_out, reproduce one call over the whole chain bit for bit.
 */
bpx_status bpx_mcmc_stretch_dev(const bpx_options* opts, const bpx_volume* vol, const float* params,
                                const float* tau, const float* state_in, const float* props_in,
                                const int32_t* acc_in, int32_t it_begin, int32_t it_end,
                                int32_t freeze_props, float* records, float* state_out,
                                float* props_out, int32_t* acc_out, uint32_t* status, void* stream);

/*
 * ---- Learned initialiser (no counterpart in the reference) ----
 * A network nin -> 256 x 4 (GELU) -> 32 maps a voxel's signals, divided by the mean of its
 * b <= 50 s/mm^2 measurements (S0_hat) and zero-padded to nin = 8*ceil(ndir/8), to the MCMC's
 * starting state and per-voxel proposal widths.  BF16 weights and activations, FP32 accumulation,
 * all contractions on the tcgen05 tensor cores.  Parameters: one FP32 vector, for layer l = 0..4
 * W_l [n_l][k_l] then b_l [n_l], k = {nin,256,256,256,256}, n = {256,256,256,256,32}.
 * Outputs: 0-2 f_k, 3-11 fibre unit vectors, 12 d*1e3, 13 d_std*1e3, 14 S0/S0_hat, 15 f0*10,
 * 16 ln(tau*S0_hat^2), 17+q ln(normalised proposal width of MCMC slot q).
 */
#define BPX_MLP_WIDTH 256
#define BPX_MLP_HIDDEN 4
#define BPX_MLP_NOUT 32
int32_t bpx_mlp_nin(int32_t ndir);
int64_t bpx_mlp_nparams(int32_t ndir);

/* x [nvox][nin] (bf16 bits) and s0hat [nvox]; per_voxel_bvals: bvals is [nvox][ndir]. */
bpx_status bpx_mlp_features_dev(const bpx_volume* vol, int32_t per_voxel_bvals, uint16_t* x,
                                float* s0hat, void* stream);
/* out [nvox][32] = network(x). */
bpx_status bpx_mlp_forward_dev(int32_t ndir, const float* params, int32_t nvox, const uint16_t* x,
                               float* out, void* stream);
/* One forward + backward pass over a batch: grads (same layout as params) and the mean loss
 * (device float) of targets/tweights [batch][32] (weighted squared error; the direction blocks use
 * the sign-invariant loss |u u^T - v v^T|^2 weighted by tweights[3+3k]). */
bpx_status bpx_mlp_train_step_dev(int32_t ndir, const float* params, float* grads, int32_t batch,
                                  const uint16_t* x, const float* targets, const float* tweights,
                                  float* loss, void* stream);
/* Adam update (bias-corrected; step counts from 1). */
bpx_status bpx_mlp_adam_dev(int64_t n, float* params, const float* grads, float* m, float* v,
                            float lr, float beta1, float beta2, float eps, int32_t step, void* stream);
/* Training targets and weights [nvox][32] from fitted states (fit layout), tau (may be NULL) and
 * adapted proposal widths [6+3K][nvox] (may be NULL: no width targets). */
bpx_status bpx_mlp_targets_dev(const bpx_options* opts, int32_t nvox, const float* params,
                               const float* tau, const float* props, const float* s0hat,
                               float* targets, float* tweights, void* stream);
/* Network outputs -> starting state params [nvox][P] (fit layout), tau [nvox], proposal widths
 * props [6+3K][nvox] (tau, props may be NULL); status [nvox] (may be NULL) is cleared. */
bpx_status bpx_mlp_decode_dev(const bpx_options* opts, int32_t nvox, const float* out,
                              const float* s0hat, float* params, float* tau, float* props,
                              uint32_t* status, void* stream);
/* Learned pipeline: features -> network -> decode -> MCMC started from the network's state with
 * the network's proposal widths (freeze_props as for bpx_mcmc_ex_dev), opts->nburn burn-in ->
 * finishing.  Same outputs as bpx_xfibres_dev. */
bpx_status bpx_xfibres_learned_dev(const bpx_options* opts, const bpx_volume* vol,
                                   const float* mlp_params, int32_t freeze_props, bpx_outputs* out,
                                   void* stream);
/* The learned pipeline on host buffers (as bpx_xfibres_host; mlp_params is a host array). */
bpx_status bpx_xfibres_learned_host(const bpx_options* opts, const bpx_volume* vol,
                                    const float* mlp_params, int32_t freeze_props,
                                    bpx_outputs* host_out);

/*
 * Voxels drawn from the forward model (training data of the learned initialiser; no counterpart
 * in the reference).  model 1 or 2, nfib 1..3; S0 = 1000, d ~ U(0.5e-3, 2e-3), d_std = U(0.1,0.5) d,
 * f1 ~ U(0.3, 0.7), f2 = U(0,1) min(0.3, 1-f1), f3 = U(0,1) min(0.15, 0.99-f1-f2), directions
 * uniform, Rician noise at SNR ~ U(snr_lo, snr_hi) on S0.  Philox keyed by seed, counted by
 * voxel_offset + voxel.  data [nvox][ndir]; truth [nvox][BPX_NSTATE] (tau = 1/sigma^2) or NULL.
 */
bpx_status bpx_synth_dev(int32_t model, int32_t nfib, int32_t nvox, int32_t ndir, uint64_t seed,
                         uint64_t voxel_offset, float snr_lo, float snr_hi, const float* bvecs,
                         const float* bvals, float* data, float* truth, void* stream);

/* C[M][N] (fp32, row-major, ldc) = A B^T on the tcgen05 tensor cores, bf16 operands: A is
 * [M][lda] (a_mn = 0) or [K][lda] (a_mn = 1), B is [N][ldb] (b_mn = 0) or [K][ldb] (b_mn = 1).
 * Leading dimensions and the contiguous extents must be multiples of 8. */
bpx_status bpx_gemm_bf16_dev(int32_t M, int32_t N, int32_t K, const uint16_t* A, int32_t lda,
                             int32_t a_mn, const uint16_t* B, int32_t ldb, int32_t b_mn, float* C,
                             int32_t ldc, void* stream);
/* Synchronously reads and clears the device error word of the tensor-core kernels (0 = none;
 * 1 or 2 = a bounded wait for a TMA copy or an MMA gave up). */
bpx_status bpx_mlp_poll_error(int32_t* code);

/*
 * ---- Batched form (no counterpart in the reference) ----
 * Many volumes ("items") with their own voxel counts, measurement counts, models and fibre counts
 * run as one CUDA-graph launch; an item may start its chains from the initialiser network
 * (mlp_params) instead of LM fits.  Items of equal (model, nfibres, ndir, bvecs, bvals, network,
 * burn-in, freeze mode) form a bucket
 * whose voxels are packed so one fit, one MCMC and one finishing launch serve them all; the chains
 * keep each item's RNG keys (vol.voxel_offset + voxel), so results equal per-item runs.  The other
 * options (rician, f0, burn-in, ...) come from `opts` and are shared by all items.
 * bpx_batch_create validates, picks each bucket's MCMC layout (opts->mcmc_tpv/mpl if set, else the
 * autotuner when autotune != 0, else the default), allocates the packed buffers and captures the
 * graph; the items' device buffers must stay valid for the batch's life.  bpx_batch_run launches
 * the graph on `stream` (asynchronous).  Items with vol.grad (gradnonlin) are not batched.
 */
typedef struct bpx_item {
  bpx_volume vol;       /* device buffers */
  int32_t model;        /* 1..3 */
  int32_t nfibres;      /* 1..3 */
  bpx_outputs out;      /* device buffers; NULL fields are not written */
  const float* mlp_params;  /* device: initialiser network for vol.ndir (learned start), or NULL (LM fits) */
  int32_t nburn;            /* burn-in of this item's chains; < 0: opts->nburn */
  int32_t freeze_props;     /* learned items: as bpx_mcmc_ex_dev */
} bpx_item;
typedef struct bpx_batch bpx_batch;
bpx_status bpx_batch_create(const bpx_options* opts, const bpx_item* items, int32_t nitems,
                            int32_t autotune, bpx_batch** batch);
bpx_status bpx_batch_run(bpx_batch* batch, void* stream);
/* Bucket descriptions, 7 ints each: model, nfibres, ndir, tpv, mpl, voxels, items.  Returns the
 * number of buckets (writes at most max). */
int32_t bpx_batch_buckets(const bpx_batch* batch, int32_t* desc, int32_t max);
bpx_status bpx_batch_destroy(bpx_batch* batch);

/*
 * Autotuner: times every compiled MCMC layout (threads per voxel tpv, measurements per lane mpl;
 * 128/tpv voxels per block) that covers ndir on `sample` forward-model voxels with a 65-iteration
 * chain and returns the fastest (cached per device and option set).  seconds_per_voxel, if not
 * NULL, receives one entry per compiled layout (bpx_mcmc_layouts order; -1 = not a candidate).
 * Synchronous.
 */
bpx_status bpx_autotune_layout(const bpx_options* opts, int32_t ndir, const float* bvecs,
                               const float* bvals, int32_t sample, int32_t* tpv, int32_t* mpl,
                               float* seconds_per_voxel, void* stream);

/*
 * bedpostx_postproc_gpu.sh arithmetic (CUDA/bedpostx_postproc_gpu.sh:20-49) from finished outputs
 * (out->th, ph, mean_f, dyads on the device, as bpx_finish_dev leaves them): per fibre the
 * sample means of th and ph (fslmaths -Tmean), the dispersion 1 - max|eigenvalue| of the mean
 * dyadic tensor (make_dyadic_vectors.cc), for fibres 2..K the dyads masked where mean_f >= thr
 * (maskdyads, thr 0.05 in bedpostx) and those scaled by mean_f{k}/mean_f1 (_modf{k}), and
 * mean_fsumsamples.  Rows of fibre 1 in dyads_thr/dyads_modf are not written.  NULL outputs are
 * skipped.
 */
typedef struct bpx_postproc {
  float* mean_th;     /* [nfib][nvox] mean_th{k}samples */
  float* mean_ph;     /* [nfib][nvox] mean_ph{k}samples */
  float* dispersion;  /* [nfib][nvox] dyads{k}_dispersion */
  float* dyads_thr;   /* [nfib][3][nvox] dyads{k}_thr0.05 (k >= 2) */
  float* dyads_modf;  /* [nfib][3][nvox] dyads{k}_thr0.05_modf{k} (k >= 2) */
  float* mean_fsum;   /* [nvox] mean_fsumsamples */
} bpx_postproc;
bpx_status bpx_postproc_dev(const bpx_options* opts, int32_t nvox, const bpx_outputs* out, float thr,
                            bpx_postproc* post, void* stream);

/*
 * ---- probtrackx on the samples (simple mode: seeds -> fdt_paths) ----
 * The consumer of merged_th/ph/f{k}samples (probtrackx.cc:25-96 -> ptx_simple.cc:16-70,
 * Seedmanager::run and Streamliner::streamline in streamlines.cc:209-416,1023-1127,
 * Tractvolsx::sample in tractvolsx.h:101-255, Particle in particle.h).  For every seed point,
 * nparticles particles each track one streamline in both directions from the seed: per step the
 * position is rounded probabilistically to a voxel, one of the voxel's nsamples posterior samples
 * is drawn, the fibre closest to the current direction among those with f > fibthresh is taken,
 * the step stops at the curvature threshold c_thr, and the particle moves steplength mm.  Every
 * voxel a kept streamline passes through is counted once per streamline (fdt_paths), and kept
 * streamlines are counted (waytotal).  Random numbers are Philox-4x32-10 keyed by the seed and
 * counted by (particle, half, step), so a run is reproducible (the reference uses rand()).
 */
typedef struct bpx_track_options {
  int32_t nparticles;  /* -P, --nsamples: particles per seed point   (default 5000) */
  int32_t nsteps;      /* -S, --nsteps: steps per streamline (both halves together; default 2000) */
  float steplength;    /* --steplength, mm                           (default 0.5) */
  float c_thr;         /* -c, --cthr: curvature threshold |cos|       (default 0.2) */
  float fibthresh;     /* --fibthresh: f below which a fibre is ignored (default 0.01) */
  float distthresh;    /* --distthresh: halves shorter than this (mm) are dropped (default 0) */
  int32_t randfib;     /* --randfib 0..3: how the first step's fibre is chosen (default 0) */
  int32_t fibst;       /* --fibst: first fibre (1-based) when randfib is 0 (default 1) */
  int32_t usef;        /* -f, --usef: a step is taken with probability f */
  int32_t sampvox;     /* --sampvox: seed positions jittered within the seed voxel */
  uint64_t seed;       /* random seed */
  int32_t pathdist;    /* --pd: the d-th distinct voxel of a kept streamline adds d (path length
                          correction), not 1 (Counter::update_pathdist, streamlines.cc:662-690) */
  int32_t loopcheck;   /* -l, --loopcheck: a half stops where it runs against the direction it
                          last had in the same cell of a 5x coarser grid (streamlines.cc:248-263) */
  int32_t modeuler;    /* --modeuler: modified Euler steps, along the mean of the sampled direction
                          and the one sampled a step ahead (streamlines.cc:352-361) */
  int32_t per_seed;    /* 1: paths holds one volume per seed point, [nseeds][nz][ny][nx] (simple
                          mode's fdt_paths_<x>_<y>_<z>, counts reset between seeds: ptx_simple.cc:
                          50-62); 0: one volume summed over the seeds (seedmask mode's fdt_paths,
                          ptx_seedmask.cc) */
  int32_t reserved[1]; /* zero */
} bpx_track_options;

/* The bedpostx outputs probtrackx reads, on the device.  Sample arrays [nfib][nsamples][nz][ny][nx]
 * (x fastest: the merged_{th,ph,f}{k}samples volumes one after the other); mask [nz][ny][nx]
 * (nodif_brain_mask, > 0 inside); voxel size dx, dy, dz in mm.  Optional masks on the same grid
 * (NULL: none), tested at the rounded position of every step inside the brain mask
 * (streamlines.cc:279-330): avoid (--avoid, the reference's rubbish mask, != 0 inside) rejects a
 * half that enters it; stop (--stop) ends a half where it enters it; waypoints (--waypoints) holds
 * bit w set inside waypoint mask w < nwaypoints (<= 32), and a streamline is kept only when its two
 * halves together passed every one (Seedmanager::run's reject flags 0/1/2, streamlines.cc:1078-1098). */
typedef struct bpx_track_volume {
  int32_t nx, ny, nz;
  float dx, dy, dz;
  int32_t nfib, nsamples;
  const float* th;
  const float* ph;
  const float* f;
  const float* mask;
  const float* avoid;
  const float* stop;
  const uint32_t* waypoints;
  int32_t nwaypoints;
  /* seeds to targets (--targetmasks with --os2t; Counter::update_seedcounts, streamlines.cc:700-748):
   * targets holds bit t set inside target mask t < ntargets (<= 32), and seeds_to_targets
   * [ntargets][nseeds] (OUTPUT, int32, added to) counts for every seed the kept streamlines whose
   * path (first kept half, then second) enters target t at a path length >= distthresh.  Not with
   * pathdist (the reference then adds path lengths). */
  int32_t ntargets;
  const uint32_t* targets;
  int32_t* seeds_to_targets;
  /* --omatrix2 (Counter::update_matrix2_row, streamlines.cc:772-808): a tract-space grid of
   * lr_nx x lr_ny x lr_nz voxels of lr_dx x lr_dy x lr_dz mm, to which a path position maps by its
   * mm coordinates (vox_to_vox with the identity: round(x * dx / lr_dx)); m2_lookup
   * [lr_nz][lr_ny][lr_nx] gives each tract-space voxel's column (-1 outside the --target2 mask);
   * matrix2 [nseeds][m2_ncols] (OUTPUT, int32, added to) counts for every seed the kept
   * streamlines through each column, once per streamline (with pathdist the d-th new column adds
   * d).  Column 0 is never counted, as in the reference, whose test is "column != 0". */
  int32_t m2_ncols;
  int32_t lr_nx, lr_ny, lr_nz;
  float lr_dx, lr_dy, lr_dz;
  const int32_t* m2_lookup;
  int32_t* matrix2;
  /* --omatrix1 (Counter::initialise_matrix1, update_matrix1, streamlines.cc:493-510, 751-770): m1_lookup
   * [nz][ny][nx] gives each seed-mask voxel its column (-1 elsewhere: m1_ncols columns, numbered in
   * z, y, x order as the seeds of seedmask mode are); matrix1 [nseeds][m1_ncols] (OUTPUT, int32,
   * added to) counts for every seed the kept streamlines through each seed-mask voxel, once per
   * streamline, adding what that voxel's fdt_paths count gets (with pathdist the d-th new voxel adds
   * d): the reference's per-seed path distribution read at the seed mask. */
  int32_t m1_ncols;
  const int32_t* m1_lookup;
  int32_t* matrix1;
  /* --prefdir (streamlines.cc:124-125, 286-291; Tractvolsx::sample, tractvolsx.h:209-225): a preferred
   * direction per voxel, [3][nz][ny][nx] (x, y, z components), or NULL.  After a streamline's first
   * sample, each step takes the fibre closest to the vector at its rounded position, or to the
   * current direction where that vector is zero (the rule without --prefdir). */
  const float* prefdir;
} bpx_track_volume;

void bpx_track_options_default(bpx_track_options* opts);
/*
 * Tracks opts->nparticles streamlines from each of nseeds seed points (seeds [nseeds][3], voxel
 * coordinates of the volume, x y z) and ADDS each kept streamline's distinct voxels to
 * paths [nz][ny][nx], or to its seed's volume of paths [nseeds][nz][ny][nx] with opts->per_seed
 * (int32 counts, fdt_paths: the reference's volume<int> m_prob, wrapping past 2^31 as it does), and
 * the kept streamlines to *waytotal (device int64); the caller zeroes both first.  Integer sums make the result independent of the order in which streamlines finish.
 * Uses workspace memory (see Concurrency): the samples repacked, 16 * (nfib + 1) bytes per voxel
 * and sample, and per particle in flight a visit table of 8 * 2^ceil(log2(2 * (nsteps + 2))) bytes
 * (twice that with matrix2) and with loopcheck a coarse-cell table of 24 bytes per entry; 1024
 * particles in flight per multiprocessor, fewer if the tables would pass 16 GB (5 GB on a B200 at
 * nsteps 2000 without options).
 */
bpx_status bpx_probtrack_dev(const bpx_track_options* opts, const bpx_track_volume* vol, int32_t nseeds,
                             const float* seeds, int32_t* paths, int64_t* waytotal, void* stream);

/* Free the per-device workspace cache of the current device. */
bpx_status bpx_release_workspace(void);

/*
 * Workspace handles (the re-entrant counterpart of the reference's process-wide state, which makes
 * xfibres_gpu() single-threaded: CUDA/xfibres_gpu.h:15-23 with the xfibresOptions singleton).
 * A handle owns private grow-only workspaces on the device current at bpx_handle_create.
 * bpx_handle_bind(h) makes every workspace-using call on this host thread use h's workspaces
 * (bind NULL to return to the shared per-device ones); a handle is bound to one thread at a time
 * and its calls follow the one-stream rule among themselves.  bpx_handle_destroy frees the
 * workspaces (cudaFree waits for the device's work) and unbinds it from the calling thread; a handle
 * bound on another thread must be unbound there (bpx_handle_bind(NULL)) before it is destroyed.
 */
typedef struct bpx_handle bpx_handle;
bpx_status bpx_handle_create(bpx_handle** h);
bpx_status bpx_handle_bind(bpx_handle* h);
bpx_status bpx_handle_destroy(bpx_handle* h);

#ifdef __cplusplus
}
#endif
#endif /* BPX_H */
