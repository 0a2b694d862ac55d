// refgpu_harness.cu -- TEST INFRASTRUCTURE ONLY: the reference's own CUDA kernels, run on inputs
// the tests choose, so the oracle can be checked against the reference's arithmetic.
//
// The reference's device code is compiled from its own source files where they lie in the
// reference tree (CUDA/PVM_single.cu, CUDA/PVM_single_c.cu, CUDA/PVM_multi.cu and
// CUDA/runmcmc_kernels.cu, #included at build time by oracle/Makefile, never copied into this
// repository).  The only additions are the declarations that the reference's host-side header
// CUDA/diffmodels.cuh needs from FSL's newmat (ColumnVector, Matrix) and the two_pi constant of
// FSL's diffmodels.h, which its device code does not use beyond f2x_gpu/x2f_gpu.
//
// The host entry points below launch the reference kernels the way the reference's host code does
// (grid, block and dynamic shared memory as in CUDA/diffmodels.cu:98-242 and CUDA/runmcmc.cu:57-316)
// and one small harness kernel that calls the reference's cost/gradient/Hessian device functions
// (cf_PVM_*, grad_PVM_*, hess_PVM_*) on given parameters.  Only tests/ load the resulting library
// (oracle/_ref/librefgpu.so); the product (libbpx.so) never links or loads it.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <thrust/device_vector.h>
#include <thrust/host_vector.h>

using std::string;
using std::vector;
struct ColumnVector {};  // newmat types named by the host declarations in CUDA/diffmodels.cuh
struct Matrix {};
#define two_pi 0.636619772  // FSL diffmodels.h

#include "PVM_single.cu"
#include "PVM_single_c.cu"
#include "PVM_multi.cu"
#include "runmcmc_kernels.cu"

namespace {

#define RG_CUDA(call)                                                                    \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess) {                                                             \
      std::snprintf(g_err, sizeof(g_err), "%s: %s", #call, cudaGetErrorString(e_));     \
      return 1;                                                                          \
    }                                                                                    \
  } while (0)

char g_err[512] = "";
float g_ms[3] = {0.f, 0.f, 0.f};  // device time of the last call's kernels: fit; MCMC init + burn-in; recording

// device buffer that frees itself
template <typename T>
struct Buf {
  T* p = nullptr;
  size_t n = 0;
  ~Buf() {
    if (p) cudaFree(p);
  }
  cudaError_t alloc(size_t count) {
    n = count;
    return cudaMalloc(&p, (count ? count : 1) * sizeof(T));
  }
  cudaError_t put(const T* h, size_t count) {
    cudaError_t e = alloc(count);
    if (e != cudaSuccess) return e;
    return count ? cudaMemcpy(p, h, count * sizeof(T), cudaMemcpyHostToDevice) : cudaSuccess;
  }
  cudaError_t get(T* h, size_t count) const {
    return count ? cudaMemcpy(h, p, count * sizeof(T), cudaMemcpyDeviceToHost) : cudaSuccess;
  }
};

// Cost, gradient and Hessian of one LM model at the raw parameters of each voxel (one block of
// THREADS_BLOCK_FIT threads per voxel, as the reference's fit kernels run them).  kind 0:
// PVM_single, 1: PVM_single_c, 2: PVM_multi (gbo = Gamma_for_ball_only).  Shared memory holds the
// scratch the reference's device functions expect.
__global__ void lm_eval_kernel(int kind, const float* data, const float* bvecs, const float* bvals, float R,
                               float invR, int ndirections, int nfib, int nparams, bool f0, int gbo,
                               const float* params, double* cf_out, float* grad_out, float* hess_out) {
  extern __shared__ double sh[];
  double* cfv = sh;                                       // 1
  float* J = (float*)&cfv[1];                             // THREADS_BLOCK_FIT * nparams
  float* reduction = J + THREADS_BLOCK_FIT * nparams;     // THREADS_BLOCK_FIT
  float* myparams = reduction + THREADS_BLOCK_FIT;        // nparams
  float* grad = myparams + nparams;                       // nparams
  float* hess = grad + nparams;                           // nparams * nparams
  float* fs = hess + nparams * nparams;                   // nfib
  float* f_deriv = fs + nfib;                             // nfib * nfib
  float* x = f_deriv + nfib * nfib;                       // 3 * nfib
  float* _a = x + 3 * nfib;                               // 1 (also _d)
  float* _b = _a + 1;                                     // 1
  float* sumf = _b + 1;                                   // 1
  const int t = threadIdx.x, v = blockIdx.x;
  const float* y = data + (size_t)v * ndirections;
  if (t < nparams) myparams[t] = params[(size_t)v * nparams + t];
  __syncthreads();
  if (kind == 0) {
    cf_PVM_single(myparams, y, bvecs, bvals, ndirections, nfib, nparams, f0, t, reduction, fs, x, _a, sumf, cfv);
    __syncthreads();
    grad_PVM_single(myparams, y, bvecs, bvals, ndirections, nfib, nparams, f0, t, J, reduction, fs, x, _a, sumf, grad);
    __syncthreads();
    hess_PVM_single(myparams, bvecs, bvals, ndirections, nfib, nparams, f0, t, J, reduction, fs, x, _a, sumf, hess);
  } else if (kind == 1) {
    cf_PVM_single_c(myparams, y, bvecs, bvals, ndirections, nfib, nparams, f0, t, reduction, fs, x, _a, sumf, cfv);
    __syncthreads();
    grad_PVM_single_c(myparams, y, bvecs, bvals, ndirections, nfib, nparams, f0, t, J, reduction, fs, f_deriv, x,
                      _a, sumf, grad);
    __syncthreads();
    hess_PVM_single_c(myparams, bvecs, bvals, ndirections, nfib, nparams, f0, t, J, reduction, fs, f_deriv, x, _a,
                      sumf, hess);
  } else {
    cf_PVM_multi(myparams, y, bvecs, bvals, R, invR, ndirections, nfib, nparams, f0, t, gbo, reduction, fs, x, _a,
                 _b, sumf, cfv);
    __syncthreads();
    grad_PVM_multi(myparams, y, bvecs, bvals, R, invR, ndirections, nfib, nparams, f0, t, gbo, J, reduction, fs, x,
                   _a, _b, sumf, grad);
    __syncthreads();
    hess_PVM_multi(myparams, bvecs, bvals, R, invR, ndirections, nfib, nparams, f0, t, gbo, J, reduction, fs, x, _a,
                   _b, sumf, hess);
  }
  __syncthreads();
  if (t == 0) cf_out[v] = *cfv;
  if (t < nparams) grad_out[(size_t)v * nparams + t] = grad[t];
  for (int i = t; i < nparams * nparams; i += blockDim.x) hess_out[(size_t)v * nparams * nparams + i] = hess[i];
}

// polar angle and azimuth of every gradient direction in double (MISCMATHS::cart2sph, as
// CUDA/xfibres_gpu.cu:421-446 uses it to fill alpha/beta)
void angles(int ndir, const float* bvecs, std::vector<double>& alpha, std::vector<double>& beta) {
  alpha.resize(ndir);
  beta.resize(ndir);
  for (int m = 0; m < ndir; ++m) {
    const double x = bvecs[m], y = bvecs[ndir + m], z = bvecs[2 * ndir + m];
    const double mag = std::sqrt(x * x + y * y + z * z);
    alpha[m] = mag == 0 ? M_PI / 2 : std::acos(z / mag);
    beta[m] = (x == 0 && y == 0) ? M_PI / 2 : std::atan2(y, x);
  }
}

}  // namespace

extern "C" {

const char* refgpu_last_error(void) { return g_err; }

// device milliseconds (CUDA events around the kernels only) of the last refgpu_fit (ms[0]) and
// refgpu_mcmc (ms[1]: init_Fibres_Multifibres + randoms + burn-in; ms[2]: recording) calls
void refgpu_last_times(float* ms) {
  for (int i = 0; i < 3; ++i) ms[i] = g_ms[i];
}

// Cost (double), gradient and Hessian (float) of the reference's LM models at raw parameters
// params [nvox][nparams]; see lm_eval_kernel.
int refgpu_lm_eval(int kind, int nfib, int f0, int gbo, float R, int nvox, int ndir, const float* data,
                   const float* bvecs, const float* bvals, const float* params, double* cf, float* grad,
                   float* hess) {
  const int np = 3 * nfib + 2 + (kind == 2 ? 1 : 0) + (f0 ? 1 : 0);
  Buf<float> d_data, d_bvecs, d_bvals, d_params, d_grad, d_hess;
  Buf<double> d_cf;
  RG_CUDA(d_data.put(data, (size_t)nvox * ndir));
  RG_CUDA(d_bvecs.put(bvecs, (size_t)3 * ndir));
  RG_CUDA(d_bvals.put(bvals, (size_t)ndir));
  RG_CUDA(d_params.put(params, (size_t)nvox * np));
  RG_CUDA(d_cf.alloc(nvox));
  RG_CUDA(d_grad.alloc((size_t)nvox * np));
  RG_CUDA(d_hess.alloc((size_t)nvox * np * np));
  const size_t shared = sizeof(double) + sizeof(float) * (THREADS_BLOCK_FIT * np + THREADS_BLOCK_FIT + 2 * np +
                                                          np * np + nfib + nfib * nfib + 3 * nfib + 3);
  const float invR = 1.0f / (2.0f * R + 1.0f);
  if (nvox > 0) {
    lm_eval_kernel<<<nvox, THREADS_BLOCK_FIT, shared>>>(kind, d_data.p, d_bvecs.p, d_bvals.p, R, invR, ndir, nfib,
                                                        np, f0 != 0, gbo, d_params.p, d_cf.p, d_grad.p, d_hess.p);
    RG_CUDA(cudaGetLastError());
    RG_CUDA(cudaDeviceSynchronize());
  }
  RG_CUDA(d_cf.get(cf, nvox));
  RG_CUDA(d_grad.get(grad, (size_t)nvox * np));
  RG_CUDA(d_hess.get(hess, (size_t)nvox * np * np));
  return 0;
}

// The reference's LM fit kernels, launched as CUDA/diffmodels.cu launches them.
//   kind 0 fit_PVM_single_kernel, 1 fit_PVM_single_c_kernel: params [nvox][np] start values in,
//     finalised parameters out (np = 3*nfib + 2 (+1 f0));
//   kind 2 fit_PVM_multi_kernel: start = finalised PVM_single_c parameters [nvox][np-1], out
//     [nvox][np] (np = 3*nfib + 3 (+1 f0)), gbo = Gamma_for_ball_only (0 model 2, 2 model 3).
int refgpu_fit(int kind, int nfib, int f0, int gbo, float R, int nvox, int ndir, const float* data,
               const float* bvecs, const float* bvals, const float* start, float* params_out) {
  const int np = 3 * nfib + 2 + (kind == 2 ? 1 : 0) + (f0 ? 1 : 0);
  const int np_in = kind == 2 ? np - 1 : np;
  Buf<float> d_data, d_bvecs, d_bvals, d_in, d_out;
  RG_CUDA(d_data.put(data, (size_t)nvox * ndir));
  RG_CUDA(d_bvecs.put(bvecs, (size_t)3 * ndir));
  RG_CUDA(d_bvals.put(bvals, (size_t)ndir));
  RG_CUDA(d_in.put(start, (size_t)nvox * np_in));
  if (nvox == 0) return 0;
  const dim3 grid(nvox), block(THREADS_BLOCK_FIT);
  if (kind == 2) RG_CUDA(d_out.alloc((size_t)nvox * np));
  cudaEvent_t e0, e1;
  RG_CUDA(cudaEventCreate(&e0));
  RG_CUDA(cudaEventCreate(&e1));
  RG_CUDA(cudaEventRecord(e0));
  if (kind == 0) {
    // CUDA/diffmodels.cu:98-104
    const int shared = 6 * sizeof(double) +
                       (THREADS_BLOCK_FIT * np + THREADS_BLOCK_FIT + 5 * np + 2 * np * np + 4 * nfib + 2) * sizeof(float) +
                       (2 + np) * sizeof(int);
    fit_PVM_single_kernel<<<grid, block, shared>>>(d_data.p, d_bvecs.p, d_bvals.p, nvox, ndir, nfib, np, f0 != 0,
                                                  false, d_in.p);
    RG_CUDA(cudaGetLastError());
  } else if (kind == 1) {
    // CUDA/diffmodels.cu:182-188
    const int shared = 6 * sizeof(double) +
                       (THREADS_BLOCK_FIT * np + THREADS_BLOCK_FIT + 5 * np + 2 * np * np + 4 * nfib + nfib * nfib + 6) *
                           sizeof(float) +
                       (2 + np) * sizeof(int);
    fit_PVM_single_c_kernel<<<grid, block, shared>>>(d_data.p, d_bvecs.p, d_bvals.p, nvox, ndir, nfib, np, false,
                                                    f0 != 0, false, false, d_in.p);
    RG_CUDA(cudaGetLastError());
  } else {
    // CUDA/diffmodels.cu:232-240
    const int shared = 6 * sizeof(double) +
                       (THREADS_BLOCK_FIT * np + THREADS_BLOCK_FIT + 5 * np + 2 * np * np + 4 * nfib + 3) * sizeof(float) +
                       (2 + np) * sizeof(int);
    const float invR = 1.0f / (2.0f * R + 1.0f);
    fit_PVM_multi_kernel<<<grid, block, shared>>>(d_data.p, d_in.p, d_bvecs.p, d_bvals.p, R, invR, nvox, ndir, nfib,
                                                 np, gbo, f0 != 0, false, d_out.p);
    RG_CUDA(cudaGetLastError());
  }
  RG_CUDA(cudaEventRecord(e1));
  RG_CUDA(cudaDeviceSynchronize());
  RG_CUDA(cudaEventElapsedTime(&g_ms[0], e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  RG_CUDA((kind == 2 ? d_out : d_in).get(params_out, (size_t)nvox * np));
  return 0;
}

// Options of the reference's MCMC kernels (the xfibresOptions fields runmcmc.cu passes).
struct refgpu_mcmc_opts {
  int model, nfib, f0, rician, ardf0, all_ard, no_ard;
  float fudge, R_mean, R_std, R_fudge;
  int nburn, njumps, sampleevery, upe;
  double seed;
};

// init_Fibres_Multifibres_kernel + (optionally) setup_randoms_kernel and the burn-in and
// recording launches of runmcmc_kernel, as CUDA/runmcmc.cu:27-316 runs them, on voxels whose
// start parameters are params [nvox][np_fit] (fit layout) and tau [nvox].
//   lik, prior [nvox]: the energies init_Fibres_Multifibres_kernel computes (may be NULL);
//   records [6+3*nfib][nsamples][nvox] in the row order d, f0, tau, d_std, R, S0, then th, ph, f
//     per fibre (NULL: the chain is not run).  Rows an option does not record stay zero.
// The kernels index voxels without a bound check, so the voxels are padded to a multiple of
// VOXELS_BLOCK_MCMC (copies of the last voxel) and every array is sized for the padded count.
int refgpu_mcmc(const refgpu_mcmc_opts* o, int nvox, int ndir, const float* data, const float* bvecs,
                const float* bvals, const float* params, const float* tau, float* lik, float* prior,
                float* records) {
  if (nvox <= 0) return 0;
  const int K = o->nfib;
  const int np_fit = 2 + 3 * K + (o->model >= 2 ? 1 : 0) + (o->f0 ? 1 : 0);
  const int npad = (nvox + VOXELS_BLOCK_MCMC - 1) / VOXELS_BLOCK_MCMC * VOXELS_BLOCK_MCMC;
  std::vector<float> hd((size_t)npad * ndir), hp((size_t)npad * np_fit), ht(npad);
  for (int v = 0; v < npad; ++v) {
    const int s = v < nvox ? v : nvox - 1;
    std::memcpy(&hd[(size_t)v * ndir], data + (size_t)s * ndir, sizeof(float) * ndir);
    std::memcpy(&hp[(size_t)v * np_fit], params + (size_t)s * np_fit, sizeof(float) * np_fit);
    ht[v] = tau ? tau[s] : 0.f;
  }
  std::vector<double> alpha, beta;
  angles(ndir, bvecs, alpha, beta);
  Buf<float> d_data, d_bvals, d_params, d_tau;
  Buf<double> d_alpha, d_beta, d_angtmp, d_signals, d_iso;
  Buf<FibreGPU> d_fib;
  Buf<MultifibreGPU> d_mf;
  RG_CUDA(d_data.put(hd.data(), hd.size()));
  RG_CUDA(d_bvals.put(bvals, ndir));
  RG_CUDA(d_params.put(hp.data(), hp.size()));
  RG_CUDA(d_tau.put(ht.data(), ht.size()));
  RG_CUDA(d_alpha.put(alpha.data(), ndir));
  RG_CUDA(d_beta.put(beta.data(), ndir));
  RG_CUDA(d_angtmp.alloc((size_t)npad * ndir * K));
  RG_CUDA(d_signals.alloc((size_t)npad * ndir * K));
  RG_CUDA(d_iso.alloc((size_t)npad * ndir));
  RG_CUDA(d_fib.alloc((size_t)npad * K));
  RG_CUDA(d_mf.alloc(npad));
  RG_CUDA(cudaMemset(d_fib.p, 0, sizeof(FibreGPU) * npad * K));
  RG_CUDA(cudaMemset(d_mf.p, 0, sizeof(MultifibreGPU) * npad));
  const dim3 grid(npad / VOXELS_BLOCK_MCMC), block(THREADS_VOXEL_MCMC * VOXELS_BLOCK_MCMC);
  // event pairs around the kernels only (not the allocations between them): init, randoms, burn-in,
  // recording
  cudaEvent_t ev[8];
  for (int i = 0; i < 8; ++i) RG_CUDA(cudaEventCreate(&ev[i]));
  RG_CUDA(cudaEventRecord(ev[0]));
  // CUDA/runmcmc.cu:86-89
  const int sh_init =
      VOXELS_BLOCK_MCMC * ((THREADS_VOXEL_MCMC) * sizeof(double) + (3 * K + 9) * sizeof(float) + sizeof(int));
  init_Fibres_Multifibres_kernel<<<grid, block, sh_init>>>(
      d_data.p, d_params.p, d_tau.p, d_bvals.p, d_alpha.p, d_beta.p, o->R_mean, o->R_std, o->R_fudge, ndir, K, np_fit,
      o->model, o->fudge, o->f0 != 0, o->rician != 0, o->ardf0 != 0, o->all_ard != 0, o->no_ard != 0, false,
      d_angtmp.p, d_fib.p, d_mf.p, d_signals.p, d_iso.p);
  RG_CUDA(cudaGetLastError());
  RG_CUDA(cudaEventRecord(ev[1]));
  RG_CUDA(cudaDeviceSynchronize());
  if (lik || prior) {
    std::vector<MultifibreGPU> mf(npad);
    RG_CUDA(d_mf.get(mf.data(), npad));
    for (int v = 0; v < nvox; ++v) {
      if (lik) lik[v] = mf[v].m_likelihood_en;
      if (prior) prior[v] = mf[v].m_prior_en;
    }
  }
  if (!records) {
    for (int i = 0; i < 8; ++i) cudaEventDestroy(ev[i]);
    return 0;
  }
  // setup_randoms_kernel (CUDA/runmcmc.cu:92-99)
  Buf<curandState> d_rand;
  RG_CUDA(d_rand.alloc(npad));
  const int rblocks = (npad + THREADS_BLOCK_RAND - 1) / THREADS_BLOCK_RAND;
  RG_CUDA(cudaEventRecord(ev[2]));
  setup_randoms_kernel<<<rblocks, THREADS_BLOCK_RAND>>>(d_rand.p, o->seed, npad);
  RG_CUDA(cudaGetLastError());
  RG_CUDA(cudaEventRecord(ev[3]));
  // runmcmc_kernel launches (CUDA/runmcmc.cu:135-200, 237-311)
  int nparams = (o->f0 ? 3 : 2) + 3 * K;
  if (o->model >= 2) nparams++;
  if (o->model == 3) nparams++;
  if (o->rician) nparams++;
  const int ns = o->njumps / o->sampleevery;
  Buf<double> d_oldsig, d_oldiso, d_oldang;
  RG_CUDA(d_oldsig.alloc((size_t)npad * ndir * K));
  RG_CUDA(d_oldiso.alloc((size_t)npad * ndir));
  RG_CUDA(d_oldang.alloc((size_t)npad * ndir));
  Buf<float> r_null, rf0, rtau, rs0, rd, rdstd, rR, rth, rph, rf;
  RG_CUDA(r_null.alloc(1));
  const size_t n1 = (size_t)npad * ns, nk = (size_t)npad * ns * K;
  RG_CUDA(rf0.alloc(n1));
  RG_CUDA(rtau.alloc(n1));
  RG_CUDA(rs0.alloc(n1));
  RG_CUDA(rd.alloc(n1));
  RG_CUDA(rdstd.alloc(n1));
  RG_CUDA(rR.alloc(n1));
  RG_CUDA(rth.alloc(nk));
  RG_CUDA(rph.alloc(nk));
  RG_CUDA(rf.alloc(nk));
  for (Buf<float>* b : {&rf0, &rtau, &rs0, &rd, &rdstd, &rR, &rth, &rph, &rf})
    RG_CUDA(cudaMemset(b->p, 0, b->n * sizeof(float)));
  const int sh_mcmc = VOXELS_BLOCK_MCMC * ((THREADS_VOXEL_MCMC) * sizeof(double) + (10 * K + 27) * sizeof(float) +
                                           (7 * K + 20) * sizeof(int) + sizeof(curandState));
  RG_CUDA(cudaEventRecord(ev[4]));
  if (o->nburn > 0) {
    runmcmc_kernel<<<grid, block, sh_mcmc>>>(
        d_data.p, d_bvals.p, d_alpha.p, d_beta.p, d_rand.p, o->R_mean, o->R_std, o->R_fudge, ndir, K, nparams, o->model,
        o->fudge, o->f0 != 0, o->ardf0 != 0, !o->no_ard, o->rician != 0, false, o->upe, o->nburn, 0, 0, 0, d_oldsig.p,
        d_oldiso.p, d_angtmp.p, d_oldang.p, d_fib.p, d_mf.p, d_signals.p, d_iso.p, r_null.p, r_null.p, r_null.p,
        r_null.p, r_null.p, r_null.p, r_null.p, r_null.p, r_null.p);
    RG_CUDA(cudaGetLastError());
  }
  RG_CUDA(cudaEventRecord(ev[5]));
  runmcmc_kernel<<<grid, block, sh_mcmc>>>(
      d_data.p, d_bvals.p, d_alpha.p, d_beta.p, d_rand.p, o->R_mean, o->R_std, o->R_fudge, ndir, K, nparams, o->model,
      o->fudge, o->f0 != 0, o->ardf0 != 0, !o->no_ard, o->rician != 0, false, o->upe, o->njumps, o->nburn,
      o->sampleevery, ns, d_oldsig.p, d_oldiso.p, d_angtmp.p, d_oldang.p, d_fib.p, d_mf.p, d_signals.p, d_iso.p,
      rf0.p, rtau.p, rs0.p, rd.p, rdstd.p, rR.p, rth.p, rph.p, rf.p);
  RG_CUDA(cudaGetLastError());
  RG_CUDA(cudaEventRecord(ev[6]));
  RG_CUDA(cudaDeviceSynchronize());
  float t_init = 0.f, t_rand = 0.f, t_burn = 0.f;
  RG_CUDA(cudaEventElapsedTime(&t_init, ev[0], ev[1]));
  RG_CUDA(cudaEventElapsedTime(&t_rand, ev[2], ev[3]));
  RG_CUDA(cudaEventElapsedTime(&t_burn, ev[4], ev[5]));
  RG_CUDA(cudaEventElapsedTime(&g_ms[2], ev[5], ev[6]));
  g_ms[1] = t_init + t_rand + t_burn;
  for (int i = 0; i < 8; ++i) cudaEventDestroy(ev[i]);
  // the reference's record arrays: r[vox*ns + s] and rk[vox*ns*K + k*ns + s]
  std::vector<float> h1(n1), hk(nk);
  const Buf<float>* rows1[6] = {&rd, &rf0, &rtau, &rdstd, &rR, &rs0};
  for (int r = 0; r < 6; ++r) {
    RG_CUDA(rows1[r]->get(h1.data(), n1));
    for (int s = 0; s < ns; ++s)
      for (int v = 0; v < nvox; ++v) records[((size_t)r * ns + s) * nvox + v] = h1[(size_t)v * ns + s];
  }
  const Buf<float>* rowsk[3] = {&rth, &rph, &rf};
  for (int q = 0; q < 3; ++q) {
    RG_CUDA(rowsk[q]->get(hk.data(), nk));
    for (int k = 0; k < K; ++k)
      for (int s = 0; s < ns; ++s)
        for (int v = 0; v < nvox; ++v)
          records[((size_t)(6 + 3 * k + q) * ns + s) * nvox + v] = hk[(size_t)v * ns * K + (size_t)k * ns + s];
  }
  return 0;
}

}  // extern "C"
