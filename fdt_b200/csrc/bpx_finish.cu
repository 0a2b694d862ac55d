// bpx_finish.cu -- sample finishing on the GPU.
//
// Replaces record_finish_voxels + Samples::record / finish_voxel / save
// (CUDA/xfibres_gpu.cu:659-738, CUDA/samples.cu:134-347), which the reference runs on the host
// after copying every record back: per voxel the sample means, the principal eigenvector of
// each fibre's mean dyadic tensor, and the fibres re-ordered by decreasing sum of f over samples
// into the th/ph/f sample arrays.  One thread per voxel; the [row][sample][voxel] layout makes
// every read and write coalesced across a warp.
#include <cstdint>

#include "bpx_device.cuh"
#include "bpx_internal.h"

namespace bpx {

// principal eigenvector of a symmetric 3x3 (cyclic Jacobi, FP64), largest |component| positive;
// returns the largest eigenvalue
__device__ double principal_vector(double (&A)[3][3], double (&out)[3]) {
  double V[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  for (int sweep = 0; sweep < 50; ++sweep) {
    const double off = A[0][1] * A[0][1] + A[0][2] * A[0][2] + A[1][2] * A[1][2];
    if (off < 1e-300) break;
#pragma unroll
    for (int p = 0; p < 3; ++p)
#pragma unroll
      for (int q = p + 1; q < 3; ++q) {
        const double apq = A[p][q];
        if (fabs(apq) < 1e-300) continue;
        const double theta = (A[q][q] - A[p][p]) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
        const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const double akp = A[k][p], akq = A[k][q];
          A[k][p] = c * akp - s * akq;
          A[k][q] = s * akp + c * akq;
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const double apk = A[p][k], aqk = A[q][k];
          A[p][k] = c * apk - s * aqk;
          A[q][k] = s * apk + c * aqk;
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const double vkp = V[k][p], vkq = V[k][q];
          V[k][p] = c * vkp - s * vkq;
          V[k][q] = s * vkp + c * vkq;
        }
      }
  }
  int best = 0;
  if (A[1][1] > A[best][best]) best = 1;
  if (A[2][2] > A[best][best]) best = 2;
  double col[3];
#pragma unroll
  for (int r = 0; r < 3; ++r) col[r] = (best == 0) ? V[r][0] : (best == 1 ? V[r][1] : V[r][2]);
  int big = 0;
  if (fabs(col[1]) > fabs(col[big])) big = 1;
  if (fabs(col[2]) > fabs(col[big])) big = 2;
  const double sg = col[big] < 0 ? -1.0 : 1.0;
#pragma unroll
  for (int r = 0; r < 3; ++r) out[r] = sg * col[r];
  return A[best][best];
}

template <int K>
__device__ void finish_voxel(const FinishArgs& a, int v) {
  const int ns = a.nsamples, nvox = a.nvox;
  const size_t row = (size_t)ns * nvox;
  const float* rec = a.records + v;
  // the fibre order first, from the sums of f over the samples (the f rows, a fifth of the
  // records): sort (sum f, index) ascending and read it backwards (CUDA/samples.cu:299-330)
  double sumf[K];
#pragma unroll
  for (int k = 0; k < K; ++k) sumf[k] = 0;
  for (int s = 0; s < ns; ++s) {
#pragma unroll
    for (int k = 0; k < K; ++k) sumf[k] += rec[(8 + 3 * k) * row + (size_t)s * nvox];
  }
  int slot[K];  // output position of fibre k: the number of fibres that come before it
#pragma unroll
  for (int i = 0; i < K; ++i) {
    int rank = 0;
#pragma unroll
    for (int j = 0; j < K; ++j)
      if (j != i && (sumf[j] > sumf[i] || (sumf[j] == sumf[i] && j > i))) ++rank;
    slot[i] = rank;
  }
  // one pass over the records: sums, dyadic tensors, and every sample copied to its sorted slot
  // (each output row is written once, whole sectors at a time across the warp)
  double sums[6] = {0, 0, 0, 0, 0, 0}, dy[K][3][3];
#pragma unroll
  for (int k = 0; k < K; ++k)
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) dy[k][i][j] = 0;
  const bpx_outputs& out = a.out;
  for (int s = 0; s < ns; ++s) {
    const size_t o = (size_t)s * nvox;
#pragma unroll
    for (int r = 0; r < 6; ++r) sums[r] += rec[r * row + o];
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const float th = rec[(6 + 3 * k) * row + o], ph = rec[(7 + 3 * k) * row + o];
      float st, ct, sp, cp;
      sincosf(th, &st, &ct);
      sincosf(ph, &sp, &cp);
      const double x[3] = {(double)st * cp, (double)st * sp, (double)ct};
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) dy[k][i][j] += x[i] * x[j];
      const size_t oo = ((size_t)slot[k] * ns + s) * nvox + v;
      if (out.th) out.th[oo] = th;
      if (out.ph) out.ph[oo] = ph;
      if (out.f) out.f[oo] = rec[(8 + 3 * k) * row + o];
    }
  }
  const double inv = 1.0 / ns;
  if (out.mean_d) out.mean_d[v] = (float)(sums[0] * inv);
  if (out.mean_f0) out.mean_f0[v] = (float)(sums[1] * inv);
  if (out.mean_tau) out.mean_tau[v] = (float)(sums[2] * inv);
  if (out.mean_dstd) out.mean_dstd[v] = (float)(sums[3] * inv);
  if (out.mean_R) out.mean_R[v] = (float)(sums[4] * inv);
  if (out.mean_S0) out.mean_S0[v] = (float)(sums[5] * inv);
#pragma unroll
  for (int o = 0; o < K; ++o) {
    int src = 0;
#pragma unroll
    for (int i = 0; i < K; ++i)
      if (slot[i] == o) src = i;
    double sf = 0, A[3][3];
#pragma unroll
    for (int i = 0; i < K; ++i)
      if (i == src) {
        sf = sumf[i];
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
          for (int c = 0; c < 3; ++c) A[r][c] = dy[i][r][c];
      }
    if (out.mean_f) out.mean_f[(size_t)o * nvox + v] = (float)(sf * inv);
    if (out.dyads) {
      double pv[3];
      principal_vector(A, pv);
#pragma unroll
      for (int r = 0; r < 3; ++r) out.dyads[((size_t)o * 3 + r) * nvox + v] = (float)pv[r];
    }
  }
}

// One thread per voxel (grid-stride).  The f rows are read first to fix the fibre order, then
// every record once more while the sums are formed and the samples copied to their sorted slots.
template <int K>
__global__ void finish_kernel(FinishArgs a) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < a.nvox; v += gridDim.x * blockDim.x) finish_voxel<K>(a, v);
}

// bedpostx_postproc_gpu.sh arithmetic (CUDA/bedpostx_postproc_gpu.sh:20-49) on the finished
// outputs, one thread per voxel: fslmaths -Tmean of merged_th/ph, the dispersion of each fibre's
// mean dyadic tensor (make_dyadic_vectors.cc:60-92: 1 - max |eigenvalue|), maskdyads
// (dyads{k} where mean_f{k} >= thr, fslmaths -thr -bin -mul), the _modf{k} scaling by
// mean_f{k}/mean_f1 (fslmaths -div gives 0 where the divisor is 0) and mean_fsumsamples.
template <int K>
__global__ void postproc_kernel(PostArgs a) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= a.nvox) return;
  const int ns = a.nsamples, nvox = a.nvox;
  const bpx_postproc& p = a.post;
  float mf[K];
  double fsum = 0.0;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    mf[k] = a.mean_f[(size_t)k * nvox + v];
    fsum += mf[k];
    double sth = 0, sph = 0, A[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int s = 0; s < ns; ++s) {
      const size_t o = ((size_t)k * ns + s) * nvox + v;
      const float th = a.th[o], ph = a.ph[o];
      sth += th;
      sph += ph;
      float st, ct, sp, cp;
      sincosf(th, &st, &ct);
      sincosf(ph, &sp, &cp);
      const double x[3] = {(double)st * cp, (double)st * sp, (double)ct};
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) A[i][j] += x[i] * x[j] / ns;
    }
    if (p.mean_th) p.mean_th[(size_t)k * nvox + v] = (float)(sth / ns);
    if (p.mean_ph) p.mean_ph[(size_t)k * nvox + v] = (float)(sph / ns);
    if (p.dispersion) {
      double pv[3];
      const double lmax = principal_vector(A, pv);  // the tensor is positive semi-definite
      p.dispersion[(size_t)k * nvox + v] = (float)(1.0 - fabs(lmax));
    }
  }
  if (p.mean_fsum) p.mean_fsum[v] = (float)fsum;
#pragma unroll
  for (int k = 1; k < K; ++k) {
    const bool keep = mf[k] >= a.thr && mf[k] != 0.f;
    const float ratio = mf[0] != 0.f ? mf[k] / mf[0] : 0.f;
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      const size_t o = ((size_t)k * 3 + r) * nvox + v;
      const float dt = keep ? a.dyads[o] : 0.f;
      if (p.dyads_thr) p.dyads_thr[o] = dt;
      if (p.dyads_modf) p.dyads_modf[o] = dt * ratio;
    }
  }
}

cudaError_t launch_postproc(const PostArgs& a, cudaStream_t s) {
  if (a.nvox == 0) return cudaSuccess;
  const int threads = 128, grid = (a.nvox + threads - 1) / threads;
  switch (a.nfib) {
    case 1: postproc_kernel<1><<<grid, threads, 0, s>>>(a); break;
    case 2: postproc_kernel<2><<<grid, threads, 0, s>>>(a); break;
    case 3: postproc_kernel<3><<<grid, threads, 0, s>>>(a); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_finish(const FinishArgs& a, cudaStream_t s) {
  if (a.nvox == 0) return cudaSuccess;
  const int threads = 128;
  const int grid = (a.nvox + threads - 1) / threads;
  switch (a.nfib) {
    case 1: finish_kernel<1><<<grid, threads, 0, s>>>(a); break;
    case 2: finish_kernel<2><<<grid, threads, 0, s>>>(a); break;
    case 3: finish_kernel<3><<<grid, threads, 0, s>>>(a); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace bpx
