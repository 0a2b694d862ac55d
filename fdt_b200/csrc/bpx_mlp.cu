// bpx_mlp.cu -- the learned initialiser: a network that maps a voxel's normalised signals to the
// MCMC's starting state and per-voxel proposal widths, its training step, and the learned
// pipeline entry.  No counterpart in the reference (xfibres_gpu starts every chain from LM fits,
// CUDA/xfibres_gpu.cu:82-118, and adapts the proposal widths during the chain,
// CUDA/runmcmc_kernels.cu:1341-1395).
//
// Network: x (ndir signals / S0_hat, padded to nin = 8*ceil(ndir/8)) -> 256 -> 256 -> 256 -> 256
// (GELU after each) -> 32 outputs.  BF16 weights and activations, FP32 accumulation, FP32 master
// parameters.  Every contraction (forward, dX, dW) runs on the tcgen05 GEMM of bpx_gemm.cu with
// the bias, GELU and GELU-derivative fused into its epilogue.
//
// Flat parameter vector (FP32): for layer l = 0..4, W_l [n_l][k_l] row-major then b_l [n_l];
// k = {nin, 256, 256, 256, 256}, n = {256, 256, 256, 256, 32}.
//
// Output vector (32): 0-2 f_k, 3-11 fibre unit vectors v_k, 12 d*1e3, 13 d_std*1e3, 14 S0/S0_hat,
// 15 f0*10, 16 ln(tau*S0_hat^2), 17.. ln of the normalised proposal width of MCMC slot q, in [-14, 2]
// (q = 0..5+3K in the slot order f0, tau, d, d_std, R, S0, (th, ph, f)_k; widths of S0 are
// divided by S0_hat, of d and d_std multiplied by 1e3, of tau divided by tau).
#include <mutex>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <string>

#include "bpx.h"
#include "bpx_device.cuh"
#include "bpx_gemm.h"
#include "bpx_internal.h"

namespace bpx {
namespace mlp {

constexpr int kWidth = BPX_MLP_WIDTH;
constexpr int kLayers = BPX_MLP_HIDDEN + 1;
constexpr int kOut = BPX_MLP_NOUT;
constexpr int kOutProps = 17;  // first proposal-width output
// Range of the normalised log widths.  A chain adapts the angle widths of a fibre whose fraction
// is near zero without bound (every proposal is accepted; CUDA/runmcmc_kernels.cu caps them at
// 1e10), but a width past e^2 (> 2 pi for an angle, > 1 for a fraction) proposes no differently.
constexpr float kLogWidthMin = -14.f, kLogWidthMax = 2.f;
constexpr int kMaxChunk = 32768;  // inference rows per pass (bounds the activation buffers)

struct Geom {
  int nin;
  int k[kLayers], n[kLayers];
  size_t woff[kLayers], boff[kLayers], wbf[kLayers];
  size_t nparams, nw;
};

Geom geom(int ndir) {
  Geom g;
  g.nin = (ndir + 7) / 8 * 8;
  size_t o = 0, w = 0;
  for (int l = 0; l < kLayers; ++l) {
    g.k[l] = l == 0 ? g.nin : kWidth;
    g.n[l] = l == kLayers - 1 ? kOut : kWidth;
    g.woff[l] = o;
    g.wbf[l] = w;
    o += (size_t)g.k[l] * g.n[l];
    w += (size_t)g.k[l] * g.n[l];
    g.boff[l] = o;
    o += g.n[l];
  }
  g.nparams = o;
  g.nw = w;
  return g;
}

struct WeightMap {
  size_t woff[kLayers], wbf[kLayers + 1];
};

__global__ void cast_weights_kernel(const float* __restrict__ params, WeightMap m, uint16_t* __restrict__ wbf) {
  const size_t total = m.wbf[kLayers];
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    int l = 0;
#pragma unroll
    for (int t = 1; t < kLayers; ++t)
      if (i >= m.wbf[t]) l = t;
    wbf[i] = __bfloat16_as_ushort(__float2bfloat16_rn(params[m.woff[l] + (i - m.wbf[l])]));
  }
}

// Normalised signals: S0_hat = mean of the measurements with b <= 50 s/mm^2 (the largest signal
// when there are none); x = y / S0_hat in BF16, zero past ndir.  One warp per voxel.
__global__ void features_kernel(int nvox, int ndir, int nin, const float* __restrict__ data,
                                const float* __restrict__ bvals, int per_voxel_b, uint16_t* __restrict__ x,
                                float* __restrict__ s0hat) {
  const int lane = threadIdx.x & 31;
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int v = w; v < nvox; v += nwarps) {
    const float* y = data + (size_t)v * ndir;
    const float* b = per_voxel_b ? bvals + (size_t)v * ndir : bvals;
    float s = 0.f, c = 0.f, mx = 0.f;
    for (int m = lane; m < ndir; m += 32) {
      const float yy = y[m];
      if (b[m] <= 50.f) {
        s += yy;
        c += 1.f;
      }
      mx = fmaxf(mx, yy);
    }
    s = group_sum<32>(s);
    c = group_sum<32>(c);
    mx = group_max<32>(mx);
    float s0 = c > 0.f ? s / c : mx;
    if (!(s0 > 0.f) || !isfinite(s0)) s0 = 1.f;
    const float inv = 1.f / s0;
    uint16_t* xr = x + (size_t)v * nin;
    for (int m = lane; m < nin; m += 32) {
      const float val = m < ndir ? y[m] * inv : 0.f;
      xr[m] = __bfloat16_as_ushort(__float2bfloat16_rn(isfinite(val) ? val : 0.f));
    }
    if (lane == 0) s0hat[v] = s0;
  }
}

// Loss of one voxel and its gradient with respect to the outputs (averaged over the batch):
//   sum_j w_j (o_j - t_j)^2 over the scalar outputs, plus, for fibre k, w_{3+3k} times the
//   sign-invariant direction loss |u u^T - v v^T|_F^2 = |u|^4 - 2 (u.v)^2 + 1 (|v| = 1).
__global__ void loss_kernel(int batch, const float* __restrict__ out, const float* __restrict__ t,
                            const float* __restrict__ tw, uint16_t* __restrict__ dz, float* __restrict__ loss) {
  __shared__ float red[8];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  float L = 0.f;
  if (i < batch) {
    const float* o = out + (size_t)i * kOut;
    const float* tt = t + (size_t)i * kOut;
    const float* ww = tw + (size_t)i * kOut;
    float g[kOut];
    const float inv_b = 1.f / (float)batch;
#pragma unroll
    for (int j = 0; j < kOut; ++j) g[j] = 0.f;
#pragma unroll
    for (int j = 0; j < kOut; ++j) {
      if (j >= 3 && j < 12) continue;
      const float e = o[j] - tt[j];
      L += ww[j] * e * e;
      g[j] = 2.f * ww[j] * e * inv_b;
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const float wd = ww[3 + 3 * k];
      const float ux = o[3 + 3 * k], uy = o[4 + 3 * k], uz = o[5 + 3 * k];
      const float vx = tt[3 + 3 * k], vy = tt[4 + 3 * k], vz = tt[5 + 3 * k];
      const float uu = ux * ux + uy * uy + uz * uz, uv = ux * vx + uy * vy + uz * vz;
      L += wd * (uu * uu - 2.f * uv * uv + 1.f);
      const float a = 4.f * wd * uu * inv_b, c = -4.f * wd * uv * inv_b;
      g[3 + 3 * k] = a * ux + c * vx;
      g[4 + 3 * k] = a * uy + c * vy;
      g[5 + 3 * k] = a * uz + c * vz;
    }
    uint16_t* d = dz + (size_t)i * kOut;
#pragma unroll
    for (int j = 0; j < kOut; ++j) d[j] = __bfloat16_as_ushort(__float2bfloat16_rn(g[j]));
  }
  L = group_sum<32>(L);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = L;
  __syncthreads();
  if (threadIdx.x == 0) {
    float s = 0.f;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
    atomicAdd(loss, s / (float)batch);
  }
}

// db[n] = sum over rows of dz[r][n] (bf16 in, fp32 out); block = 256 threads covers 32 columns.
__global__ void colsum_kernel(int rows, int cols, const uint16_t* __restrict__ dz, float* __restrict__ db) {
  __shared__ float red[8][33];
  const int c = blockIdx.x * 32 + (threadIdx.x & 31);
  const int r0 = threadIdx.x >> 5;
  float s = 0.f;
  if (c < cols)
    for (int r = r0; r < rows; r += 8) s += __bfloat162float(__ushort_as_bfloat16(dz[(size_t)r * cols + c]));
  red[r0][threadIdx.x & 31] = s;
  __syncthreads();
  if (r0 == 0 && c < cols) {
    float t = 0.f;
    for (int j = 0; j < 8; ++j) t += red[j][threadIdx.x & 31];
    db[c] = t;
  }
}

__global__ void adam_kernel(size_t n, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
  }
}

struct Layout {
  int model, K, f0, rician, np, ns;
};

// Training targets from a fitted state (LM fit layout [S0, d, (d_std), (f, th, ph)_k, (f0)]) and,
// when given, the proposal widths a plain chain adapted to ([NS][nvox]).
__global__ void targets_kernel(Layout L, int nvox, const float* __restrict__ params, const float* __restrict__ tau,
                               const float* __restrict__ props, const float* __restrict__ s0hat,
                               float* __restrict__ t, float* __restrict__ tw) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nvox) return;
  const float* p = params + (size_t)v * L.np;
  float* o = t + (size_t)v * kOut;
  float* w = tw + (size_t)v * kOut;
  for (int j = 0; j < kOut; ++j) {
    o[j] = 0.f;
    w[j] = 0.f;
  }
  const int add = L.model >= 2 ? 1 : 0;
  const float s0 = s0hat[v];
  for (int k = 0; k < L.K; ++k) {
    const float f = p[2 + add + 3 * k], th = p[3 + add + 3 * k], ph = p[4 + add + 3 * k];
    float st, ct, sp, cp;
    sincosf(th, &st, &ct);
    sincosf(ph, &sp, &cp);
    o[k] = f;
    w[k] = 1.f;
    o[3 + 3 * k] = st * cp;
    o[4 + 3 * k] = st * sp;
    o[5 + 3 * k] = ct;
    w[3 + 3 * k] = fminf(fmaxf(f, 0.f), 1.f);
  }
  o[12] = p[1] * 1e3f;
  w[12] = 1.f;
  if (L.model >= 2) {
    o[13] = p[2] * 1e3f;
    w[13] = 1.f;
  }
  o[14] = p[0] / s0;
  w[14] = 1.f;
  if (L.f0) {
    o[15] = p[L.np - 1] * 10.f;
    w[15] = 1.f;
  }
  const float tv = (L.rician && tau) ? tau[v] : 0.f;
  if (L.rician && tau && tv > 0.f) {
    o[16] = logf(tv * s0 * s0);
    w[16] = 0.1f;
  }
  if (props) {
    for (int q = 0; q < L.ns; ++q) {
      const bool on = (q == kSlotD) || (q == kSlotS0) || (q >= kSlotFibre0) || (q == kSlotTau && L.rician) ||
                      (q == kSlotF0 && L.f0) || (q == kSlotDstd && L.model >= 2) || (q == kSlotR && L.model == 3);
      float pw = props[(size_t)q * nvox + v];
      if (q == kSlotS0) pw /= s0;
      if (q == kSlotD || q == kSlotDstd) pw *= 1e3f;
      if (q == kSlotTau) pw = tv > 0.f ? pw / tv : 0.f;
      if (on && pw > 0.f && isfinite(pw)) {
        o[kOutProps + q] = fminf(fmaxf(logf(pw), kLogWidthMin), kLogWidthMax);
        w[kOutProps + q] = 0.1f;
      }
    }
  }
  // a chain that met a non-finite state leaves non-finite labels: such targets get weight 0 and
  // value 0 (a zero weight alone does not stop 0 * NaN from reaching the loss), a direction as a whole
  for (int k = 0; k < 3; ++k)
    if (!(isfinite(o[3 + 3 * k]) && isfinite(o[4 + 3 * k]) && isfinite(o[5 + 3 * k])))
      for (int c = 0; c < 3; ++c) {
        o[3 + 3 * k + c] = 0.f;
        w[3 + 3 * k + c] = 0.f;
      }
  for (int j = 0; j < kOut; ++j)
    if (!isfinite(o[j]) || !isfinite(w[j])) {
      o[j] = 0.f;
      w[j] = 0.f;
    }
}

// Network outputs -> MCMC starting state (fit layout), tau and proposal widths [NS][nvox]; the
// fractions are clipped to [0.001, 0.95] and scaled so that sum f + f0 < 0.98.
__global__ void decode_kernel(Layout L, int nvox, const float* __restrict__ out, const float* __restrict__ s0hat,
                              float* __restrict__ params, float* __restrict__ tau, float* __restrict__ props,
                              uint32_t* __restrict__ status) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nvox) return;
  const float* o = out + (size_t)v * kOut;
  float* p = params + (size_t)v * L.np;
  const int add = L.model >= 2 ? 1 : 0;
  const float s0 = s0hat[v];
  float f[BPX_MAX_FIBRES], sum = 0.f;
  for (int k = 0; k < L.K; ++k) {
    f[k] = fminf(fmaxf(o[k], 0.001f), 0.95f);
    sum += f[k];
  }
  float f0 = L.f0 ? fminf(fmaxf(o[15] * 0.1f, 0.001f), 0.5f) : 0.f;
  const float tot = sum + f0;
  if (tot > 0.98f) {
    const float sc = 0.98f / tot;
    for (int k = 0; k < L.K; ++k) f[k] *= sc;
    f0 *= sc;
  }
  const float d = fminf(fmaxf(o[12] * 1e-3f, 1e-5f), 0.0049f);
  p[0] = fmaxf(o[14], 0.05f) * s0;
  p[1] = d;
  if (L.model >= 2) p[2] = fminf(fmaxf(o[13] * 1e-3f, 1e-6f), 0.0099f);
  for (int k = 0; k < L.K; ++k) {
    float ux = o[3 + 3 * k], uy = o[4 + 3 * k], uz = o[5 + 3 * k];
    const float nn = sqrtf(ux * ux + uy * uy + uz * uz);
    if (nn > 1e-12f) {
      ux /= nn;
      uy /= nn;
      uz /= nn;
    } else {
      ux = 0.f;
      uy = 0.f;
      uz = 1.f;
    }
    p[2 + add + 3 * k] = f[k];
    p[3 + add + 3 * k] = acosf(fminf(fmaxf(uz, -1.f), 1.f));
    p[4 + add + 3 * k] = atan2f(uy, ux);
  }
  if (L.f0) p[L.np - 1] = f0;
  const float tv = expf(fminf(fmaxf(o[16], -20.f), 40.f)) / (s0 * s0);
  if (tau) tau[v] = tv;
  if (props) {
    for (int q = 0; q < L.ns; ++q) {
      float pw = expf(fminf(fmaxf(o[kOutProps + q], kLogWidthMin), kLogWidthMax));
      if (q == kSlotS0) pw *= s0;
      if (q == kSlotD || q == kSlotDstd) pw *= 1e-3f;
      if (q == kSlotTau) pw *= tv;
      props[(size_t)q * nvox + v] = pw;
    }
  }
  if (status) status[v] = 0u;
}

}  // namespace mlp
}  // namespace bpx

using namespace bpx;
using namespace bpx::mlp;

namespace {

size_t a256(size_t x) { return (x + 255) & ~(size_t)255; }

#define MLP_CUDA(call)                                          \
  do {                                                          \
    cudaError_t e_ = (call);                                    \
    if (e_ != cudaSuccess) return api_cuda_fail(e_, #call);     \
  } while (0)

bpx_status run_gemm(const uint16_t* a, int lda, int a_mn, const uint16_t* b, int ldb, int b_mn, int M, int N, int K,
                    int epi, float* out_f32, int ld_out, uint16_t* out_bf16, int ld_bf16, const float* bias,
                    const float* zin, int ld_zin, int* err, cudaStream_t s) {
  gemm::GemmOperands op{a, b, lda, ldb};
  gemm::GemmArgs g{};
  g.M = M;
  g.N = N;
  g.K = K;
  g.ntile = N <= 32 ? 32 : N <= 64 ? 64 : N <= 128 ? 128 : 256;
  g.a_mn = a_mn;
  g.b_mn = b_mn;
  g.epi = epi;
  g.out_f32 = out_f32;
  g.ld_out = ld_out;
  g.out_bf16 = out_bf16;
  g.ld_bf16 = ld_bf16;
  g.bias = bias;
  g.zin = zin;
  g.ld_zin = ld_zin;
  g.error = err;
  const char* why = nullptr;
  const cudaError_t e = gemm::launch(op, g, s, &why);
  if (why) return api_fail(BPX_ERR_INVALID_ARG, std::string("tcgen05 GEMM: ") + why);
  if (e != cudaSuccess) return api_cuda_fail(e, "gemm launch");
  return BPX_OK;
}

// per-device error word the GEMM's bounded waits write; read by bpx_mlp_poll_error
std::mutex g_err_mutex;
int* g_err[64] = {nullptr};
uint64_t g_err_ctx[64] = {0};  // context_id() the word was allocated in

bpx_status error_word(int** out) {
  int dev = 0;
  MLP_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return api_fail(BPX_ERR_NO_DEVICE, "device index out of range");
  std::lock_guard<std::mutex> lk(g_err_mutex);
  if (g_err[dev] && g_err_ctx[dev] != context_id()) g_err[dev] = nullptr;  // its context is gone
  if (!g_err[dev]) {
    MLP_CUDA(cudaMalloc(&g_err[dev], sizeof(int)));
    MLP_CUDA(cudaMemset(g_err[dev], 0, sizeof(int)));
    g_err_ctx[dev] = context_id();
  }
  *out = g_err[dev];
  return BPX_OK;
}

bpx_status cast_weights(const Geom& G, const float* params, uint16_t* wbf, cudaStream_t s) {
  WeightMap m;
  for (int l = 0; l < kLayers; ++l) {
    m.woff[l] = G.woff[l];
    m.wbf[l] = G.wbf[l];
  }
  m.wbf[kLayers] = G.nw;
  cast_weights_kernel<<<(unsigned)std::min<size_t>((G.nw + 255) / 256, 4096), 256, 0, s>>>(params, m, wbf);
  MLP_CUDA(cudaGetLastError());
  return BPX_OK;
}

// forward pass of rows [0, n) of x; activations in the network workspace
bpx_status forward(const Geom& G, const float* params, const uint16_t* wbf, int n, const uint16_t* x, float* out,
                   uint16_t* buf0, uint16_t* buf1, float* const* z, uint16_t* const* acts, int* err, cudaStream_t s) {
  const uint16_t* a = x;
  int lda = G.nin;
  for (int l = 0; l < kLayers - 1; ++l) {
    uint16_t* o = acts ? acts[l] : ((l & 1) ? buf1 : buf0);
    bpx_status st = run_gemm(a, lda, 0, wbf + G.wbf[l], G.k[l], 0, n, G.n[l], G.k[l], gemm::kEpiBiasGelu,
                             z ? z[l] : nullptr, G.n[l], o, G.n[l], params + G.boff[l], nullptr, 0, err, s);
    if (st != BPX_OK) return st;
    a = o;
    lda = G.n[l];
  }
  const int l = kLayers - 1;
  return run_gemm(a, lda, 0, wbf + G.wbf[l], G.k[l], 0, n, G.n[l], G.k[l], gemm::kEpiBias, out, kOut, nullptr, 0,
                  params + G.boff[l], nullptr, 0, err, s);
}

Layout layout_of(const bpx_options* o) {
  Layout L;
  L.model = o->model;
  L.K = o->nfibres;
  L.f0 = o->f0;
  L.rician = o->rician;
  L.np = bpx_nparams_fit(o);
  L.ns = 6 + 3 * o->nfibres;
  return L;
}

}  // namespace

namespace bpx {

size_t mlp_weight_elems(int ndir) { return geom(ndir).nw; }

bpx_status mlp_forward_buffers(int ndir, const float* params, int nvox, const uint16_t* x, float* out, uint16_t* wbf,
                               uint16_t* buf0, uint16_t* buf1, int chunk_rows, cudaStream_t s) {
  NvtxRange nvtx_range("bpx.network");
  const Geom G = geom(ndir);
  int* err = nullptr;
  bpx_status st = error_word(&err);
  if (st == BPX_OK) st = cast_weights(G, params, wbf, s);
  for (int r0 = 0; st == BPX_OK && r0 < nvox; r0 += chunk_rows) {
    const int n = std::min(chunk_rows, nvox - r0);
    st = forward(G, params, wbf, n, x + (size_t)r0 * G.nin, out + (size_t)r0 * kOut, buf0, buf1, nullptr, nullptr, err,
                 s);
  }
  return st;
}

}  // namespace bpx

extern "C" {

int32_t bpx_mlp_nin(int32_t ndir) { return ndir < 1 ? -1 : (ndir + 7) / 8 * 8; }

int64_t bpx_mlp_nparams(int32_t ndir) { return ndir < 1 ? -1 : (int64_t)geom(ndir).nparams; }

bpx_status bpx_gemm_bf16_dev(int32_t M, int32_t N, int32_t K, const uint16_t* A, int32_t lda, int32_t a_mn,
                             const uint16_t* B, int32_t ldb, int32_t b_mn, float* C, int32_t ldc, void* stream) {
  if (!A || !B || !C) return api_fail(BPX_ERR_INVALID_ARG, "bpx_gemm_bf16_dev: NULL operand");
  bpx_status st = api_check_device();
  if (st != BPX_OK) return st;
  int* err = nullptr;
  st = error_word(&err);
  if (st != BPX_OK) return st;
  return run_gemm(A, lda, a_mn != 0, B, ldb, b_mn != 0, M, N, K, gemm::kEpiStoreF32, C, ldc, nullptr, 0, nullptr,
                  nullptr, 0, err, (cudaStream_t)stream);
}

bpx_status bpx_mlp_poll_error(int32_t* code) {
  if (!code) return api_fail(BPX_ERR_INVALID_ARG, "code is NULL");
  int* err = nullptr;
  bpx_status st = error_word(&err);
  if (st != BPX_OK) return st;
  int h = 0;
  MLP_CUDA(cudaMemcpy(&h, err, sizeof(int), cudaMemcpyDeviceToHost));
  MLP_CUDA(cudaMemset(err, 0, sizeof(int)));
  *code = h;
  return BPX_OK;
}

bpx_status bpx_mlp_features_dev(const bpx_volume* vol, int32_t per_voxel_bvals, uint16_t* x, float* s0hat,
                                void* stream) {
  bpx_status st = api_check_vol(vol);
  if (st != BPX_OK) return st;
  if (vol->nvox == 0) return BPX_OK;
  if (!x || !s0hat) return api_fail(BPX_ERR_INVALID_ARG, "bpx_mlp_features_dev: NULL output");
  st = api_check_device();
  if (st != BPX_OK) return st;
  const int nin = bpx_mlp_nin(vol->ndir);
  const int blocks = std::min((vol->nvox + 7) / 8, sm_count() * 16);
  features_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(vol->nvox, vol->ndir, nin, vol->data, vol->bvals,
                                                             per_voxel_bvals, x, s0hat);
  MLP_CUDA(cudaGetLastError());
  return BPX_OK;
}

bpx_status bpx_mlp_forward_dev(int32_t ndir, const float* params, int32_t nvox, const uint16_t* x, float* out,
                               void* stream) {
  if (ndir < 1 || nvox < 0 || !params || (nvox > 0 && (!x || !out)))
    return api_fail(BPX_ERR_INVALID_ARG, "bpx_mlp_forward_dev: bad arguments");
  if (nvox == 0) return BPX_OK;
  bpx_status st = api_check_device();
  if (st != BPX_OK) return st;
  const Geom G = geom(ndir);
  const int chunk = std::min<int>(nvox, kMaxChunk);
  const size_t b_w = a256(G.nw * 2), b_act = a256((size_t)chunk * kWidth * 2);
  void* ws = nullptr;
  st = api_workspace(kWsNetwork, b_w + 2 * b_act, &ws);
  if (st != BPX_OK) return st;
  int* err = nullptr;
  st = error_word(&err);
  if (st != BPX_OK) return st;
  char* p = (char*)ws;
  uint16_t* wbf = (uint16_t*)p;
  uint16_t* buf0 = (uint16_t*)(p + b_w);
  uint16_t* buf1 = (uint16_t*)(p + b_w + b_act);
  cudaStream_t s = (cudaStream_t)stream;
  st = cast_weights(G, params, wbf, s);
  if (st != BPX_OK) return st;
  for (int r0 = 0; r0 < nvox; r0 += chunk) {
    const int n = std::min(chunk, nvox - r0);
    st = forward(G, params, wbf, n, x + (size_t)r0 * G.nin, out + (size_t)r0 * kOut, buf0, buf1, nullptr, nullptr,
                 err, s);
    if (st != BPX_OK) return st;
  }
  return BPX_OK;
}

bpx_status bpx_mlp_train_step_dev(int32_t ndir, const float* params, float* grads, int32_t batch, const uint16_t* x,
                                  const float* targets, const float* tweights, float* loss, void* stream) {
  if (ndir < 1 || batch < 1 || !params || !grads || !x || !targets || !tweights || !loss)
    return api_fail(BPX_ERR_INVALID_ARG, "bpx_mlp_train_step_dev: bad arguments");
  bpx_status st = api_check_device();
  if (st != BPX_OK) return st;
  const Geom G = geom(ndir);
  const size_t B = (size_t)batch;
  const size_t b_w = a256(G.nw * 2), b_a = a256(B * kWidth * 2), b_z = a256(B * kWidth * 4);
  const size_t b_out = a256(B * kOut * 4), b_dz5 = a256(B * kOut * 2);
  void* ws = nullptr;
  st = api_workspace(kWsNetwork, b_w + 4 * b_a + 4 * b_z + b_out + b_dz5 + 2 * b_a, &ws);
  if (st != BPX_OK) return st;
  int* err = nullptr;
  st = error_word(&err);
  if (st != BPX_OK) return st;
  char* p = (char*)ws;
  uint16_t* wbf = (uint16_t*)p;
  p += b_w;
  uint16_t* acts[4];
  float* z[4];
  for (int i = 0; i < 4; ++i, p += b_a) acts[i] = (uint16_t*)p;
  for (int i = 0; i < 4; ++i, p += b_z) z[i] = (float*)p;
  float* out = (float*)p;
  p += b_out;
  uint16_t* dz5 = (uint16_t*)p;
  p += b_dz5;
  uint16_t* dzb[2] = {(uint16_t*)p, (uint16_t*)(p + b_a)};
  cudaStream_t s = (cudaStream_t)stream;
  st = cast_weights(G, params, wbf, s);
  if (st != BPX_OK) return st;
  st = forward(G, params, wbf, batch, x, out, nullptr, nullptr, z, acts, err, s);
  if (st != BPX_OK) return st;
  MLP_CUDA(cudaMemsetAsync(loss, 0, sizeof(float), s));
  loss_kernel<<<(batch + 255) / 256, 256, 0, s>>>(batch, out, targets, tweights, dz5, loss);
  MLP_CUDA(cudaGetLastError());
  // backward: g = dL/d(layer output); dW_l = g^T a_l, db_l = colsum(g), g <- (g W_l) * gelu'(z_l)
  const uint16_t* g = dz5;
  int ldg = kOut;
  for (int l = kLayers - 1; l >= 0; --l) {
    const uint16_t* al = l == 0 ? x : acts[l - 1];
    st = run_gemm(g, ldg, 1, al, G.k[l], 1, G.n[l], G.k[l], batch, gemm::kEpiStoreF32, grads + G.woff[l], G.k[l],
                  nullptr, 0, nullptr, nullptr, 0, err, s);
    if (st != BPX_OK) return st;
    colsum_kernel<<<(G.n[l] + 31) / 32, 256, 0, s>>>(batch, G.n[l], g, grads + G.boff[l]);
    MLP_CUDA(cudaGetLastError());
    if (l == 0) break;
    uint16_t* gn = dzb[l & 1];
    st = run_gemm(g, ldg, 0, wbf + G.wbf[l], G.k[l], 1, batch, G.k[l], G.n[l], gemm::kEpiGeluGrad, nullptr, 0, gn,
                  G.k[l], nullptr, z[l - 1], G.k[l], err, s);
    if (st != BPX_OK) return st;
    g = gn;
    ldg = G.k[l];
  }
  return BPX_OK;
}

bpx_status bpx_mlp_adam_dev(int64_t n, float* params, const float* grads, float* m, float* v, float lr, float beta1,
                            float beta2, float eps, int32_t step, void* stream) {
  if (n < 0 || step < 1 || (n > 0 && (!params || !grads || !m || !v)))
    return api_fail(BPX_ERR_INVALID_ARG, "bpx_mlp_adam_dev: bad arguments");
  if (n == 0) return BPX_OK;
  bpx_status st = api_check_device();
  if (st != BPX_OK) return st;
  const float c1 = 1.f / (1.f - powf(beta1, (float)step)), c2 = 1.f / (1.f - powf(beta2, (float)step));
  const unsigned blocks = (unsigned)std::min<int64_t>((n + 255) / 256, (int64_t)sm_count() * 8);
  adam_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>((size_t)n, params, grads, m, v, lr, beta1, beta2, eps, c1, c2);
  MLP_CUDA(cudaGetLastError());
  return BPX_OK;
}

bpx_status bpx_mlp_targets_dev(const bpx_options* opts, int32_t nvox, const float* params, const float* tau,
                               const float* props, const float* s0hat, float* targets, float* tweights,
                               void* stream) {
  bpx_status st = api_check_opts(opts);
  if (st != BPX_OK) return st;
  if (nvox < 0 || (nvox > 0 && (!params || !s0hat || !targets || !tweights)))
    return api_fail(BPX_ERR_INVALID_ARG, "bpx_mlp_targets_dev: bad arguments");
  if (nvox == 0) return BPX_OK;
  st = api_check_device();
  if (st != BPX_OK) return st;
  targets_kernel<<<(nvox + 127) / 128, 128, 0, (cudaStream_t)stream>>>(layout_of(opts), nvox, params, tau, props, s0hat,
                                                                       targets, tweights);
  MLP_CUDA(cudaGetLastError());
  return BPX_OK;
}

bpx_status bpx_mlp_decode_dev(const bpx_options* opts, int32_t nvox, const float* out, const float* s0hat,
                              float* params, float* tau, float* props, uint32_t* status, void* stream) {
  bpx_status st = api_check_opts(opts);
  if (st != BPX_OK) return st;
  if (nvox < 0 || (nvox > 0 && (!out || !s0hat || !params)))
    return api_fail(BPX_ERR_INVALID_ARG, "bpx_mlp_decode_dev: bad arguments");
  if (nvox == 0) return BPX_OK;
  st = api_check_device();
  if (st != BPX_OK) return st;
  decode_kernel<<<(nvox + 127) / 128, 128, 0, (cudaStream_t)stream>>>(layout_of(opts), nvox, out, s0hat, params, tau,
                                                                      props, status);
  MLP_CUDA(cudaGetLastError());
  return BPX_OK;
}

bpx_status bpx_xfibres_learned_dev(const bpx_options* opts, const bpx_volume* vol, const float* mlp_params,
                                   int32_t freeze_props, bpx_outputs* out, void* stream) {
  NvtxRange nvtx_range("bpx.xfibres_learned");
  bpx_status st = api_check_opts(opts);
  if (st == BPX_OK) st = api_check_vol(vol);
  if (st != BPX_OK) return st;
  if (!out || !mlp_params) return api_fail(BPX_ERR_INVALID_ARG, "out or mlp_params is NULL");
  if (freeze_props < 0 || freeze_props > 2) return api_fail(BPX_ERR_INVALID_ARG, "freeze_props must be 0, 1 or 2");
  if (vol->nvox == 0) return BPX_OK;
  const int ns = bpx_nsamples(opts);
  if (ns < 1) return api_fail(BPX_ERR_INVALID_ARG, "no samples (njumps < sampleevery)");
  st = api_check_device();
  if (st != BPX_OK) return st;
  const size_t nvox = vol->nvox;
  const int nin = bpx_mlp_nin(vol->ndir);
  const size_t np = bpx_nparams_fit(opts), nsl = 6 + 3 * opts->nfibres, nrec = BPX_NREC(opts->nfibres);
  const size_t b_x = a256(nvox * nin * 2), b_v = a256(nvox * 4), b_out = a256(nvox * kOut * 4);
  const size_t b_par = a256(nvox * np * 4), b_props = a256(nsl * nvox * 4), b_rec = a256(nrec * ns * nvox * 4);
  void* ws = nullptr;
  st = api_workspace(kWsLearned, b_x + 3 * b_v + b_out + b_par + b_props + b_rec, &ws);
  if (st != BPX_OK) return st;
  char* p = (char*)ws;
  uint16_t* x = (uint16_t*)p;
  p += b_x;
  float* s0hat = (float*)p;
  p += b_v;
  float* tau = (float*)p;
  p += b_v;
  uint32_t* status = out->status ? out->status : (uint32_t*)p;
  p += b_v;
  float* netout = (float*)p;
  p += b_out;
  float* params = (float*)p;
  p += b_par;
  float* props = (float*)p;
  p += b_props;
  float* rec = (float*)p;
  if (opts->rician) {
    st = bpx_prepare_data_dev(vol->nvox, vol->ndir, const_cast<float*>(vol->data), stream);
    if (st != BPX_OK) return st;
  }
  st = bpx_mlp_features_dev(vol, opts->gradnonlin, x, s0hat, stream);
  if (st == BPX_OK) st = bpx_mlp_forward_dev(vol->ndir, mlp_params, vol->nvox, x, netout, stream);
  if (st == BPX_OK) st = bpx_mlp_decode_dev(opts, vol->nvox, netout, s0hat, params, tau, props, status, stream);
  if (st == BPX_OK)
    st = bpx_mcmc_ex_dev(opts, vol, params, opts->rician ? tau : nullptr, props, nullptr, freeze_props, rec, status,
                         stream);
  if (st == BPX_OK) st = bpx_finish_dev(opts, vol->nvox, rec, out, stream);
  return st;
}

}  // extern "C"
