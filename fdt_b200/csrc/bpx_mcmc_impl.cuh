// bpx_mcmc_impl.cuh -- the MCMC kernel of the bedpostx path (template; instantiated per model
// in bpx_mcmc_m{1,2,3}.cu).
//
// Replaces init_Fibres_Multifibres_kernel + runmcmc_kernel (burn-in and recording launches)
// of CUDA/runmcmc_kernels.cu:193-1474 with one launch that runs each voxel's whole chain.
//
// Layout: a group of TPV lanes owns one voxel; lane l of the group holds measurements
// l, l+TPV, ... (at most MPL of them) as packed pairs plus one unpaired tail.  Registers hold
// what changes during the chain: the per-fibre stick signals and the isotropic signal.  Shared
// memory holds what is read-only or rarely written: the (g, b) table, each thread's data y and
// padding weights, the backups of signals a proposal overwrites, the group's proposal widths,
// acceptance counts and fibre state (angles, directions, priors).  The scalar chain state is
// replicated in every lane of the group, so the accept/reject logic needs no broadcast;
// likelihood sums use an xor-butterfly over the group.  A proposal overwrites the signals it
// changes in place (old values backed up in shared memory) and restores them if rejected.
//
// Random numbers: slot s of iteration it of voxel v uses Philox-4x32-10 with counter
// (it, s, v) and key = seed.  At the start of each iteration lane l computes slots l, l+TPV, ...
// once, and proposals fetch theirs with a shuffle.
//
// Deviations from the reference, all of which leave the chain's target distribution unchanged:
//   * FP32 signals and likelihoods (the reference uses FP64); energy differences are formed as
//     (M/2) ln(SS_old/SS_new) (Gaussian) or M ln(tau_new/tau_old) + sum(t_new - t_old) (Rician)
//     with the Rician terms written as log y - tau (y-p)^2/2 + [logI0(z) - z], so no large
//     cancelling sums appear in FP32.
//   * log I0, sin and cos from polynomials fitted for this library (bpx_device.cuh), at FP32
//     accuracy, in place of the reference's A&S polynomials and the CUDA math library.
//   * a proposal rejected by its prior skips the likelihood (the reference evaluates and
//     discards it); its random numbers are consumed either way, being slot-keyed.
//   * fibre directions enter as dot products (g.v)^2 instead of the reference's three cosines of
//     spherical angles (CUDA/runmcmc_kernels.cu:389-398, same quantity).
#pragma once

#include <cstdint>
#include <type_traits>

#include "bpx_device.cuh"
#include "bpx_internal.h"

namespace bpx {

template <int MODEL>
struct SigParams {
  // model 1 (or model 2 with d_std < 1e-5): s = 2^(e1 * b * c), iso = 2^(e1 * b)
  // model 2: s = 2^(-alpha * log2(1 + beta * b * c))
  // model 3: s = 2^(e3 * b * ((1-R) c + R))
  float e1, alpha, beta, e3, omR, R;
  bool mono;
};

template <int MODEL>
__device__ __forceinline__ SigParams<MODEL> sig_params(float d, float dstd, float R) {
  SigParams<MODEL> sp;
  sp.e1 = -d * kLog2e;
  sp.mono = (MODEL == 1) || (dstd < 1e-5f);
  if (MODEL >= 2) {
    const float s2 = dstd * dstd;
    sp.alpha = d * d / s2;
    sp.beta = s2 / d;
  } else {
    sp.alpha = 0.f;
    sp.beta = 0.f;
  }
  if (MODEL == 3) {
    const float invR = 1.0f / (2.0f * R + 1.0f);
    sp.e3 = -3.0f * d * invR * kLog2e;
    sp.omR = 1.0f - R;
    sp.R = R;
  } else {
    sp.e3 = 0.f;
    sp.omR = 0.f;
    sp.R = 0.f;
  }
  return sp;
}

// compute_signal (CUDA/runmcmc_kernels.cu:67-83)
template <int MODEL>
__device__ __forceinline__ float stick_signal(const SigParams<MODEL>& sp, float b, float c) {
  if (MODEL == 1) return ex2_approx(sp.e1 * b * c);
  if (MODEL == 2) {
    if (sp.mono) return ex2_approx(sp.e1 * b * c);
    return ex2_approx(-sp.alpha * lg2_approx(1.0f + sp.beta * b * c));
  }
  return ex2_approx(sp.e3 * b * (sp.omR * c + sp.R));
}

// compute_iso_signal (CUDA/runmcmc_kernels.cu:84-95)
template <int MODEL>
__device__ __forceinline__ float iso_signal(const SigParams<MODEL>& sp, float b) {
  if (MODEL == 1 || sp.mono) return ex2_approx(sp.e1 * b);
  return ex2_approx(-sp.alpha * lg2_approx(1.0f + sp.beta * b));
}

struct Priors {
  float fudge, R_mean, R_std, R_fudge;
  int ardf0, can_use_ard;
};

// theta prior -log|sin(th)/2| (CUDA/runmcmc_kernels.cu:1142-1147), given sin(th)
__device__ __forceinline__ float th_prior(float th, float sin_th) {
  return th == 0.f ? 0.f : -ln_approx(fabsf(sin_th * 0.5f));
}

// R prior (CUDA/runmcmc_kernels.cu:1058-1083); returns true if R is rejected
__device__ __forceinline__ bool r_prior(const Priors& pr, float R, float d, float& prior) {
  float upper_R = 2.0f * pr.R_mean;
  float lower_R = pr.R_mean - 2.0f * pr.R_std;
  if (pr.R_mean > 0.5f) upper_R = 1.0f;
  if (lower_R < 0.0f) lower_R = 1e-8f;
  if (pr.R_fudge > 0.0f && d > kUpperDiff / 2.0f) {
    if (R < 1e-8f || R > upper_R) return true;
    prior = pr.R_fudge * ln_approx(R);
    return false;
  }
  if (R <= lower_R || R > upper_R) return true;
  prior = (R - pr.R_mean) * (R - pr.R_mean) / (pr.R_std * pr.R_std);
  return false;
}

// per-lane measurement arrays of the energy kernel (one state per voxel, no chain)
template <int MODEL, int K, bool RIC, int TPV, int MPL>
struct Lanes {
  float y[MPL], b[MPL], c[K][MPL], s[K][MPL], iso[MPL];
  int nj;  // measurements held by this lane
};

// energy difference E_old - E_new of the likelihood part
template <bool RIC>
__device__ __forceinline__ float dlik(float st_old, float st_new, float tau_old, float tau_new, float halfM, float M) {
  if (!RIC) return halfM * logf(st_old / st_new);
  return M * logf(tau_new / tau_old) + (st_new - st_old);
}

// likelihood energy difference when tau is unchanged (the Rician M ln(tau'/tau) term is zero)
template <bool RIC>
__device__ __forceinline__ float dlik_same_tau(float st_old, float st_new, float halfM) {
  if (!RIC) return halfM * logf(st_old / st_new);
  return st_new - st_old;
}

// all lanes of this lane's group agree on a group-uniform flag; with one group per warp the flag
// is warp-uniform already, otherwise a vote over the warp tells whether any group disagrees
template <int TPV>
__device__ __forceinline__ bool group_all(bool x) {
  if constexpr (TPV == 32) return x;
  return __all_sync(0xffffffffu, x);
}

// a rejected proposal's signals go back to their backups: with one group per warp the decision
// is warp-uniform and the caller only gets here on rejection, so the backup is taken as it is
template <int TPV, typename T>
__device__ __forceinline__ T keep_or_restore(bool ok, T cur, T old) {
  if constexpr (TPV == 32) return old;
  if constexpr (sizeof(T) == 8) return make_float2(ok ? cur.x : old.x, ok ? cur.y : old.y);
  return ok ? cur : old;
}

// select element kf (runtime, < K) of a register array without local memory
template <int K, typename T>
__device__ __forceinline__ T pick(const T (&a)[K], int kf) {
  T r = a[0];
#pragma unroll
  for (int k = 1; k < K; ++k)
    if (k == kf) r = a[k];
  return r;
}

// ---- scalar / packed-pair arithmetic ------------------------------------------------------
// A lane's measurements are processed two at a time with the sm_100 packed FP32x2 instructions
// (one issue slot for two FMAs); an odd measurement left over uses the scalar forms.
__device__ __forceinline__ float vfma(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ float2 vfma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float vmul(float a, float b) { return a * b; }
__device__ __forceinline__ float2 vmul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float vadd(float a, float b) { return a + b; }
__device__ __forceinline__ float2 vadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
template <typename V>
__device__ __forceinline__ V vbc(float x);
template <>
__device__ __forceinline__ float vbc<float>(float x) { return x; }
template <>
__device__ __forceinline__ float2 vbc<float2>(float x) { return make_float2(x, x); }
__device__ __forceinline__ float vex2(float x) { return ex2_approx(x); }
__device__ __forceinline__ float2 vex2(float2 x) { return make_float2(ex2_approx(x.x), ex2_approx(x.y)); }
__device__ __forceinline__ float vlg2(float x) { return lg2_approx(x); }
__device__ __forceinline__ float2 vlg2(float2 x) { return make_float2(lg2_approx(x.x), lg2_approx(x.y)); }
__device__ __forceinline__ float vhsum(float x) { return x; }
__device__ __forceinline__ float vhsum(float2 x) { return x.x + x.y; }

// Rician log-likelihood terms without their log(y) part, sum_m w (-tau (y-p)^2/2 + logI0(z) - z)
// with p = S0 base and z = tau p y, for one or two measurements, accumulated as
//   -tau/2 rr + ln2 lg2(prod) - zs,   rr += w r^2,
// where each measurement multiplies prod by I0(z) (z < kI0Split, and zs gains z) or by e^-z I0(z)
// (z >= kI0Split).  The reference's logIo (fibre.h:31-51 / CUDA/runmcmc_kernels.cu:126-145) uses the
// Abramowitz & Stegun 9.8.1/9.8.2 polynomials split at 3.75 (degrees 6 and 8); the kI0Small/kI0Large
// polynomials of bpx_device.cuh, split at 4.75, have degrees 6 and 5 at the same accuracy (log I0
// within 6e-7 after FP32 rounding).  Both branches are evaluated, branch-free, since the measurements
// of one warp fall on both sides of the split; the unselected branch may be inf or NaN (rsqrt of a
// small z), which the select discards.  Every factor lies in (0, 22] (I0(4.75) = 21.8), so a product of five stays in
// FP32's normal range for z below ~1e14 and one log2 per product replaces one per measurement.
// Padding measurements (y = 0, w = 0) give z = 0 and the factor kI0Small(0) = 1.
__device__ __forceinline__ void rician_pick(float z, float q, float pr, float& sel, float& zs) {
  const bool small = z < kI0Split;
  sel = small ? q : pr;
  zs = small ? z : 0.f;
}
template <typename V, bool W = true>
__device__ __forceinline__ void rician_acc(V y, V w, V base, V nS0, V tS0, V& rr, V& prod, V& zs) {
  const V r = vfma(nS0, base, y);
  const V z = vmul(tS0, vmul(y, base));
  const V u = vmul(z, z);
  V q = vfma(u, vbc<V>(kI0Small(6)), vbc<V>(kI0Small(5)));
#pragma unroll
  for (int i = 4; i >= 0; --i) q = vfma(u, q, vbc<V>(kI0Small(i)));
  V rs;
  if constexpr (sizeof(V) == 8) {
    rs = make_float2(rsqrt_approx(z.x), rsqrt_approx(z.y));
  } else {
    rs = rsqrt_approx(z);
  }
  const V v = vmul(rs, rs);
  V p = vfma(v, vbc<V>(kI0Large(5)), vbc<V>(kI0Large(4)));
#pragma unroll
  for (int i = 3; i >= 0; --i) p = vfma(v, p, vbc<V>(kI0Large(i)));
  const V pr = vmul(p, rs);
  V sel, zz;
  if constexpr (sizeof(V) == 8) {
    rician_pick(z.x, q.x, pr.x, sel.x, zz.x);
    rician_pick(z.y, q.y, pr.y, sel.y, zz.y);
  } else {
    rician_pick(z, q, pr, sel, zz);
  }
  prod = vmul(prod, sel);
  zs = vadd(zs, zz);
  rr = W ? vfma(vmul(r, w), r, rr) : vfma(r, r, rr);  // w is 1 wherever W is false
}

// signals of one or two measurements (compute_signal / compute_iso_signal, CUDA/runmcmc_kernels.cu:67-95).
// MONO selects the model-2 mono-exponential form (d_std < 1e-5) at compile time: callers branch on
// sp.mono once around their measurement loops, so each form costs only its own MUFU operations.
template <int MODEL, bool MONO, typename V>
__device__ __forceinline__ V stick_v(const SigParams<MODEL>& sp, V b, V bbeta, V c) {
  if (MODEL == 1 || (MODEL == 2 && MONO)) return vex2(vmul(vmul(vbc<V>(sp.e1), b), c));
  if (MODEL == 2) return vex2(vmul(vbc<V>(-sp.alpha), vlg2(vfma(bbeta, c, vbc<V>(1.0f)))));
  return vex2(vmul(vmul(vbc<V>(sp.e3), b), vfma(vbc<V>(sp.omR), c, vbc<V>(sp.R))));
}
template <int MODEL, bool MONO, typename V>
__device__ __forceinline__ V iso_v(const SigParams<MODEL>& sp, V b, V bbeta) {
  if (MODEL == 1 || MONO) return vex2(vmul(vbc<V>(sp.e1), b));
  return vex2(vmul(vbc<V>(-sp.alpha), vlg2(vadd(bbeta, vbc<V>(1.0f)))));
}

// Runs body(std::true_type) for the mono-exponential form (model 1, or d_std < 1e-5: the model-2
// sticks and the model-2/3 isotropic signal), body(std::false_type) otherwise.
template <int MODEL, typename F>
__device__ __forceinline__ void with_signal_form(const SigParams<MODEL>& sp, F&& body) {
  if (MODEL >= 2 && !sp.mono)
    body(std::false_type{});
  else
    body(std::true_type{});
}

// Gaussian likelihood contribution of one or two measurements, w (y - S0 base)^2
template <int K, typename V, bool W = true>
__device__ __forceinline__ V gauss_v(V y, V w, V isov, const V (&sk)[K], V nS0, const V (&fk)[K], V f0, V wiso) {
  V base = vfma(wiso, isov, f0);
#pragma unroll
  for (int k = 0; k < K; ++k) base = vfma(fk[k], sk[k], base);
  const V r = vfma(nS0, base, y);
  return W ? vmul(vmul(r, w), r) : vmul(r, r);  // w is 1 wherever W is false
}

// Rows of the per-group fibre state in shared memory (K entries each).
enum FibreStateRow : int { kFsTh = 0, kFsPh, kFsVx, kFsVy, kFsVz, kFsPth, kFsPf, kFsRows };

// Proposal-slot descriptors, two bits per slot: kind (0: f0, tau, S0 or a fraction; 1: theta or
// phi of a fibre; 2: d, d_std or R) and fibre index; one bit per slot: theta slots.
constexpr int slot_kind(int s) {
  return (s >= kSlotFibre0 && (s - kSlotFibre0) % 3 != 2) ? 1 : ((s == kSlotD || s == kSlotDstd || s == kSlotR) ? 2 : 0);
}
template <int K>
constexpr uint32_t slot_bits(int what) {
  uint32_t m = 0;
  for (int s = 0; s < 6 + 3 * K; ++s) {
    const int fib = s - kSlotFibre0;
    if (what == 0) m |= (uint32_t)slot_kind(s) << (2 * s);
    if (what == 1 && fib >= 0) m |= (uint32_t)(fib / 3) << (2 * s);
    if (what == 2 && fib >= 0 && fib % 3 == 0) m |= 1u << s;
  }
  return m;
}

// STRETCH: compiled with the checkpoint/resume arguments of McmcArgs (it_begin/it_end, state and
// acceptance counts in and out); without it the kernel runs the whole chain from the LM state.
// WPAD: which residuals carry the padding weights w.  2: all (the general case); 1: only the
// unpaired measurement's (M >= 2 * (MPL / 2) * TPV: the pairs hold no padding); 0: none
// (M = TPV * MPL).  Where w is 1 the multiply is skipped: the same sums, bit for bit.
template <int MODEL, int K, bool RIC, int TPV, int MPL, bool STRETCH, int WPAD = 2>
__global__ void __launch_bounds__(kMcmcThreads, mcmc_min_blocks<MPL>()) mcmc_kernel(McmcArgs a) {
  constexpr int NS = 6 + 3 * K;             // proposal slots
  constexpr int NR = (NS + TPV - 1) / TPV;  // Philox blocks per lane per iteration
  constexpr int GPW = 32 / TPV;             // groups (voxels) per warp
  constexpr int GPB = kMcmcThreads / TPV;   // groups per block
  constexpr int NP = MPL / 2;               // measurement pairs per lane
  constexpr bool TAIL = (MPL & 1) != 0;     // one unpaired measurement per lane
  constexpr int NG = TPV * MPL;             // float4 (g, b) entries per copy
  constexpr uint32_t kSlotKinds = slot_bits<K>(0), kSlotFibres = slot_bits<K>(1), kSlotTheta = slot_bits<K>(2);
  extern __shared__ float4 smem4[];
  const int lane = threadIdx.x & 31;
  const int gl = lane % TPV;
  const int gw = lane / TPV;
  const int gblk = threadIdx.x / TPV;
  const int tid = threadIdx.x;
  const int warps_total = gridDim.x * (blockDim.x >> 5);
  const int warp_id = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int M = a.ndir;
  const float halfM = 0.5f * (float)M, fM = (float)M;
  const int total = a.nburn + a.njumps;
  const int ns = a.nsamples;
  Priors pr;
  pr.fudge = a.fudge;
  pr.R_mean = a.R_mean;
  pr.R_std = a.R_std;
  pr.R_fudge = a.R_fudge;
  pr.ardf0 = a.ardf0;
  pr.can_use_ard = !a.no_ard;
  const bool use_f0 = a.f0 != 0;
  // slots proposed by this model: f0 with --f0, tau when Rician, d_std for models 2-3, R for model 3
  const uint32_t enabled = ((1u << NS) - 1u) & ~((use_f0 ? 0u : 1u << kSlotF0) | (RIC ? 0u : 1u << kSlotTau) |
                                                  (MODEL >= 2 ? 0u : 1u << kSlotDstd) | (MODEL == 3 ? 0u : 1u << kSlotR));

  // shared memory: the (g_x, g_y, g_z, b) table in pair order (one copy per block, or per group
  // under gradnonlin); each thread's data y and padding weights w (read-only during the chain, so
  // kept out of registers); per-thread backups of the signals a proposal overwrites; per-group
  // proposal widths and acceptance counts.  Pair p of lane l is entries p*TPV+l = {gx0,gx1,gy0,gy1} and
  // (NP+p)*TPV+l = {gz0,gz1,b0,b1} for measurements l+2p*TPV and l+(2p+1)*TPV (consecutive lanes
  // read consecutive 16-byte entries, free of bank conflicts); the unpaired measurement
  // l+(MPL-1)*TPV is entry 2*NP*TPV+l.  Measurements past M read zeros.
  const int ncopy = a.gradnonlin ? GPB : 1;
  float4* gb = smem4 + (a.gradnonlin ? gblk * NG : 0);
  float4* ywp = smem4 + ncopy * NG;                      // {y0, y1, w0, w1} of pair p: ywp[p * threads + tid]
  float2* ywt = (float2*)(ywp + NP * kMcmcThreads);      // {y, w} of the unpaired measurement: ywt[tid]
  float* after = (float*)(ywt + kMcmcThreads);
  float2* bkp = (float2*)after + tid;  // pair backup c: bkp[c * kMcmcThreads]
  float* bkt = after + 2 * (K + 1) * NP * kMcmcThreads + tid;
  float* sprop = after + (2 * NP + 1) * (K + 1) * kMcmcThreads + gblk * NS;
  int* sacc = (int*)(after + (2 * NP + 1) * (K + 1) * kMcmcThreads + GPB * NS) + gblk * NS;
  // per-group fibre state th, ph, v_x, v_y, v_z, theta prior and fraction prior (kFs* rows of K);
  // every lane of a group writes the same values, so each lane reads back what it wrote
  float* fst = after + (2 * NP + 1) * (K + 1) * kMcmcThreads + 2 * GPB * NS + gblk * kFsRows * K;
  auto fill_gb = [&](float4* dst, const float* bv, const float* bl, int first_l, int step) {
    for (int e = first_l; e < NP * TPV; e += step) {
      const int p = e / TPV, l = e % TPV;
      const int m0 = l + 2 * p * TPV, m1 = m0 + TPV;
      const float gx0 = m0 < M ? bv[m0] : 0.f, gy0 = m0 < M ? bv[M + m0] : 0.f, gz0 = m0 < M ? bv[2 * M + m0] : 0.f;
      const float b0 = m0 < M ? bl[m0] : 0.f;
      const float gx1 = m1 < M ? bv[m1] : 0.f, gy1 = m1 < M ? bv[M + m1] : 0.f, gz1 = m1 < M ? bv[2 * M + m1] : 0.f;
      const float b1 = m1 < M ? bl[m1] : 0.f;
      dst[e] = make_float4(gx0, gx1, gy0, gy1);
      dst[NP * TPV + e] = make_float4(gz0, gz1, b0, b1);
    }
    if (TAIL)
      for (int l = first_l; l < TPV; l += step) {
        const int m = l + (MPL - 1) * TPV;
        dst[2 * NP * TPV + l] =
            m < M ? make_float4(bv[m], bv[M + m], bv[2 * M + m], bl[m]) : make_float4(0.f, 0.f, 0.f, 0.f);
      }
  };
  if (!a.gradnonlin) {
    fill_gb(gb, a.bvecs, a.bvals, tid, blockDim.x);
    __syncthreads();
  }

  for (int round = 0;; ++round) {
    const int first = (warp_id + round * warps_total) * GPW;
    if (first >= a.nvox) break;
    const int vreal = first + gw;
    const bool valid = vreal < a.nvox;
    const int v = valid ? vreal : a.nvox - 1;
    const uint64_t gvox = a.voxel_keys ? a.voxel_keys[v] : a.voxel_offset + (uint64_t)v;
    if (a.gradnonlin) {
      __syncwarp();
      fill_gb(gb, a.bvecs + (size_t)v * 3 * M, a.bvals + (size_t)v * M, gl, TPV);
      __syncwarp();
    }

    // ---- this lane's measurements: pairs (y2, w2) and the unpaired one (yt, wt) ----
    float2 y2[NP], w2[NP], i2[NP], s2[K][NP];  // y2, w2: only until they are stored in shared memory
    float yt = 0.f, wt = 0.f, it_ = 0.f, st[K];
    bool bad = false;
    const float* yv = a.data + (size_t)v * M;
#pragma unroll
    for (int p = 0; p < NP; ++p) {
      const int m0 = gl + 2 * p * TPV, m1 = m0 + TPV;
      y2[p].x = m0 < M ? __ldg(yv + m0) : 0.f;
      y2[p].y = m1 < M ? __ldg(yv + m1) : 0.f;
      w2[p].x = m0 < M ? 1.f : 0.f;
      w2[p].y = m1 < M ? 1.f : 0.f;
      bad |= !isfinite(y2[p].x) || !isfinite(y2[p].y);
    }
    if (TAIL) {
      const int m = gl + (MPL - 1) * TPV;
      yt = m < M ? __ldg(yv + m) : 0.f;
      wt = m < M ? 1.f : 0.f;
      bad |= !isfinite(yt);
    }
    bad = group_sum<TPV>(bad ? 1.f : 0.f) > 0.f;
#pragma unroll
    for (int p = 0; p < NP; ++p) ywp[p * kMcmcThreads + tid] = make_float4(y2[p].x, y2[p].y, w2[p].x, w2[p].y);
    if (TAIL) ywt[tid] = make_float2(yt, wt);

    // ---- init_Fibres_Multifibres (CUDA/runmcmc_kernels.cu:255-504), or a saved chain state ----
    // (state_in rows as the records: d, f0, tau, d_std, R, S0, then th, ph, f per fibre)
    const bool from_state = STRETCH && a.state_in != nullptr;
    const float* prm = from_state ? nullptr : a.params + (size_t)v * a.np_fit;
    auto srow = [&](int r) { return a.state_in[(size_t)r * a.nvox + v]; };
    float S0, d, dstd = 0.f, R = 0.f, f0, tau;
    if (from_state) {
      S0 = srow(5);
      d = srow(0);
      if (MODEL >= 2) dstd = srow(3);
      if (MODEL == 3) R = srow(4);
      f0 = use_f0 ? srow(1) : 0.f;
      tau = RIC ? srow(2) : 0.f;
    } else {
      S0 = prm[0];
      d = prm[1];
      if (d < 0.f || d > kUpperDiff) d = 2e-3f;
      if (MODEL >= 2) {
        dstd = prm[2];
        const float upper = MODEL == 3 ? 0.004f : 0.01f;
        if (dstd < 0.f || dstd > upper) dstd = d / 10.f;
        R = MODEL == 3 ? a.R_mean : 0.f;
      }
      f0 = use_f0 ? prm[a.np_fit - 1] : 0.f;
      tau = (RIC && a.tau) ? a.tau[v] : 0.f;
    }
    constexpr int add = MODEL >= 2 ? 1 : 0;
    float f[K];
    uint32_t lam = 0;  // ARD flag of fibre k in bit k
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const float th0 = from_state ? srow(6 + 3 * k) : prm[2 + 3 * k + 1 + add];
      const float ph0 = from_state ? srow(7 + 3 * k) : prm[2 + 3 * k + 2 + add];
      f[k] = from_state ? srow(8 + 3 * k) : prm[2 + 3 * k + add];
      const bool lk = (k == 0) ? (a.all_ard != 0) : (a.no_ard == 0);
      lam |= lk ? 1u << k : 0u;
      float fp = 0.f;
      if (!(f[k] <= 0.f || f[k] >= 1.f)) fp = pr.fudge * (lk ? ln_approx(f[k]) : 0.f);
      float sn, cs, sp, cp;
      sincos_fast(th0, sn, cs);
      sincos_fast(ph0, sp, cp);
      fst[kFsTh * K + k] = th0;
      fst[kFsPh * K + k] = ph0;
      fst[kFsVx * K + k] = sn * cp;
      fst[kFsVy * K + k] = sn * sp;
      fst[kFsVz * K + k] = cs;
      fst[kFsPth * K + k] = th_prior(th0, sn);
      fst[kFsPf * K + k] = fp;
    }
    float p_d = 0.f, p_dstd = 0.f, p_R = 0.f, p_f0 = 0.f;
    if (MODEL == 3 && d >= 0.f && d <= kUpperDiff) p_d = (1.0f - 3.0f) * ln_approx(d) + 4000.0f * d;
    if (MODEL >= 2) {
      const float upper = MODEL == 3 ? 0.004f : 0.01f;
      if (dstd > 0.f && dstd <= upper) p_dstd = ln_approx(dstd);
      if (MODEL == 3) {
        float prr = 0.f;
        if (!r_prior(pr, R, d, prr)) p_R = prr;
      }
    }
    if (use_f0 && !(f0 <= 0.f || f0 >= 1.f) && a.ardf0) p_f0 = ln_approx(f0);

    // all signals of the state with signal parameters sp and directions v_k into s2/st/i2/it_,
    // backing up the overwritten ones when backup is true
    auto all_signals = [&](const SigParams<MODEL>& sp, bool sticks, bool isob, bool backup) {
      with_signal_form<MODEL>(sp, [&](auto form) {
        constexpr bool MONO = decltype(form)::value;
        const float2 beta2 = make_float2(sp.beta, sp.beta);
#pragma unroll
        for (int p = 0; p < NP; ++p) {
          const float4 ga = gb[p * TPV + gl], gc = gb[(NP + p) * TPV + gl];
          const float2 gx = make_float2(ga.x, ga.y), gy = make_float2(ga.z, ga.w), gz = make_float2(gc.x, gc.y);
          const float2 b = make_float2(gc.z, gc.w);
          const float2 bbeta = vmul(beta2, b);
          if (sticks) {
#pragma unroll
            for (int k = 0; k < K; ++k) {
              float2 dp = vmul(gx, vbc<float2>(fst[kFsVx * K + k]));
              dp = vfma(gy, vbc<float2>(fst[kFsVy * K + k]), dp);
              dp = vfma(gz, vbc<float2>(fst[kFsVz * K + k]), dp);
              if (backup) bkp[(k * NP + p) * kMcmcThreads] = s2[k][p];
              s2[k][p] = stick_v<MODEL, MONO, float2>(sp, b, bbeta, vmul(dp, dp));
            }
          }
          if (isob) {
            if (backup) bkp[(K * NP + p) * kMcmcThreads] = i2[p];
            i2[p] = iso_v<MODEL, MONO, float2>(sp, b, bbeta);
          }
        }
        if (TAIL) {
          const float4 g = gb[2 * NP * TPV + gl];
          const float bbeta = sp.beta * g.w;
          if (sticks) {
#pragma unroll
            for (int k = 0; k < K; ++k) {
              const float dp = g.x * fst[kFsVx * K + k] + g.y * fst[kFsVy * K + k] + g.z * fst[kFsVz * K + k];
              if (backup) bkt[k * kMcmcThreads] = st[k];
              st[k] = stick_v<MODEL, MONO, float>(sp, g.w, bbeta, dp * dp);
            }
          }
          if (isob) {
            if (backup) bkt[K * kMcmcThreads] = it_;
            it_ = iso_v<MODEL, MONO, float>(sp, g.w, bbeta);
          }
        }
      });
    };
    // the likelihood statistic of a state, summed over the group
    auto lik_of = [&](float S0x, const float (&fx)[K], float f0x, float taux) {
      float fsum = f0x;
#pragma unroll
      for (int k = 0; k < K; ++k) fsum += fx[k];
      const float wiso = 1.0f - fsum;
      float2 fk2[K];
#pragma unroll
      for (int k = 0; k < K; ++k) fk2[k] = vbc<float2>(fx[k]);
      const float2 nS02 = vbc<float2>(-S0x), f02 = vbc<float2>(f0x), wiso2 = vbc<float2>(wiso);
      float acc;
      if constexpr (RIC) {
        const float2 tS02 = vbc<float2>(taux * S0x);
        float2 rr = make_float2(0.f, 0.f), prod = make_float2(1.f, 1.f), zs = make_float2(0.f, 0.f);
        float lgp = 0.f;  // log2 of the products already closed (at most five factors per product)
#pragma unroll
        for (int p = 0; p < NP; ++p) {
          const float4 yw = ywp[p * kMcmcThreads + tid];
          float2 base = vfma(wiso2, i2[p], f02);
#pragma unroll
          for (int k = 0; k < K; ++k) base = vfma(fk2[k], s2[k][p], base);
          rician_acc<float2, (WPAD >= 2)>(make_float2(yw.x, yw.y), make_float2(yw.z, yw.w), base, nS02, tS02, rr, prod,
                                          zs);
          if (p % 4 == 3 && p + 1 < NP) {
            lgp += lg2_approx(prod.x) + lg2_approx(prod.y);
            prod = make_float2(1.f, 1.f);
          }
        }
        if (TAIL) {
          const float2 ytw = ywt[tid];
          float base = fmaf(wiso, it_, f0x);
#pragma unroll
          for (int k = 0; k < K; ++k) base = fmaf(fx[k], st[k], base);
          rician_acc<float, (WPAD >= 1)>(ytw.x, ytw.y, base, -S0x, taux * S0x, rr.x, prod.x, zs.x);
        }
        acc = -0.5f * taux * (rr.x + rr.y) + kLn2 * (lgp + lg2_approx(prod.x) + lg2_approx(prod.y)) - (zs.x + zs.y);
      } else {
        float2 acc2 = make_float2(0.f, 0.f);
#pragma unroll
        for (int p = 0; p < NP; ++p) {
          float2 sk[K];
#pragma unroll
          for (int k = 0; k < K; ++k) sk[k] = s2[k][p];
          const float4 yw = ywp[p * kMcmcThreads + tid];
          acc2 = vadd(acc2, gauss_v<K, float2, (WPAD >= 2)>(make_float2(yw.x, yw.y), make_float2(yw.z, yw.w), i2[p], sk,
                                                            nS02, fk2, f02, wiso2));
        }
        acc = vhsum(acc2);
        if (TAIL) {
          const float2 ytw = ywt[tid];
          acc += gauss_v<K, float, (WPAD >= 1)>(ytw.x, ytw.y, it_, st, -S0x, fx, f0x, wiso);
        }
      }
      return group_sum<TPV>(acc);
    };

    // signal parameters of the current state (changed only by accepted d, d_std or R proposals)
    SigParams<MODEL> spc = sig_params<MODEL>(d, dstd, R);
    all_signals(spc, true, true, false);
    float lik = lik_of(S0, f, f0, tau);
    // initialise_props (or widths given per voxel), acceptance counters
    if (gl == 0) {
#pragma unroll
      for (int q = 0; q < NS; ++q) {
        float pq = 0.2f;
        if (q == kSlotS0) pq = S0 / 10.f;
        if (q == kSlotD) pq = d / 10.f;
        if (q == kSlotDstd) pq = dstd / 10.f;
        if (q == kSlotTau) pq = tau / 2.f;
        if (q == kSlotR) pq = R / 10.f;
        if (a.props_in) pq = a.props_in[(size_t)q * a.nvox + v];
        sprop[q] = pq;
        sacc[q] = (STRETCH && a.acc_in) ? a.acc_in[(size_t)q * a.nvox + v] : 0;
      }
    }
    __syncwarp();

    // iterations [it_begin, it_end) of the chain; samples recorded before it_begin keep their slots
    const int it_begin = STRETCH ? a.it_begin : 0;
    const int it_end = (STRETCH && a.it_end > 0) ? a.it_end : total;
    int sample = it_begin > a.nburn ? min((it_begin - a.nburn) / a.sampleevery, ns) : 0;
    for (int it = it_begin; it < it_end; ++it) {
      // this iteration's randoms: lane gl holds slots gl, gl+TPV, ...
      float rn[NR], rl[NR];
#pragma unroll
      for (int q = 0; q < NR; ++q) {
        const int slot = gl + q * TPV;
        rn[q] = 0.f;
        rl[q] = 0.f;
        if (slot < NS) slot_randoms(a.seed, gvox, (uint32_t)it, (uint32_t)slot, rn[q], rl[q]);
      }
#pragma unroll 1
      for (int slot = 0; slot < NS; ++slot) {
        if (!((enabled >> slot) & 1u)) continue;
        float n, lu;
        {
          float rq = rn[0], lq = rl[0];
#pragma unroll
          for (int q = 1; q < NR; ++q)
            if (q == slot / TPV) {
              rq = rn[q];
              lq = rl[q];
            }
          n = __shfl_sync(0xffffffffu, rq, slot % TPV, TPV);
          lu = __shfl_sync(0xffffffffu, lq, slot % TPV, TPV);
        }
        const float prop = sprop[slot];
        // ---------- the proposal: state, prior, and the signals it changes (updated in place) ----------
        // kind 0: f0, tau, S0 or a fraction (likelihood only); 1: theta/phi of fibre kf (one stick);
        // 2: d, d_std or R (every signal that depends on it)
        const int kind = (int)((kSlotKinds >> (2 * slot)) & 3u);
        const int kf = (int)((kSlotFibres >> (2 * slot)) & 3u);
        const bool is_th = (kSlotTheta >> slot) & 1u;
        float S0n = S0, taun = tau, f0n = f0, fn[K];
#pragma unroll
        for (int k = 0; k < K; ++k) fn[k] = f[k];
        float pold = 0.f, pnew = 0.f, thn = 0.f, phn = 0.f, nvx = 0.f, nvy = 0.f, nvz = 0.f, dn = d, dsn = dstd, Rn = R;
        bool rej = false, sticks = false, isob = false;
        if (kind == 1) {
          const float tho = fst[kFsTh * K + kf], pho = fst[kFsPh * K + kf];
          thn = is_th ? tho + n * prop : tho;
          phn = is_th ? pho : pho + n * prop;
          float sn, cs, sp_, cp;
          sincos_fast(thn, sn, cs);
          sincos_fast(phn, sp_, cp);
          pold = is_th ? fst[kFsPth * K + kf] : 0.f;
          pnew = is_th ? th_prior(thn, sn) : 0.f;
          nvx = sn * cp;
          nvy = sn * sp_;
          nvz = cs;
          with_signal_form<MODEL>(spc, [&](auto form) {
            constexpr bool MONO = decltype(form)::value;
            const SigParams<MODEL>& sp = spc;
            const float2 beta2 = make_float2(sp.beta, sp.beta);
            const float2 nvx2 = vbc<float2>(nvx), nvy2 = vbc<float2>(nvy), nvz2 = vbc<float2>(nvz);
#pragma unroll
            for (int k = 0; k < K; ++k)
              if (k == kf) {
#pragma unroll
                for (int p = 0; p < NP; ++p) {
                  const float4 ga = gb[p * TPV + gl], gc = gb[(NP + p) * TPV + gl];
                  float2 dp = vmul(make_float2(ga.x, ga.y), nvx2);
                  dp = vfma(make_float2(ga.z, ga.w), nvy2, dp);
                  dp = vfma(make_float2(gc.x, gc.y), nvz2, dp);
                  const float2 b = make_float2(gc.z, gc.w);
                  bkp[p * kMcmcThreads] = s2[k][p];
                  s2[k][p] = stick_v<MODEL, MONO, float2>(sp, b, vmul(beta2, b), vmul(dp, dp));
                }
                if (TAIL) {
                  const float4 g = gb[2 * NP * TPV + gl];
                  const float dp = g.x * nvx + g.y * nvy + g.z * nvz;
                  bkt[0] = st[k];
                  st[k] = stick_v<MODEL, MONO, float>(sp, g.w, sp.beta * g.w, dp * dp);
                }
              }
          });
        } else if (kind == 2) {
          if (slot == kSlotD) {
            dn = d + n * prop;
            rej = (dn < 0.f || dn > kUpperDiff);
            pold = p_d;
            pnew = (rej || MODEL != 3) ? p_d : (1.0f - 3.0f) * ln_approx(dn) + 4000.0f * dn;
            sticks = true;
            isob = true;
          } else if (slot == kSlotDstd) {
            dsn = dstd + n * prop;
            const float upper = MODEL == 3 ? 0.004f : 0.01f;
            rej = (dsn <= 0.f || dsn > upper);
            pold = p_dstd;
            pnew = rej ? p_dstd : ln_approx(dsn);
            sticks = MODEL == 2;
            isob = true;
          } else {
            Rn = R + n * prop;
            float pr2 = p_R;
            rej = r_prior(pr, Rn, d, pr2);
            pold = p_R;
            pnew = rej ? p_R : pr2;
            sticks = true;
          }
          if (!group_all<TPV>(rej)) all_signals(sig_params<MODEL>(dn, dsn, Rn), sticks, isob, true);
        } else if (slot >= kSlotFibre0) {
          const float fkn = pick<K>(f, kf) + n * prop;
          rej = (fkn <= 0.f || fkn >= 1.f);
          const bool lj = (lam >> kf) & 1u;
          pold = fst[kFsPf * K + kf];
          pnew = rej ? pold : pr.fudge * ((pr.can_use_ard && lj) ? ln_approx(fkn) : 0.f);
          float fs = f0;
#pragma unroll
          for (int k = 0; k < K; ++k) {
            if (k == kf) fn[k] = fkn;
            fs += fn[k];
          }
          rej = rej || (fs > 1.f);
        } else if (slot == kSlotF0) {
          f0n = f0 + n * prop;
          rej = (f0n <= 0.f || f0n >= 1.f);
          pold = p_f0;
          pnew = rej ? p_f0 : (a.ardf0 ? ln_approx(f0n) : 0.f);
          float fs = f0n;
#pragma unroll
          for (int k = 0; k < K; ++k) fs += f[k];
          rej = rej || (fs > 1.f);
        } else if (slot == kSlotTau) {
          taun = tau + n * prop;
          rej = taun <= 0.f;
        } else {
          S0n = S0 + n * prop;
          rej = S0n < 0.f;
        }
        // ---------- likelihood of the proposed state and the decision (one body for every kind) ----------
        float likn = lik;
        const bool live = !group_all<TPV>(rej);
        if (live) likn = lik_of(S0n, fn, f0n, taun);
        const float dl = slot == kSlotTau ? dlik<RIC>(lik, likn, tau, taun, halfM, fM) : dlik_same_tau<RIC>(lik, likn, halfM);
        const bool ok = !rej && ((pold - pnew) + dl > lu);
        // ---------- restore the signals of a rejected proposal, or commit an accepted one ----------
        if (kind == 1) {
          if (!group_all<TPV>(ok)) {
#pragma unroll
            for (int k = 0; k < K; ++k)
              if (k == kf) {
#pragma unroll
                for (int p = 0; p < NP; ++p) s2[k][p] = keep_or_restore<TPV>(ok, s2[k][p], bkp[p * kMcmcThreads]);
                if (TAIL) st[k] = keep_or_restore<TPV>(ok, st[k], bkt[0]);
              }
          }
        } else if (kind == 2) {
          if (live && !group_all<TPV>(ok)) {
#pragma unroll
            for (int p = 0; p < NP; ++p) {
              if (sticks) {
#pragma unroll
                for (int k = 0; k < K; ++k)
                  s2[k][p] = keep_or_restore<TPV>(ok, s2[k][p], bkp[(k * NP + p) * kMcmcThreads]);
              }
              if (isob) i2[p] = keep_or_restore<TPV>(ok, i2[p], bkp[(K * NP + p) * kMcmcThreads]);
            }
            if (TAIL) {
              if (sticks) {
#pragma unroll
                for (int k = 0; k < K; ++k) st[k] = keep_or_restore<TPV>(ok, st[k], bkt[k * kMcmcThreads]);
              }
              if (isob) it_ = keep_or_restore<TPV>(ok, it_, bkt[K * kMcmcThreads]);
            }
          }
        }
        if (ok) {
          lik = likn;
          if (kind == 1) {
            fst[kFsTh * K + kf] = thn;
            fst[kFsPh * K + kf] = phn;
            fst[kFsVx * K + kf] = nvx;
            fst[kFsVy * K + kf] = nvy;
            fst[kFsVz * K + kf] = nvz;
            if (is_th) fst[kFsPth * K + kf] = pnew;
          } else if (kind == 2) {
            if (slot == kSlotD) {
              d = dn;
              p_d = pnew;
            } else if (slot == kSlotDstd) {
              dstd = dsn;
              p_dstd = pnew;
            } else {
              R = Rn;
              p_R = pnew;
            }
            spc = sig_params<MODEL>(d, dstd, R);
          } else if (slot >= kSlotFibre0) {
#pragma unroll
            for (int k = 0; k < K; ++k) f[k] = fn[k];
            fst[kFsPf * K + kf] = pnew;
          } else if (slot == kSlotF0) {
            f0 = f0n;
            p_f0 = pnew;
          } else if (slot == kSlotTau) {
            tau = taun;
          } else {
            S0 = S0n;
          }
          if (gl == 0) sacc[slot] += 1;
        }
      }
      // ---------------- record (CUDA/runmcmc_kernels.cu:1326-1339) ----------------
      if (it >= a.nburn && ((it - a.nburn + 1) % a.sampleevery) == 0 && sample < ns) {
        if (valid && gl == 0) {
          const size_t stride = (size_t)ns * a.nvox;
          float* r = a.records + (size_t)sample * a.nvox + v;
          r[0 * stride] = d;
          r[1 * stride] = f0;
          r[2 * stride] = tau;
          r[3 * stride] = dstd;
          r[4 * stride] = R;
          r[5 * stride] = S0;
#pragma unroll
          for (int k = 0; k < K; ++k) {
            r[(6 + 3 * k) * stride] = fst[kFsTh * K + k];
            r[(7 + 3 * k) * stride] = fst[kFsPh * K + k];
            r[(8 + 3 * k) * stride] = f[k];
          }
        }
        ++sample;
      }
      // ---------------- update_proposals (CUDA/runmcmc_kernels.cu:1341-1395) ----------------
      // each slot is proposed once per iteration, so since the last update acc + rej = upe
      const bool adapt = a.freeze_props == 0 || (a.freeze_props == 2 && it < a.nburn);
      if (adapt && ((it + 1) % a.upe) == 0) {
        __syncwarp();
        if (gl == 0) {
          const float upe = (float)a.upe;
#pragma unroll
          for (int q = 0; q < NS; ++q) {
            const bool on = (q == kSlotD) || (q == kSlotS0) || (q >= kSlotFibre0) || (q == kSlotTau && RIC) ||
                            (q == kSlotF0 && use_f0) || (q == kSlotDstd && MODEL >= 2) || (q == kSlotR && MODEL == 3);
            if (on) {
              const float acc = (float)sacc[q];
              sprop[q] = fminf(sprop[q] * sqrtf((acc + 1.0f) / (upe - acc + 1.0f)), kMaxProp);
            }
            sacc[q] = 0;
          }
        }
        __syncwarp();
      }
    }
    if (STRETCH && valid && gl == 0 && a.state_out) {
      const size_t n = a.nvox;
      float* so = a.state_out + v;
      so[0 * n] = d;
      so[1 * n] = f0;
      so[2 * n] = tau;
      so[3 * n] = dstd;
      so[4 * n] = R;
      so[5 * n] = S0;
#pragma unroll
      for (int k = 0; k < K; ++k) {
        so[(6 + 3 * k) * n] = fst[kFsTh * K + k];
        so[(7 + 3 * k) * n] = fst[kFsPh * K + k];
        so[(8 + 3 * k) * n] = f[k];
      }
    }
    if (STRETCH && valid && gl == 0 && a.acc_out) {
#pragma unroll
      for (int q = 0; q < NS; ++q) a.acc_out[(size_t)q * a.nvox + v] = sacc[q];
    }
    if (valid && gl == 0 && a.props_out) {
#pragma unroll
      for (int q = 0; q < NS; ++q) a.props_out[(size_t)q * a.nvox + v] = sprop[q];
    }
    if (valid && gl == 0 && a.status) {
      uint32_t stt = a.status[v];
      if (!isfinite(lik)) stt |= BPX_VOX_NONFINITE_ENERGY;
      if (bad) stt |= BPX_VOX_NONFINITE_DATA;
      a.status[v] = stt;
    }
    __syncwarp();
  }
}

// likelihood statistic of one state, summed over the group: SS (Gaussian) or
// sum_m [-tau (y-p)^2/2 + logI0(z) - z] (Rician, accumulated as the MCMC kernel does)
template <int MODEL, int K, bool RIC, int TPV, int MPL>
__device__ __forceinline__ float lik_stat(const Lanes<MODEL, K, RIC, TPV, MPL>& L, const float (&isoa)[MPL],
                                          const float (&sk)[K][MPL], float S0, const float (&f)[K],
                                          float f0, float tau) {
  float fsum = f0;
#pragma unroll
  for (int k = 0; k < K; ++k) fsum += f[k];
  const float wiso = 1.0f - fsum;
  float rr = 0.f, prod = 1.f, zs = 0.f, lgp = 0.f;
#pragma unroll
  for (int j = 0; j < MPL; ++j) {
    if (j < L.nj) {
      float base = fmaf(wiso, isoa[j], f0);
#pragma unroll
      for (int k = 0; k < K; ++k) base = fmaf(f[k], sk[k][j], base);
      if (!RIC) {
        const float r = fmaf(-S0, base, L.y[j]);
        rr = fmaf(r, r, rr);
      } else {
        rician_acc<float>(L.y[j], 1.0f, base, -S0, tau * S0, rr, prod, zs);
      }
    }
    if (RIC && j % 5 == 4) {
      lgp += lg2_approx(prod);
      prod = 1.f;
    }
  }
  if (!RIC) return group_sum<TPV>(rr);
  return group_sum<TPV>(-0.5f * tau * rr + kLn2 * (lgp + lg2_approx(prod)) - zs);
}

// Energies of given states (for the FP32-vs-FP64 likelihood check): one group per voxel.
template <int MODEL, int K, bool RIC, int TPV, int MPL>
__global__ void __launch_bounds__(kMcmcThreads) energy_kernel(EnergyArgs a) {
  constexpr int GPW = 32 / TPV;
  const int lane = threadIdx.x & 31;
  const int gl = lane % TPV;
  const int gw = lane / TPV;
  const int warps_total = gridDim.x * (blockDim.x >> 5);
  const int warp_id = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int M = a.ndir;
  for (int round = 0;; ++round) {
    const int first = (warp_id + round * warps_total) * GPW;
    if (first >= a.nvox) break;
    const int vreal = first + gw;
    const bool valid = vreal < a.nvox;
    const int v = valid ? vreal : a.nvox - 1;
    const float* st = a.states + (size_t)v * BPX_NSTATE;
    const float S0 = st[0], d = st[1], dstd = st[2], R = st[3], tau = st[4];
    const float f0 = a.f0 ? st[5] : 0.f;
    float f[K];
    Lanes<MODEL, K, RIC, TPV, MPL> L;
    const float* yv = a.data + (size_t)v * M;
    const float* bv = a.gradnonlin ? a.bvecs + (size_t)v * 3 * M : a.bvecs;
    const float* bl = a.gradnonlin ? a.bvals + (size_t)v * M : a.bvals;
    const SigParams<MODEL> sp = sig_params<MODEL>(d, dstd, R);
    L.nj = 0;
    float logy_part = 0.f;
#pragma unroll
    for (int j = 0; j < MPL; ++j) {
      const int m = gl + j * TPV;
      L.y[j] = m < M ? yv[m] : 0.f;
      L.b[j] = m < M ? bl[m] : 0.f;
      if (m < M) {
        L.nj = j + 1;
        if (RIC) logy_part += logf(L.y[j]);
      }
    }
#pragma unroll
    for (int k = 0; k < K; ++k) {
      f[k] = st[8 + 3 * k];
      float s_, c_, sp_, cp_;
      sincos_fast(st[6 + 3 * k], s_, c_);
      sincos_fast(st[7 + 3 * k], sp_, cp_);
#pragma unroll
      for (int j = 0; j < MPL; ++j) {
        const int m = gl + j * TPV;
        float dp = 0.f;
        if (m < M) dp = bv[m] * s_ * cp_ + bv[M + m] * s_ * sp_ + bv[2 * M + m] * c_;
        L.c[k][j] = dp * dp;
        L.s[k][j] = stick_signal<MODEL>(sp, L.b[j], L.c[k][j]);
      }
    }
#pragma unroll
    for (int j = 0; j < MPL; ++j) L.iso[j] = iso_signal<MODEL>(sp, L.b[j]);
    const float stat = lik_stat<MODEL, K, RIC, TPV, MPL>(L, L.iso, L.s, S0, f, f0, tau);
    float lik;
    if (!RIC)
      lik = 0.5f * (float)M * logf(stat / 2.0f);
    else
      lik = -(float)M * logf(tau) - (group_sum<TPV>(logy_part) + stat);
    // prior energy as init_Fibres_Multifibres_kernel composes it
    Priors pr;
    pr.fudge = a.fudge;
    pr.R_mean = a.R_mean;
    pr.R_std = a.R_std;
    pr.R_fudge = a.R_fudge;
    float p = 0.f;
    if (MODEL == 3 && d >= 0.f && d <= kUpperDiff) p += (1.0f - 3.0f) * ln_approx(d) + 4000.0f * d;
    if (MODEL >= 2) {
      const float upper = MODEL == 3 ? 0.004f : 0.01f;
      if (dstd > 0.f && dstd <= upper) p += ln_approx(dstd);
      if (MODEL == 3) {
        float prr = 0.f;
        if (!r_prior(pr, R, d, prr)) p += prr;
      }
    }
    if (a.f0 && !(f0 <= 0.f || f0 >= 1.f) && a.ardf0) p += ln_approx(f0);
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const bool lj = (k == 0) ? (a.all_ard != 0) : (a.no_ard == 0);
      float fp = 0.f;
      if (!(f[k] <= 0.f || f[k] >= 1.f)) fp = a.fudge * (lj ? ln_approx(f[k]) : 0.f);
      float sn_, cs_;
      sincos_fast(st[6 + 3 * k], sn_, cs_);
      p += th_prior(st[6 + 3 * k], sn_) + fp;
    }
    if (valid && gl == 0) {
      if (a.lik) a.lik[v] = lik;
      if (a.prior) a.prior[v] = p;
    }
  }
}

template <int MODEL, int K, bool RIC, int TPV, int MPL>
cudaError_t launch_mcmc_t(const McmcArgs& a, cudaStream_t s) {
  const bool stretch = a.it_begin != 0 || a.it_end != 0 || a.state_in || a.state_out || a.acc_in || a.acc_out;
  constexpr int NS = 6 + 3 * K, GPB = kMcmcThreads / TPV;
  constexpr int NP = MPL / 2;
  auto kern = stretch ? mcmc_kernel<MODEL, K, RIC, TPV, MPL, true> : mcmc_kernel<MODEL, K, RIC, TPV, MPL, false>;
  // the whole-brain layout with no padding in its pairs (M >= 256) or none at all (M = 288), the
  // whole chain: those residuals skip w
  if constexpr (TPV == 32 && MPL == 9) {
    if (!stretch && a.ndir == TPV * MPL)
      kern = mcmc_kernel<MODEL, K, RIC, TPV, MPL, false, 0>;
    else if (!stretch && a.ndir >= 2 * NP * TPV)
      kern = mcmc_kernel<MODEL, K, RIC, TPV, MPL, false, 1>;
  }
  const size_t smem = (size_t)(a.gradnonlin ? GPB : 1) * TPV * MPL * sizeof(float4) +
                      (size_t)NP * kMcmcThreads * sizeof(float4) + (size_t)kMcmcThreads * sizeof(float2) +
                      (size_t)(2 * NP + 1) * (K + 1) * kMcmcThreads * sizeof(float) + (size_t)GPB * NS * 8 +
                      (size_t)GPB * kFsRows * K * sizeof(float);
  if (smem > 48 * 1024) {
    cudaError_t ea = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (ea != cudaSuccess) return ea;
  }
  int per_sm = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kMcmcThreads, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) per_sm = 1;
  const int vox_per_block = (kMcmcThreads / 32) * (32 / TPV);
  int grid = (a.nvox + vox_per_block - 1) / vox_per_block;
  const int cap = sm_count() * per_sm;
  if (grid > cap) grid = cap;
  if (grid < 1) grid = 1;
  kern<<<grid, kMcmcThreads, smem, s>>>(a);
  return cudaGetLastError();
}

template <int MODEL, int K, bool RIC, int TPV, int MPL>
cudaError_t launch_energy_t(const EnergyArgs& a, cudaStream_t s) {
  const int vox_per_block = (kMcmcThreads / 32) * (32 / TPV);
  int grid = (a.nvox + vox_per_block - 1) / vox_per_block;
  const int cap = sm_count() * 8;
  if (grid > cap) grid = cap;
  if (grid < 1) grid = 1;
  energy_kernel<MODEL, K, RIC, TPV, MPL><<<grid, kMcmcThreads, 0, s>>>(a);
  return cudaGetLastError();
}

// Layouts compiled for every (model, K, rician): (TPV, MPL) with capacity TPV*MPL.
#define BPX_LAYOUTS(X) X(4, 9) X(8, 8) X(8, 9) X(16, 9) X(32, 9) X(32, 16)

template <int MODEL>
cudaError_t launch_mcmc_model(const McmcArgs& a, int nfib, bool ric, McmcLayout lay, cudaStream_t s) {
#define BPX_TRY(T, P)                                                              \
  if (lay.tpv == T && lay.mpl == P) {                                              \
    if (nfib == 1) return ric ? launch_mcmc_t<MODEL, 1, true, T, P>(a, s) : launch_mcmc_t<MODEL, 1, false, T, P>(a, s); \
    if (nfib == 2) return ric ? launch_mcmc_t<MODEL, 2, true, T, P>(a, s) : launch_mcmc_t<MODEL, 2, false, T, P>(a, s); \
    if (nfib == 3) return ric ? launch_mcmc_t<MODEL, 3, true, T, P>(a, s) : launch_mcmc_t<MODEL, 3, false, T, P>(a, s); \
  }
  BPX_LAYOUTS(BPX_TRY)
#undef BPX_TRY
  return cudaErrorInvalidValue;
}

template <int MODEL>
cudaError_t launch_energy_model(const EnergyArgs& a, int nfib, bool ric, McmcLayout lay, cudaStream_t s) {
#define BPX_TRY(T, P)                                                              \
  if (lay.tpv == T && lay.mpl == P) {                                              \
    if (nfib == 1) return ric ? launch_energy_t<MODEL, 1, true, T, P>(a, s) : launch_energy_t<MODEL, 1, false, T, P>(a, s); \
    if (nfib == 2) return ric ? launch_energy_t<MODEL, 2, true, T, P>(a, s) : launch_energy_t<MODEL, 2, false, T, P>(a, s); \
    if (nfib == 3) return ric ? launch_energy_t<MODEL, 3, true, T, P>(a, s) : launch_energy_t<MODEL, 3, false, T, P>(a, s); \
  }
  BPX_LAYOUTS(BPX_TRY)
#undef BPX_TRY
  return cudaErrorInvalidValue;
}

}  // namespace bpx
