// bpx_device.cuh -- device helpers shared by the fit, MCMC and finishing kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "bpx.h"

namespace bpx {

constexpr float kTwoPiGpu = 0.636619772f;  // CUDA/diffmodels_utils.h:13 (2/pi as the reference writes it)
constexpr double kTwoPiGpuD = 0.636619772;
constexpr float kFSmall = 0.001f;           // CUDA/diffmodels_utils.h:16
constexpr float kUpperDiff = 0.005f;        // CUDA/runmcmc_kernels.cu:24
constexpr float kMaxProp = 1e10f;           // CUDA/runmcmc_kernels.cu:23

// Proposal slots of one MCMC iteration.  Each (voxel, iteration, slot) owns one Philox block,
// so a slot's random numbers do not depend on which other proposals are enabled.
enum Slot : uint32_t {
  kSlotF0 = 0,
  kSlotTau = 1,
  kSlotD = 2,
  kSlotDstd = 3,
  kSlotR = 4,
  kSlotS0 = 5,
  kSlotFibre0 = 6  // th_k = 6+3k, ph_k = 7+3k, f_k = 8+3k
};

// ---- Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, SC11) ----
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t lo0 = 0xD2511F53u * c.x;
    const uint32_t hi0 = __umulhi(0xD2511F53u, c.x);
    const uint32_t lo1 = 0xCD9E8D57u * c.z;
    const uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z);
    c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
    k.x += 0x9E3779B9u;
    k.y += 0xBB67AE85u;
  }
  return c;
}

// MUFU-based fast transcendentals (single instruction each).
__device__ __forceinline__ float ex2_approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float lg2_approx(float x) {
  float y;
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float rsqrt_approx(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float rcp_approx(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

constexpr float kLog2e = 1.4426950408889634f;
constexpr float kLn2 = 0.6931471805599453f;

// Random numbers of one proposal slot: a standard normal (Box-Muller on two 24-bit uniforms)
// and ln(u) of the acceptance uniform u in (0,1].  The same 24-bit uniforms are exact in the
// FP64 oracle, which therefore draws the same numbers.
__device__ __forceinline__ void slot_randoms(uint64_t seed, uint64_t vox, uint32_t it,
                                             uint32_t slot, float& normal, float& log_u) {
  const uint4 r = philox4x32_10(make_uint4(it, slot, (uint32_t)vox, (uint32_t)(vox >> 32)),
                                make_uint2((uint32_t)seed, (uint32_t)(seed >> 32)));
  const float u0 = (float)((r.x >> 8) + 1u) * (1.0f / 16777216.0f);
  const float u1 = (float)(r.y >> 8) * (1.0f / 16777216.0f);
  const float u2 = (float)((r.z >> 8) + 1u) * (1.0f / 16777216.0f);
  float s, c;
  sincospif(2.0f * u1, &s, &c);
  normal = sqrtf(-2.0f * logf(u0)) * c;
  log_u = logf(u2);
}

// Butterfly sum over aligned groups of G lanes (G a power of two <= 32).  Every lane of the
// group ends with the same value (each pairwise add is commutative).
template <int G>
__device__ __forceinline__ float group_sum(float x) {
#pragma unroll
  for (int o = G / 2; o >= 1; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}
template <int G>
__device__ __forceinline__ double group_sum(double x) {
#pragma unroll
  for (int o = G / 2; o >= 1; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}
template <int G>
__device__ __forceinline__ float group_max(float x) {
#pragma unroll
  for (int o = G / 2; o >= 1; o >>= 1) x = fmaxf(x, __shfl_xor_sync(0xffffffffu, x, o));
  return x;
}
template <int G>
__device__ __forceinline__ float group_min(float x) {
#pragma unroll
  for (int o = G / 2; o >= 1; o >>= 1) x = fminf(x, __shfl_xor_sync(0xffffffffu, x, o));
  return x;
}

// transforms of CUDA/diffmodels_utils.h:19-41
__device__ __forceinline__ float x2f(float x) { return fabsf(kTwoPiGpu * atanf(x)); }
__device__ __forceinline__ float f2x(float f) { return tanf(f / kTwoPiGpu); }
__device__ __forceinline__ float beta2f(float b) {
  const float s = sinf(b);
  return s * s;
}
__device__ __forceinline__ float f2beta(float f) { return asinf(sqrtf(f)); }
__device__ __forceinline__ float sgnf(float x) { return x > 0.f ? 1.f : (x < 0.f ? -1.f : 0.f); }
__device__ __forceinline__ float pm1(float x) { return x > 0.f ? 1.f : -1.f; }

// log of the modified Bessel function I0 minus its argument, for z >= 0: the polynomial forms of
// fibre.h:31-51 / CUDA/runmcmc_kernels.cu:126-145 (Abramowitz & Stegun 9.8.1, 9.8.2), written as
// logI0(z) - z so that the Rician log-likelihood terms stay O(1).  Branch-free: both polynomials
// are evaluated and one log2 is taken of the selected one (measurements of one warp fall on
// both sides of z = 3.75, so a branch would run both sides anyway).
__device__ __forceinline__ float logI0_minus_z(float z) {
  const bool small = z < 3.75f;
  float a = z * (1.0f / 3.75f);
  a *= a;
  const float q =
      1.0f + a * (3.5156229f + a * (3.0899424f + a * (1.2067492f + a * (0.2659732f + a * (0.0360768f + a * 0.0045813f)))));
  const float rs = rsqrt_approx(fmaxf(z, 3.75f));
  const float c = 3.75f * rs * rs;
  const float p =
      0.39894228f + c * (0.01328592f + c * (0.00225319f + c * (-0.00157565f + c * (0.00916281f + c * (-0.02057706f + c * (0.02635537f + c * (-0.01647633f + c * 0.00392377f)))))));
  const float l = lg2_approx(small ? q : p * rs) * kLn2;
  return small ? l - z : l;
}

}  // namespace bpx
