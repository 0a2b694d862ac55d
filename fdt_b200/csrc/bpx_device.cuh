// bpx_device.cuh -- device helpers shared by the fit, MCMC and finishing kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "bpx.h"

namespace bpx {

constexpr double kTwoPiGpuD = 0.636619772;  // CUDA/diffmodels_utils.h:13 (2/pi as the reference writes it)
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

constexpr float kLog2e = 1.4426950408889634f;
constexpr float kLn2 = 0.6931471805599453f;

// ln(x) from the MUFU log2 (absolute error about 1e-7): the chain's prior energies.
__device__ __forceinline__ float ln_approx(float x) { return kLn2 * lg2_approx(x); }

// Polynomial coefficients fitted for this library to the exact functions (fdt_b200/polyfit.py):
// I0(z) in powers of z^2 below kI0Split, e^-z I0(z) sqrt(z) in powers of 1/z above it, and sin/cos
// on [-pi/4, pi/4] (relative minimax for sin, absolute for cos, below 4e-9 before FP32 rounding).
// BEGIN generated by python -m fdt_b200.polyfit
constexpr float kI0Split = 4.75f;
__host__ __device__ constexpr float kI0Small(int i) { return i == 0 ? 1.0f : i == 1 ? 0.24999896f : i == 2 ? 0.015626252f : i == 3 ? 0.00043356538f : i == 4 ? 6.8553645e-06f : i == 5 ? 6.218488e-08f : 6.707401e-10f; }
__host__ __device__ constexpr float kI0Large(int i) { return i == 0 ? 0.39894244f : i == 1 ? 0.04983106f : i == 2 ? 0.029434934f : i == 3 ? 0.0128485765f : i == 4 ? 0.096278094f : 0.20845851f; }
__host__ __device__ constexpr float kSinQ(int i) { return i == 0 ? -0.16666655f : i == 1 ? 0.008332156f : -0.00019514632f; }
__host__ __device__ constexpr float kCosQ(int i) { return i == 0 ? 0.041666646f : i == 1 ? -0.0013887362f : 2.443773e-05f; }
// END generated

// sin and cos of r for |r| <= pi/4 (slightly beyond)
__device__ __forceinline__ void sincos_quarter(float r, float& s, float& c) {
  const float u = r * r;
  float p = fmaf(u, kSinQ(2), kSinQ(1));
  p = fmaf(u, p, kSinQ(0));
  s = fmaf(r * u, p, r);
  float q = fmaf(u, kCosQ(2), kCosQ(1));
  q = fmaf(u, q, kCosQ(0));
  q = fmaf(u, q, -0.5f);
  c = fmaf(u, q, 1.0f);
}

// Quadrant q (mod 4) of a reduced argument: sin and cos of r + q pi/2.
__device__ __forceinline__ void sincos_rotate(int q, float s, float c, float& sn, float& cs) {
  const bool sw = (q & 1) != 0;
  const float a = sw ? c : s, b = sw ? s : c;
  sn = __int_as_float(__float_as_int(a) ^ ((q & 2) << 30));
  cs = __int_as_float(__float_as_int(b) ^ (((q + 1) & 2) << 30));
}

// sin and cos of x in radians, within 2 ulp for |x| < 1e5: Cody-Waite reduction by pi/2 in three
// FMA steps (Cody and Waite, Software Manual for the Elementary Functions, 1980), then
// sincos_quarter.  pi/2 = 1.57079637f - 4.37113883e-08f - 1.71512451e-15f (to 1e-23).
__device__ __forceinline__ void sincos_fast(float x, float& sn, float& cs) {
  const float k = rintf(x * 0.636619772f);
  float r = fmaf(-k, 1.57079637f, x);
  r = fmaf(-k, -4.37113883e-08f, r);
  r = fmaf(-k, -1.71512451e-15f, r);
  float s, c;
  sincos_quarter(r, s, c);
  sincos_rotate((int)k, s, c, sn, cs);
}

// cos(2 pi u) for u = m 2^-24 in [0, 1): 4u - k is exact, so the reduction adds no error.
__device__ __forceinline__ float cos_2pi_u24(float u) {
  const float x4 = 4.0f * u;
  const float k = rintf(x4);
  float s, c, sn, cs;
  sincos_quarter((x4 - k) * 1.57079637f, s, c);
  sincos_rotate((int)k, s, c, sn, cs);
  return cs;
}

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
  normal = sqrtf(-2.0f * logf(u0)) * cos_2pi_u24(u1);
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

}  // namespace bpx
