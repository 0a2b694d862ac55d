// bpx_synth.cu -- voxels drawn from the forward model on the GPU: the training set of the learned
// initialiser.  No counterpart in the reference.
//
// Per voxel (Philox-4x32-10 keyed by the seed, counter (voxel, block, stream tag)):
//   S0 = 1000; d ~ U(0.5e-3, 2e-3); d_std = U(0.1, 0.5) d (model 2); f1 ~ U(0.3, 0.7);
//   f2 = U(0,1) min(0.3, 1 - f1); f3 = U(0,1) min(0.15, max(0, 0.99 - f1 - f2));
//   fibre directions uniform on the sphere; SNR ~ U(snr_lo, snr_hi), sigma = S0 / SNR;
//   y = |S + sigma (n1 + i n2)| with the model-1 (ball and sticks) or model-2 (gamma-distributed
//   diffusivity) signal S.  The same distributions as the host generator fdt_b200/synth.py.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "bpx.h"
#include "bpx_device.cuh"
#include "bpx_internal.h"

namespace bpx {
namespace {

__device__ __forceinline__ float u24(uint32_t r) { return (float)((r >> 8) + 1u) * (1.0f / 16777216.0f); }

__device__ __forceinline__ uint4 draw(uint64_t seed, uint64_t vox, uint32_t block, uint32_t tag) {
  return philox4x32_10(make_uint4((uint32_t)vox, (uint32_t)(vox >> 32), block, tag),
                       make_uint2((uint32_t)seed, (uint32_t)(seed >> 32)));
}

// four standard normals from one Philox block (Box-Muller on two pairs of 24-bit uniforms)
__device__ __forceinline__ float4 normals4(uint4 r) {
  const float a = sqrtf(-2.f * logf(u24(r.x))), b = sqrtf(-2.f * logf(u24(r.z)));
  float s1, c1, s2, c2;
  sincospif(2.f * u24(r.y), &s1, &c1);
  sincospif(2.f * u24(r.w), &s2, &c2);
  return make_float4(a * c1, a * s1, b * c2, b * s2);
}

__global__ void synth_kernel(int model, int nfib, int nvox, int ndir, uint64_t seed, uint64_t voxel_offset,
                             float snr_lo, float snr_hi, const float* __restrict__ bvecs,
                             const float* __restrict__ bvals, float* __restrict__ data, float* __restrict__ truth) {
  const int lane = threadIdx.x & 31;
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int v = w; v < nvox; v += nwarps) {
    const uint64_t gv = voxel_offset + (uint64_t)v;
    const uint4 r0 = draw(seed, gv, 0, 0x7159u), r1 = draw(seed, gv, 1, 0x7159u);
    const float S0 = 1000.f;
    const float d = 0.5e-3f + 1.5e-3f * u24(r0.x);
    const float dstd = model >= 2 ? (0.1f + 0.4f * u24(r0.y)) * d : 0.f;
    float f[3] = {0.f, 0.f, 0.f};
    f[0] = 0.3f + 0.4f * u24(r0.z);
    if (nfib > 1) f[1] = u24(r0.w) * fminf(0.3f, 1.f - f[0]);
    if (nfib > 2) f[2] = u24(r1.x) * fminf(0.15f, fmaxf(0.f, 0.99f - f[0] - f[1]));
    const float snr = snr_lo + (snr_hi - snr_lo) * u24(r1.y);
    const float sigma = S0 / snr;
    float vx[3], vy[3], vz[3], th[3], ph[3];
    for (int k = 0; k < 3; ++k) {
      const float4 n = normals4(draw(seed, gv, 2 + k, 0x7159u));
      const float nn = sqrtf(n.x * n.x + n.y * n.y + n.z * n.z);
      vx[k] = n.x / nn;
      vy[k] = n.y / nn;
      vz[k] = n.z / nn;
      th[k] = acosf(fminf(fmaxf(vz[k], -1.f), 1.f));
      ph[k] = atan2f(vy[k], vx[k]);
    }
    float fsum = 0.f;
    for (int k = 0; k < nfib; ++k) fsum += f[k];
    const float alpha = model >= 2 ? d * d / (dstd * dstd) : 0.f, beta = model >= 2 ? dstd * dstd / d : 0.f;
    for (int m0 = 0; m0 < ndir; m0 += 64) {
      // lane handles measurements m0+2*lane and m0+2*lane+1 with one Philox block of noise
      const float4 n = normals4(draw(seed, gv, 8 + (uint32_t)(m0 / 2 + lane), 0x5e1du));
      for (int h = 0; h < 2; ++h) {
        const int m = m0 + 2 * lane + h;
        if (m >= ndir) break;
        const float gx = bvecs[m], gy = bvecs[ndir + m], gz = bvecs[2 * ndir + m], b = bvals[m];
        const float iso = model >= 2 ? expf(-alpha * log1pf(beta * b)) : expf(-b * d);
        float s = (1.f - fsum) * iso;
        for (int k = 0; k < nfib; ++k) {
          const float dp = gx * vx[k] + gy * vy[k] + gz * vz[k];
          const float c = dp * dp;
          s += f[k] * (model >= 2 ? expf(-alpha * log1pf(beta * b * c)) : expf(-b * d * c));
        }
        s *= S0;
        const float n1 = h ? n.z : n.x, n2 = h ? n.w : n.y;
        const float re = s + sigma * n1, im = sigma * n2;
        data[(size_t)v * ndir + m] = sqrtf(re * re + im * im);
      }
    }
    if (truth && lane == 0) {
      float* t = truth + (size_t)v * BPX_NSTATE;
      t[0] = S0;
      t[1] = d;
      t[2] = dstd;
      t[3] = 0.f;
      t[4] = 1.f / (sigma * sigma);
      t[5] = 0.f;
      for (int k = 0; k < 3; ++k) {
        t[6 + 3 * k] = k < nfib ? th[k] : 0.f;
        t[7 + 3 * k] = k < nfib ? ph[k] : 0.f;
        t[8 + 3 * k] = k < nfib ? f[k] : 0.f;
      }
    }
  }
}

}  // namespace
}  // namespace bpx

extern "C" bpx_status bpx_synth_dev(int32_t model, int32_t nfib, int32_t nvox, int32_t ndir, uint64_t seed,
                                    uint64_t voxel_offset, float snr_lo, float snr_hi, const float* bvecs,
                                    const float* bvals, float* data, float* truth, void* stream) {
  using namespace bpx;
  if (model < 1 || model > 2 || nfib < 1 || nfib > 3 || nvox < 0 || ndir < 1 || !(snr_lo > 0.f) ||
      !(snr_hi >= snr_lo) || (nvox > 0 && (!bvecs || !bvals || !data)))
    return api_fail(BPX_ERR_INVALID_ARG, "bpx_synth_dev: bad arguments");
  if (nvox == 0) return BPX_OK;
  bpx_status st = api_check_device();
  if (st != BPX_OK) return st;
  const int blocks = (int)std::min<long long>(((long long)nvox + 7) / 8, (long long)sm_count() * 32);
  synth_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(model, nfib, nvox, ndir, seed, voxel_offset, snr_lo, snr_hi,
                                                          bvecs, bvals, data, truth);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return api_cuda_fail(e, "synth_kernel");
  return BPX_OK;
}
