// bpx_gemm.h -- launch descriptor of the tcgen05 BF16 GEMM (bpx_gemm.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace bpx {
namespace gemm {

enum Epi : int {
  kEpiStoreF32 = 0,  // out_f32[m][n] = D
  kEpiBias = 1,      // out_f32[m][n] = D + bias[n]
  kEpiBiasGelu = 2,  // z = D + bias[n]; out_bf16 = gelu(z); out_f32 = z when given
  kEpiGeluGrad = 3,  // out_bf16 = D * gelu'(zin[m][n])
};

struct GemmOperands {
  const uint16_t* a;  // bf16, row-major: [M][lda] (K-major) or [K][lda] (MN-major)
  const uint16_t* b;  // bf16, row-major: [N][ldb] (K-major) or [K][ldb] (MN-major)
  int lda, ldb;
};

struct GemmArgs {
  int M, N, K;
  int ntile;       // output columns per CTA: 32, 64, 128 or 256
  int a_mn, b_mn;  // operand orientation: 0 = K-major, 1 = MN-major
  int epi;
  float* out_f32;
  int ld_out;
  uint16_t* out_bf16;
  int ld_bf16;
  const float* bias;
  const float* zin;
  int ld_zin;
  int* error;  // set to nonzero when a bounded wait gave up
};

// Validates the arguments (why = reason on failure) and launches on stream s.
cudaError_t launch(const GemmOperands& op, const GemmArgs& g, cudaStream_t s, const char** why);

}  // namespace gemm
}  // namespace bpx
