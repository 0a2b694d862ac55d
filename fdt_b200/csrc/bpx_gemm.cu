// bpx_gemm.cu -- BF16 GEMM on the 5th-generation tensor cores (tcgen05), FP32 accumulation in
// tensor memory, with the fused epilogues of the learned initialiser's network.  No counterpart in
// the reference (xfibres_gpu has no learned part).
//
//   D[M][N] = sum_k A(m,k) B(n,k)      A, B bf16; D fp32 in TMEM
//
// Operands are read by TMA straight from row-major global tensors in either orientation:
//   * K-major  (the contraction index is the contiguous one): A = X[M][K], B = W[N][K];
//   * MN-major (M resp. N is the contiguous one): A stored [K][M], B stored [K][N].
// Both land in shared memory in the non-swizzled canonical layout of 8x(16 B) core matrices.  A
// rank-3 tensor map over the row-major tensor, {8 contiguous elements, row, group of 8 columns}
// with strides {row pitch, 16 B}, makes one TMA copy write a whole tile in that layout:
//   K-major tile  [K/8 groups][rows][8]  -> LBO (K direction) = rows*16 B, SBO (rows) = 128 B
//   MN-major tile [MN/8 groups][K][8]    -> LBO (K direction) = 128 B,    SBO (MN)   = K*16 B
// One thread issues TMA and MMA (M = 128, N = tile width <= 256, K = 16 per instruction) through
// a two-stage mbarrier ring; four warps then read their 32 TMEM lanes each (tcgen05.ld) and run
// the epilogue.  Every mbarrier wait is bounded (about a second), after which the kernel records
// an error code, waits (bounded) for its own MMAs and releases its tensor memory.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <mutex>

#include "bpx_gemm.h"
#include "bpx_internal.h"

namespace bpx {
namespace gemm {

constexpr int kTileM = 128;
constexpr int kChunkK = 64;
constexpr int kThreads = 128;
constexpr long long kWaitCycles = 2000000000ll;  // ~1 s at 2 GHz
// epilogue staging per warp: a 32 x 32 fp32 block (rows padded to 36 floats) and a 32 x 32 bf16
// block (rows padded to 80 bytes); both pitches keep 16-byte alignment and spread a quarter-warp's
// 16-byte accesses over distinct banks
constexpr int kPitchF = 36;
constexpr int kPitchB = 80;
constexpr int kEpiWarpBytes = 32 * kPitchF * 4 + 32 * kPitchB;
static_assert((kThreads / 32) * kEpiWarpBytes <= 2 * kTileM * kChunkK * 2, "epilogue tiles must fit the A stages");
static_assert(kEpiWarpBytes % 16 == 0 && (32 * kPitchF * 4) % 16 == 0, "epilogue tiles must stay 16-byte aligned");

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  const long long t0 = clock64();
  while (true) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    if (ok) return true;
    if (clock64() - t0 > kWaitCycles) return false;
  }
}

__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2,
                                            uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
      :
      : "r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(bar)
      : "memory");
}

// shared-memory matrix descriptor: no swizzle, Blackwell descriptor version 1
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\ttcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
      :
      : "r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" : : "r"(bar) : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
}

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z) {
  return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

__device__ __forceinline__ uint16_t to_bf16(float x) {
  return __bfloat16_as_ushort(__float2bfloat16_rn(x));
}

struct Smem {
  float bias[256];  // the tile's bias columns, staged once for the epilogue (16-byte aligned)
  uint64_t full[2], empty[2], done;
  uint32_t tmem_base;
};

__global__ void __launch_bounds__(kThreads, 1)
    gemm_kernel(const __grid_constant__ CUtensorMap map_a, const __grid_constant__ CUtensorMap map_b, GemmArgs g) {
  extern __shared__ __align__(1024) unsigned char dsmem[];
  unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(dsmem) + 1023) & ~uintptr_t(1023));
  const int nt = g.ntile;
  const uint32_t a_bytes = kTileM * kChunkK * 2, b_bytes = (uint32_t)nt * kChunkK * 2;
  const uint32_t stage_bytes = a_bytes + b_bytes;
  Smem* sm = reinterpret_cast<Smem*>(base + 2 * stage_bytes);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * kTileM, n0 = blockIdx.y * nt;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" : : "r"(smem_u32(&sm->tmem_base)), "r"(nt));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (threadIdx.x == 0) {
    for (int s = 0; s < 2; ++s) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" : : "r"(smem_u32(&sm->full[s])));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" : : "r"(smem_u32(&sm->empty[s])));
    }
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" : : "r"(smem_u32(&sm->done)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = sm->tmem_base;

  if (threadIdx.x == 0) {
    const int nk = (g.K + kChunkK - 1) / kChunkK;
    const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)g.a_mn << 15) | ((uint32_t)g.b_mn << 16) |
                           ((uint32_t)(nt >> 3) << 17) | ((uint32_t)(kTileM >> 4) << 24);
    auto load = [&](int kc) {
      const int s = kc & 1;
      const uint32_t sa = smem_u32(base + s * stage_bytes), sb = sa + a_bytes;
      const uint32_t bar = smem_u32(&sm->full[s]);
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" : : "r"(bar), "r"(stage_bytes) : "memory");
      if (g.a_mn)
        tma_load_3d(sa, &map_a, 0, kc * kChunkK, m0 / 8, bar);
      else
        tma_load_3d(sa, &map_a, 0, m0, kc * (kChunkK / 8), bar);
      if (g.b_mn)
        tma_load_3d(sb, &map_b, 0, kc * kChunkK, n0 / 8, bar);
      else
        tma_load_3d(sb, &map_b, 0, n0, kc * (kChunkK / 8), bar);
    };
    bool ok = true;
    for (int kc = 0; kc < 2 && kc < nk; ++kc) load(kc);
    for (int kc = 0; kc < nk && ok; ++kc) {
      const int s = kc & 1;
      const uint32_t ph = (kc >> 1) & 1;
      if (!mbar_wait(smem_u32(&sm->full[s]), ph)) {
        ok = false;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t sa = smem_u32(base + s * stage_bytes), sb = sa + a_bytes;
#pragma unroll
      for (int ks = 0; ks < kChunkK / 16; ++ks) {
        const uint64_t da = g.a_mn ? smem_desc(sa + ks * 256, 128, kChunkK * 16)
                                   : smem_desc(sa + ks * 2 * kTileM * 16, kTileM * 16, 128);
        const uint64_t db = g.b_mn ? smem_desc(sb + ks * 256, 128, kChunkK * 16)
                                   : smem_desc(sb + ks * 2 * nt * 16, nt * 16, 128);
        mma_bf16(tmem, da, db, idesc, (kc | ks) != 0);
      }
      mma_commit(smem_u32(&sm->empty[s]));
      if (kc + 2 < nk) {
        if (!mbar_wait(smem_u32(&sm->empty[s]), ph)) {
          ok = false;
          break;
        }
        load(kc + 2);
      }
    }
    if (!ok && g.error) atomicExch(g.error, 1);
    mma_commit(smem_u32(&sm->done));  // arrives once every MMA issued above has completed
  }
  __syncwarp();
  const bool done = mbar_wait(smem_u32(&sm->done), 0);
  if (!done && g.error) atomicExch(g.error, 2);
  // every lane of a warp adds the same bias columns: stage them in shared memory once, so the
  // epilogue reads them as broadcast 16-byte loads instead of 32 global loads per column chunk
  const bool use_bias = g.bias && (g.epi == kEpiBias || g.epi == kEpiBiasGelu);
  if (use_bias)
    for (int t = threadIdx.x; t < nt; t += kThreads) sm->bias[t] = n0 + t < g.N ? g.bias[n0 + t] : 0.f;
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

  // epilogue: warp w owns accumulator rows 32w..32w+31 (TMEM lanes), 32 columns at a time.  A lane
  // holds one row of a 32x32 block, so it is turned around through a per-warp shared-memory tile:
  // lanes write their rows, then read the block back so that consecutive lanes cover consecutive
  // columns of a row, and the global stores (and the GELU-derivative's loads of z) are whole
  // 128-byte lines instead of 32 rows touched per instruction.  The tiles reuse the operand stages,
  // idle once every MMA has completed (the done barrier above).
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  float* tf = reinterpret_cast<float*>(base + warp * kEpiWarpBytes);  // [32][kPitchF] fp32 block
  unsigned char* tb = base + warp * kEpiWarpBytes + 32 * kPitchF * 4;  // [32][kPitchB] bytes, bf16 block
  const bool all_done = __all_sync(0xffffffffu, done);
  const int row0 = m0 + 32 * warp;
  auto aligned16 = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; };
  // the block's 32 rows x 32 fp32 columns, lane = row, to out (row-major, leading dimension ld)
  auto put_f32 = [&](const float (&v)[32], float* out, int ld, int col0) {
    float4* t4 = reinterpret_cast<float4*>(tf + lane * kPitchF);
#pragma unroll
    for (int q = 0; q < 8; ++q) t4[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
    __syncwarp();
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int r = 4 * i + (lane >> 3), q = lane & 7;
      const int grow = row0 + r, gcol = col0 + 4 * q;
      const float4 x = reinterpret_cast<const float4*>(tf + r * kPitchF)[q];
      if (grow < g.M && gcol < g.N) {
        float* o = out + (size_t)grow * ld + gcol;
        if (gcol + 3 < g.N && aligned16(o)) {
          *reinterpret_cast<float4*>(o) = x;
        } else {
          const float e[4] = {x.x, x.y, x.z, x.w};
          for (int j = 0; j < 4 && gcol + j < g.N; ++j) o[j] = e[j];
        }
      }
    }
    __syncwarp();
  };
  // the same for bf16 values (32 per lane, packed in pairs)
  auto put_bf16 = [&](const uint32_t (&h)[16], uint16_t* out, int ld, int col0) {
    uint4* t4 = reinterpret_cast<uint4*>(tb + lane * kPitchB);
#pragma unroll
    for (int q = 0; q < 4; ++q) t4[q] = make_uint4(h[4 * q], h[4 * q + 1], h[4 * q + 2], h[4 * q + 3]);
    __syncwarp();
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int r = 8 * i + (lane >> 2), q = lane & 3;
      const int grow = row0 + r, gcol = col0 + 8 * q;
      const uint4 x = reinterpret_cast<const uint4*>(tb + r * kPitchB)[q];
      if (grow < g.M && gcol < g.N) {
        uint16_t* o = out + (size_t)grow * ld + gcol;
        if (gcol + 7 < g.N && aligned16(o)) {
          *reinterpret_cast<uint4*>(o) = x;
        } else {
          const uint32_t w[4] = {x.x, x.y, x.z, x.w};
          for (int j = 0; j < 8 && gcol + j < g.N; ++j) o[j] = (uint16_t)(w[j >> 1] >> (16 * (j & 1)));
        }
      }
    }
    __syncwarp();
  };
  // z of the GELU derivative for the block's rows: coalesced loads into the fp32 tile, then each
  // lane reads its own row (columns past N read as 0)
  auto get_f32 = [&](const float* in, int ld, int col0, float (&zv)[32]) {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int r = 4 * i + (lane >> 3), q = lane & 7;
      const int grow = row0 + r, gcol = col0 + 4 * q;
      float4 x = make_float4(0.f, 0.f, 0.f, 0.f);
      if (grow < g.M && gcol < g.N) {
        const float* z = in + (size_t)grow * ld + gcol;
        if (gcol + 3 < g.N && aligned16(z)) {
          x = *reinterpret_cast<const float4*>(z);
        } else {
          float e[4] = {0.f, 0.f, 0.f, 0.f};
          for (int j = 0; j < 4 && gcol + j < g.N; ++j) e[j] = z[j];
          x = make_float4(e[0], e[1], e[2], e[3]);
        }
      }
      reinterpret_cast<float4*>(tf + r * kPitchF)[q] = x;
    }
    __syncwarp();
    const float4* t4 = reinterpret_cast<const float4*>(tf + lane * kPitchF);
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const float4 x = t4[q];
      zv[4 * q] = x.x;
      zv[4 * q + 1] = x.y;
      zv[4 * q + 2] = x.z;
      zv[4 * q + 3] = x.w;
    }
    __syncwarp();
  };
  for (int c = 0; c < nt / 32; ++c) {
    float v[32];
    __syncwarp();
    tmem_ld32(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(c * 32), v);
    const int col0 = n0 + c * 32;
    if (!all_done || row0 >= g.M || col0 >= g.N) continue;  // warp-uniform
    const float4* sb4 = reinterpret_cast<const float4*>(sm->bias + c * 32);
    if (use_bias) {
#pragma unroll
      for (int j = 0; j < 32; j += 4) {
        const float4 b4 = sb4[j / 4];
        v[j] += b4.x;
        v[j + 1] += b4.y;
        v[j + 2] += b4.z;
        v[j + 3] += b4.w;
      }
    }
    if (g.epi == kEpiStoreF32 || g.epi == kEpiBias) {
      put_f32(v, g.out_f32, g.ld_out, col0);
    } else if (g.epi == kEpiBiasGelu) {
      if (g.out_f32) put_f32(v, g.out_f32, g.ld_out, col0);
      uint32_t h[16];
#pragma unroll
      for (int j = 0; j < 16; ++j)
        h[j] = (uint32_t)to_bf16(gelu(v[2 * j])) | ((uint32_t)to_bf16(gelu(v[2 * j + 1])) << 16);
      put_bf16(h, g.out_bf16, g.ld_bf16, col0);
    } else {  // kEpiGeluGrad: dZ = (dZ_next W) * gelu'(z)
      float zv[32];
      get_f32(g.zin, g.ld_zin, col0, zv);
      uint32_t h[16];
#pragma unroll
      for (int j = 0; j < 16; ++j)
        h[j] = (uint32_t)to_bf16(v[2 * j] * gelu_grad(zv[2 * j])) |
               ((uint32_t)to_bf16(v[2 * j + 1] * gelu_grad(zv[2 * j + 1])) << 16);
      put_bf16(h, g.out_bf16, g.ld_bf16, col0);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" : : "r"(tmem), "r"(nt));
  }
}

// ---------------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------------
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
  static std::once_flag once;
  static EncodeTiledFn fn = nullptr;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  });
  return fn;
}

// Tensor map over a row-major bf16 tensor [rows][cols] (leading dimension ld elements) viewed as
// {8 contiguous elements, row, column group of 8}; box {8, box_rows, box_groups}.
static bool make_map(CUtensorMap* m, const uint16_t* ptr, int rows, int cols, int ld, int box_rows, int box_groups) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return false;
  const cuuint64_t dims[3] = {8, (cuuint64_t)rows, (cuuint64_t)(cols / 8)};
  const cuuint64_t strides[2] = {(cuuint64_t)ld * 2, 16};
  const cuuint32_t box[3] = {8, (cuuint32_t)box_rows, (cuuint32_t)box_groups};
  const cuuint32_t estr[3] = {1, 1, 1};
  std::memset(m, 0, sizeof(*m));
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<uint16_t*>(ptr), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

size_t smem_bytes(int ntile) { return 2 * (size_t)(kTileM * kChunkK * 2 + ntile * kChunkK * 2) + 1024 + sizeof(Smem) + 64; }

// The kernel's dynamic shared-memory limit is raised once per device to what the widest tile
// (256 columns) needs, and never lowered: a launch with a narrower tile needs less, and a CUDA graph
// whose nodes were captured with different tile widths stays launchable whatever was set last.
// (Setting the limit per launch to that launch's own need left it at the last layer's 42 KB after a
// forward pass, below the 99 KB of the hidden layers' nodes.)
constexpr int kMaxDevices = 64;
cudaError_t set_smem_limit_once() {
  static std::mutex mu;
  static uint64_t done_ctx[kMaxDevices] = {0};  // context_id() the limit was set in (0: not set)
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(mu);
  const uint64_t ctx = context_id();
  if (ctx != 0 && done_ctx[dev] == ctx) return cudaSuccess;
  e = cudaFuncSetAttribute(gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes(256));
  if (e == cudaSuccess) done_ctx[dev] = context_id();
  return e;
}

const char* check(const GemmOperands& op, const GemmArgs& g) {
  if (g.M < 1 || g.N < 1 || g.K < 1) return "GEMM sizes must be positive";
  if (g.ntile != 32 && g.ntile != 64 && g.ntile != 128 && g.ntile != 256) return "GEMM tile width must be 32, 64, 128 or 256";
  if (((uintptr_t)op.a | (uintptr_t)op.b) & 15) return "GEMM operands must be 16-byte aligned";
  if ((op.lda | op.ldb) & 7) return "GEMM leading dimensions must be multiples of 8";
  // contiguous extents must be whole groups of 8 elements
  if ((g.a_mn ? g.M : g.K) % 8 || (g.b_mn ? g.N : g.K) % 8) return "GEMM contiguous extents must be multiples of 8";
  if (g.M > (1 << 24) || g.N > (1 << 24) || g.K > (1 << 24)) return "GEMM too large";
  return nullptr;
}

cudaError_t launch(const GemmOperands& op, const GemmArgs& g, cudaStream_t s, const char** why) {
  *why = check(op, g);
  if (*why) return cudaErrorInvalidValue;
  CUtensorMap ma, mb;
  const bool ok_a = g.a_mn ? make_map(&ma, op.a, g.K, g.M, op.lda, kChunkK, kTileM / 8)
                           : make_map(&ma, op.a, g.M, g.K, op.lda, kTileM, kChunkK / 8);
  const bool ok_b = g.b_mn ? make_map(&mb, op.b, g.K, g.N, op.ldb, kChunkK, g.ntile / 8)
                           : make_map(&mb, op.b, g.N, g.K, op.ldb, g.ntile, kChunkK / 8);
  if (!ok_a || !ok_b) {
    *why = "cuTensorMapEncodeTiled failed (driver entry point missing or unsupported tensor shape)";
    return cudaErrorInvalidValue;
  }
  const size_t sm = smem_bytes(g.ntile);
  const cudaError_t attr = set_smem_limit_once();
  if (attr != cudaSuccess) return attr;
  const dim3 grid((g.M + kTileM - 1) / kTileM, (g.N + g.ntile - 1) / g.ntile);
  gemm_kernel<<<grid, kThreads, sm, s>>>(ma, mb, g);
  return cudaGetLastError();
}

}  // namespace gemm
}  // namespace bpx
