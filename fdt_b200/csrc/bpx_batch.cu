// bpx_batch.cu -- the batched form: many volumes of uneven voxel counts, measurement counts,
// models and fibre counts in one CUDA-graph launch, with a per-bucket launch-layout autotuner.
// No counterpart in the reference (xfibres_gpu runs one subpart of one volume per call,
// CUDA/xfibres_gpu.cu:29-146, with one fixed launch shape).
//
// Items are grouped into buckets of equal (model, fibres, measurements, b-matrix, start: LM fits
// or an initialiser network, burn-in).  A bucket's
// voxels are packed into one contiguous set of buffers, so one fit, one MCMC and one finishing
// launch (each grid-stride over the whole bucket) process every voxel of every item in it; the
// chains keep each item's own RNG keys (item voxel_offset + local index), so a batched run equals
// the per-item runs bit for bit.  The batch is captured once into a CUDA graph -- gather, then
// per bucket [Rician clean-up, fit or network start, MCMC, finish] on its own branch, then scatter to the items'
// output buffers -- and every bpx_batch_run is one cudaGraphLaunch.
//
// Autotuner: for a bucket, every compiled (threads-per-voxel, measurements-per-lane) layout that
// covers its measurements is timed on forward-model voxels (a short chain) and the fastest is kept
// (cached per device and bucket key).  The layout fixes both the threads per voxel and the voxels
// per 128-thread block (128 / threads-per-voxel).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "bpx.h"
#include "bpx_internal.h"

namespace bpx {
namespace {

struct ItemOut {
  bpx_outputs out;
  int nvox;
  int pad;
};

// one warp per packed voxel: copy its measurement row from the item's data
__global__ void gather_kernel(int n, int ndir, const float* const* __restrict__ src, float* __restrict__ dst) {
  const int lane = threadIdx.x & 31;
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  for (int v = w; v < n; v += nw) {
    const float* s = src[v];
    float* d = dst + (size_t)v * ndir;
    for (int m = lane; m < ndir; m += 32) d[m] = s[m];
  }
}

// one thread per packed voxel: copy every output row of the voxel into its item's buffers
__global__ void scatter_kernel(int n, int K, int ns, const int* __restrict__ item_of, const int* __restrict__ local_of,
                               const ItemOut* __restrict__ items, bpx_outputs packed) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    const ItemOut& it = items[item_of[v]];
    const int l = local_of[v], nv = it.nvox;
    const bpx_outputs& o = it.out;
    for (int r = 0; r < K * ns; ++r) {
      if (o.th) o.th[(size_t)r * nv + l] = packed.th[(size_t)r * n + v];
      if (o.ph) o.ph[(size_t)r * nv + l] = packed.ph[(size_t)r * n + v];
      if (o.f) o.f[(size_t)r * nv + l] = packed.f[(size_t)r * n + v];
    }
    if (o.mean_d) o.mean_d[l] = packed.mean_d[v];
    if (o.mean_dstd) o.mean_dstd[l] = packed.mean_dstd[v];
    if (o.mean_R) o.mean_R[l] = packed.mean_R[v];
    if (o.mean_f0) o.mean_f0[l] = packed.mean_f0[v];
    if (o.mean_tau) o.mean_tau[l] = packed.mean_tau[v];
    if (o.mean_S0) o.mean_S0[l] = packed.mean_S0[v];
    for (int k = 0; k < K; ++k)
      if (o.mean_f) o.mean_f[(size_t)k * nv + l] = packed.mean_f[(size_t)k * n + v];
    for (int r = 0; r < 3 * K; ++r)
      if (o.dyads) o.dyads[(size_t)r * nv + l] = packed.dyads[(size_t)r * n + v];
    if (o.status) o.status[l] = packed.status[v];
  }
}

size_t a256(size_t x) { return (x + 255) & ~(size_t)255; }

struct Bucket {
  int model, K, M;
  const float* bvecs;
  const float* bvals;
  const float* mlp = nullptr;  // initialiser network (learned start) or NULL (LM fits)
  int nburn = 0, freeze = 0;
  McmcLayout lay;
  std::vector<int> items;
  int n = 0;
  // device buffers (views into the batch arena)
  float* data = nullptr;
  float* params = nullptr;
  float* tau = nullptr;
  uint32_t* status = nullptr;
  float* rec = nullptr;
  void* fit_scratch = nullptr;  // LM start: FP64 parameters between the fit stages
  uint64_t* keys = nullptr;
  const float** src = nullptr;
  int* item_of = nullptr;
  int* local_of = nullptr;
  ItemOut* item_tab = nullptr;
  bpx_outputs packed{};
  // learned start: network inputs, outputs and working buffers
  uint16_t* x = nullptr;
  float* s0hat = nullptr;
  float* netout = nullptr;
  float* props = nullptr;
  uint16_t* wbf = nullptr;
  uint16_t* act0 = nullptr;
  uint16_t* act1 = nullptr;
  int chunk = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
};

// -------------------------------------------------------------------------------------------
// autotuner
// -------------------------------------------------------------------------------------------
std::mutex g_tune_mutex;
std::map<std::tuple<int, int, int, int, int, int, int, int>, McmcLayout> g_tuned;

struct DevBuf {
  void* p = nullptr;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
};

}  // namespace
}  // namespace bpx

using namespace bpx;

struct bpx_batch {
  bpx_options opts{};
  std::vector<bpx_item> items;
  std::vector<Bucket> buckets;
  void* arena = nullptr;
  cudaStream_t cap = nullptr;
  cudaEvent_t fork = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  ~bpx_batch() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    for (Bucket& b : buckets) {
      if (b.stream) cudaStreamDestroy(b.stream);
      if (b.done) cudaEventDestroy(b.done);
    }
    if (fork) cudaEventDestroy(fork);
    if (cap) cudaStreamDestroy(cap);
    if (arena) cudaFree(arena);
  }
};

namespace {

bpx_status cuda_err(cudaError_t e, const char* where) { return api_cuda_fail(e, where); }

#define BAT_CUDA(call)                                    \
  do {                                                    \
    cudaError_t e_ = (call);                              \
    if (e_ != cudaSuccess) return cuda_err(e_, #call);    \
  } while (0)

FitArgs fit_args(const bpx_options& o, const Bucket& b) {
  FitArgs a{};
  a.nvox = b.n;
  a.ndir = b.M;
  a.data = b.data;
  a.bvecs = b.bvecs;
  a.bvals = b.bvals;
  a.gradnonlin = 0;
  a.params = b.params;
  bpx_options oo = o;
  oo.model = b.model;
  oo.nfibres = b.K;
  a.np_out = bpx_nparams_fit(&oo);
  a.tau = b.tau;
  a.status = b.status;
  a.model = b.model;
  a.rician = o.rician;
  a.nonlin = o.nonlin;
  a.R = o.R_prior_mean;
  a.scratch = (double*)b.fit_scratch;
  a.flags = (uint32_t*)((char*)b.fit_scratch + (size_t)b.n * 16 * sizeof(double));
  return a;
}

McmcArgs mcmc_args(const bpx_options& o, const Bucket& b) {
  McmcArgs a{};
  bpx_options oo = o;
  oo.model = b.model;
  oo.nfibres = b.K;
  a.nvox = b.n;
  a.ndir = b.M;
  a.data = b.data;
  a.bvecs = b.bvecs;
  a.bvals = b.bvals;
  a.gradnonlin = 0;
  a.params = b.params;
  a.np_fit = bpx_nparams_fit(&oo);
  a.tau = b.tau;
  a.records = b.rec;
  a.nsamples = bpx_nsamples(&o);
  a.status = b.status;
  a.nburn = o.nburn;
  a.njumps = o.njumps;
  a.sampleevery = o.sampleevery;
  a.upe = o.updateproposalevery;
  a.f0 = o.f0;
  a.ardf0 = o.ardf0;
  a.no_ard = o.no_ard;
  a.all_ard = o.all_ard;
  a.fudge = o.fudge;
  a.R_mean = o.R_prior_mean;
  a.R_std = o.R_prior_std;
  a.R_fudge = o.R_prior_fudge;
  a.seed = o.seed;
  a.voxel_offset = 0;
  a.voxel_keys = b.keys;
  a.nburn = b.nburn;
  if (b.mlp) {
    a.props_in = b.props;
    a.freeze_props = b.freeze;
  }
  return a;
}

// times the compiled layouts that cover ndir on `sample` forward-model voxels (short chain) and
// returns the fastest; seconds per voxel of each candidate go to `timing` (-1: not a candidate)
bpx_status tune(const bpx_options* opts, int ndir, const float* bvecs, const float* bvals, int sample,
                McmcLayout* best, float* timing, cudaStream_t s) {
  int dev = 0;
  BAT_CUDA(cudaGetDevice(&dev));
  const auto key = std::make_tuple(dev, opts->model, opts->nfibres, opts->rician, opts->f0, opts->ardf0, ndir,
                                   opts->nonlin);
  if (!timing) {
    std::lock_guard<std::mutex> lk(g_tune_mutex);
    auto it = g_tuned.find(key);
    if (it != g_tuned.end()) {
      *best = it->second;
      return BPX_OK;
    }
  }
  const int nl = bpx_mcmc_layouts(nullptr, nullptr, 0);
  std::vector<int32_t> tpv(nl), mpl(nl);
  bpx_mcmc_layouts(tpv.data(), mpl.data(), nl);
  const int K = opts->nfibres, P = bpx_nparams_fit(opts);
  bpx_options t = *opts;
  t.nburn = 40;
  t.njumps = 25;
  t.sampleevery = 25;
  const int nrec = BPX_NREC(K);
  DevBuf buf;
  const size_t b_d = a256((size_t)sample * ndir * 4), b_p = a256((size_t)sample * P * 4), b_v = a256((size_t)sample * 4);
  const size_t b_r = a256((size_t)nrec * sample * 4);
  BAT_CUDA(cudaMalloc(&buf.p, b_d + b_p + 2 * b_v + b_r));
  char* p = (char*)buf.p;
  float* data = (float*)p;
  float* params = (float*)(p + b_d);
  float* tau = (float*)(p + b_d + b_p);
  uint32_t* status = (uint32_t*)(p + b_d + b_p + b_v);
  float* rec = (float*)(p + b_d + b_p + 2 * b_v);
  bpx_status st = bpx_synth_dev(opts->model == 1 ? 1 : 2, K, sample, ndir, 0x7a11ull, 0, 25.f, 25.f, bvecs, bvals, data,
                                nullptr, s);
  if (st != BPX_OK) return st;
  bpx_volume vol{};
  vol.nvox = sample;
  vol.ndir = ndir;
  vol.data = data;
  vol.bvecs = bvecs;
  vol.bvals = bvals;
  if (opts->rician) {
    st = bpx_prepare_data_dev(sample, ndir, data, s);
    if (st != BPX_OK) return st;
  }
  st = bpx_fit_dev(&t, &vol, params, tau, status, s);
  if (st != BPX_OK) return st;
  cudaEvent_t e0, e1;
  BAT_CUDA(cudaEventCreate(&e0));
  BAT_CUDA(cudaEventCreate(&e1));
  float best_t = 1e30f;
  *best = McmcLayout{0, 0};
  for (int i = 0; i < nl; ++i) {
    if (timing) timing[i] = -1.f;
    const McmcLayout lay{tpv[i], mpl[i]};
    if (lay.tpv * lay.mpl < ndir || !layout_supported(t.model, K, t.rician != 0, lay)) continue;
    t.mcmc_tpv = lay.tpv;
    t.mcmc_mpl = lay.mpl;
    float ms = 0.f;
    for (int rep = 0; rep < 2; ++rep) {  // the first run warms the instruction cache and clocks
      cudaEventRecord(e0, s);
      st = bpx_mcmc_dev(&t, &vol, params, tau, rec, status, s);
      cudaEventRecord(e1, s);
      if (st != BPX_OK) break;
      const cudaError_t e = cudaEventSynchronize(e1);
      if (e != cudaSuccess) {
        st = cuda_err(e, "autotune");
        break;
      }
      cudaEventElapsedTime(&ms, e0, e1);
    }
    if (st != BPX_OK) break;
    const float spv = ms * 1e-3f / sample;
    if (timing) timing[i] = spv;
    if (spv < best_t) {
      best_t = spv;
      *best = lay;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st != BPX_OK) return st;
  if (best->tpv == 0) return api_fail(BPX_ERR_UNSUPPORTED, "no compiled MCMC layout covers ndir=" + std::to_string(ndir));
  std::lock_guard<std::mutex> lk(g_tune_mutex);
  g_tuned[key] = *best;
  return BPX_OK;
}

}  // namespace

extern "C" {

bpx_status bpx_autotune_layout(const bpx_options* opts, int32_t ndir, const float* bvecs, const float* bvals,
                               int32_t sample, int32_t* tpv, int32_t* mpl, float* seconds_per_voxel, void* stream) {
  bpx_status st = api_check_opts(opts);
  if (st != BPX_OK) return st;
  if (ndir < 7 || ndir > bpx_max_ndir() || sample < 32 || !bvecs || !bvals || !tpv || !mpl)
    return api_fail(BPX_ERR_INVALID_ARG, "bpx_autotune_layout: bad arguments");
  st = api_check_device();
  if (st != BPX_OK) return st;
  McmcLayout best{};
  st = tune(opts, ndir, bvecs, bvals, sample, &best, seconds_per_voxel, (cudaStream_t)stream);
  if (st != BPX_OK) return st;
  *tpv = best.tpv;
  *mpl = best.mpl;
  return BPX_OK;
}

bpx_status bpx_batch_create(const bpx_options* opts, const bpx_item* items, int32_t nitems, int32_t autotune,
                            bpx_batch** out) {
  if (!out) return api_fail(BPX_ERR_INVALID_ARG, "out is NULL");
  *out = nullptr;
  bpx_status st = api_check_opts(opts);
  if (st != BPX_OK) return st;
  if (nitems < 1 || !items) return api_fail(BPX_ERR_INVALID_ARG, "no items");
  const int ns = bpx_nsamples(opts);
  if (ns < 1) return api_fail(BPX_ERR_INVALID_ARG, "no samples (njumps < sampleevery)");
  st = api_check_device();
  if (st != BPX_OK) return st;
  auto b = std::make_unique<bpx_batch>();
  b->opts = *opts;
  b->items.assign(items, items + nitems);
  // ---- buckets ----
  for (int i = 0; i < nitems; ++i) {
    const bpx_item& it = items[i];
    bpx_options oi = *opts;
    oi.model = it.model;
    oi.nfibres = it.nfibres;
    st = api_check_opts(&oi);
    if (st == BPX_OK) st = api_check_vol(&it.vol);
    if (st != BPX_OK) return st;
    if (it.vol.grad) return api_fail(BPX_ERR_UNSUPPORTED, "gradnonlin items are not batched");
    if (it.vol.nvox == 0) continue;
    const int nburn = it.nburn >= 0 ? it.nburn : opts->nburn;
    const int freeze = it.mlp_params ? it.freeze_props : 0;
    if (freeze < 0 || freeze > 2) return api_fail(BPX_ERR_INVALID_ARG, "item freeze_props must be 0, 1 or 2");
    Bucket* bk = nullptr;
    for (Bucket& c : b->buckets)
      if (c.model == it.model && c.K == it.nfibres && c.M == it.vol.ndir && c.bvecs == it.vol.bvecs &&
          c.bvals == it.vol.bvals && c.mlp == it.mlp_params && c.nburn == nburn && c.freeze == freeze)
        bk = &c;
    if (!bk) {
      b->buckets.emplace_back();
      bk = &b->buckets.back();
      bk->model = it.model;
      bk->K = it.nfibres;
      bk->M = it.vol.ndir;
      bk->bvecs = it.vol.bvecs;
      bk->bvals = it.vol.bvals;
      bk->mlp = it.mlp_params;
      bk->nburn = nburn;
      bk->freeze = freeze;
    }
    bk->items.push_back(i);
    bk->n += it.vol.nvox;
  }
  // ---- layouts ----
  for (Bucket& bk : b->buckets) {
    bpx_options oi = *opts;
    oi.model = bk.model;
    oi.nfibres = bk.K;
    if (opts->mcmc_tpv > 0 && opts->mcmc_mpl > 0) {
      bk.lay = McmcLayout{opts->mcmc_tpv, opts->mcmc_mpl};
    } else if (autotune) {
      st = tune(&oi, bk.M, bk.bvecs, bk.bvals, std::min(4096, std::max(512, bk.n)), &bk.lay, nullptr, nullptr);
      if (st != BPX_OK) return st;
    } else {
      bk.lay = choose_layout(bk.model, bk.K, opts->rician != 0, bk.M);
    }
    if (bk.lay.tpv == 0 || bk.lay.tpv * bk.lay.mpl < bk.M || !layout_supported(bk.model, bk.K, opts->rician != 0, bk.lay))
      return api_fail(BPX_ERR_UNSUPPORTED, "no compiled MCMC layout for ndir=" + std::to_string(bk.M));
  }
  // ---- arena ----
  size_t total = 0;
  std::vector<size_t> base(b->buckets.size());
  auto learned_bytes = [&](const Bucket& bk) -> size_t {
    if (!bk.mlp) return 0;
    const size_t n = bk.n, nin = bpx_mlp_nin(bk.M), chunk = std::min<size_t>(n, 32768);
    return a256(n * nin * 2) + a256(n * 4) + a256(n * BPX_MLP_NOUT * 4) + a256((6 + 3 * bk.K) * n * 4) +
           a256(mlp_weight_elems(bk.M) * 2) + 2 * a256(chunk * BPX_MLP_WIDTH * 2);
  };
  auto bucket_bytes = [&](const Bucket& bk) {
    const size_t n = bk.n, K = bk.K, P = 2 + 3 * K + (bk.model >= 2 ? 1 : 0) + (opts->f0 ? 1 : 0);
    return a256(n * bk.M * 4) + a256(n * P * 4) + 2 * a256(n * 4) + a256(BPX_NREC(K) * ns * n * 4) + a256(n * 8) +
           a256(n * 8) + 2 * a256(n * 4) + a256(bk.items.size() * sizeof(ItemOut)) + 3 * a256(K * ns * n * 4) +
           6 * a256(n * 4) + a256(K * n * 4) + a256(3 * K * n * 4) + learned_bytes(bk) +
           (bk.mlp ? 0 : a256(n * kFitScratchBytes));
  };
  for (size_t i = 0; i < b->buckets.size(); ++i) {
    base[i] = total;
    total += bucket_bytes(b->buckets[i]);
  }
  if (total) BAT_CUDA(cudaMalloc(&b->arena, total));
  for (size_t bi = 0; bi < b->buckets.size(); ++bi) {
    Bucket& bk = b->buckets[bi];
    char* p = (char*)b->arena + base[bi];
    const size_t n = bk.n, K = bk.K, P = 2 + 3 * K + (bk.model >= 2 ? 1 : 0) + (opts->f0 ? 1 : 0);
    auto take = [&](size_t bytes) {
      char* r = p;
      p += a256(bytes);
      return r;
    };
    bk.data = (float*)take(n * bk.M * 4);
    bk.params = (float*)take(n * P * 4);
    bk.tau = (float*)take(n * 4);
    bk.status = (uint32_t*)take(n * 4);
    bk.rec = (float*)take(BPX_NREC(K) * ns * n * 4);
    bk.keys = (uint64_t*)take(n * 8);
    bk.src = (const float**)take(n * 8);
    bk.item_of = (int*)take(n * 4);
    bk.local_of = (int*)take(n * 4);
    bk.item_tab = (ItemOut*)take(bk.items.size() * sizeof(ItemOut));
    bk.packed.th = (float*)take(K * ns * n * 4);
    bk.packed.ph = (float*)take(K * ns * n * 4);
    bk.packed.f = (float*)take(K * ns * n * 4);
    bk.packed.mean_d = (float*)take(n * 4);
    bk.packed.mean_dstd = (float*)take(n * 4);
    bk.packed.mean_R = (float*)take(n * 4);
    bk.packed.mean_f0 = (float*)take(n * 4);
    bk.packed.mean_tau = (float*)take(n * 4);
    bk.packed.mean_S0 = (float*)take(n * 4);
    bk.packed.status = bk.status;  // written by the fit and MCMC kernels
    bk.packed.mean_f = (float*)take(K * n * 4);
    bk.packed.dyads = (float*)take(3 * K * n * 4);
    if (!bk.mlp) bk.fit_scratch = take(n * kFitScratchBytes);
    if (bk.mlp) {
      bk.chunk = (int)std::min<size_t>(n, 32768);
      bk.x = (uint16_t*)take(n * bpx_mlp_nin(bk.M) * 2);
      bk.s0hat = (float*)take(n * 4);
      bk.netout = (float*)take(n * BPX_MLP_NOUT * 4);
      bk.props = (float*)take((6 + 3 * K) * n * 4);
      bk.wbf = (uint16_t*)take(mlp_weight_elems(bk.M) * 2);
      bk.act0 = (uint16_t*)take((size_t)bk.chunk * BPX_MLP_WIDTH * 2);
      bk.act1 = (uint16_t*)take((size_t)bk.chunk * BPX_MLP_WIDTH * 2);
    }
    // voxel maps
    std::vector<uint64_t> keys(n);
    std::vector<const float*> src(n);
    std::vector<int> item_of(n), local_of(n);
    std::vector<ItemOut> tab(bk.items.size());
    size_t v = 0;
    for (size_t j = 0; j < bk.items.size(); ++j) {
      const bpx_item& it = items[bk.items[j]];
      tab[j].out = it.out;
      tab[j].nvox = it.vol.nvox;
      for (int l = 0; l < it.vol.nvox; ++l, ++v) {
        keys[v] = it.vol.voxel_offset + (uint64_t)l;
        src[v] = it.vol.data + (size_t)l * bk.M;
        item_of[v] = (int)j;
        local_of[v] = l;
      }
    }
    BAT_CUDA(cudaMemcpy(bk.keys, keys.data(), n * 8, cudaMemcpyHostToDevice));
    BAT_CUDA(cudaMemcpy(bk.src, src.data(), n * 8, cudaMemcpyHostToDevice));
    BAT_CUDA(cudaMemcpy(bk.item_of, item_of.data(), n * 4, cudaMemcpyHostToDevice));
    BAT_CUDA(cudaMemcpy(bk.local_of, local_of.data(), n * 4, cudaMemcpyHostToDevice));
    BAT_CUDA(cudaMemcpy(bk.item_tab, tab.data(), tab.size() * sizeof(ItemOut), cudaMemcpyHostToDevice));
    BAT_CUDA(cudaStreamCreateWithFlags(&bk.stream, cudaStreamNonBlocking));
    BAT_CUDA(cudaEventCreateWithFlags(&bk.done, cudaEventDisableTiming));
  }
  for (const Bucket& bk : b->buckets)
    if (bk.mlp) {  // create the network kernels' error word now, outside the capture
      int32_t code = 0;
      st = bpx_mlp_poll_error(&code);
      if (st != BPX_OK) return st;
      break;
    }
  // ---- capture: fork one branch per bucket, join ----
  BAT_CUDA(cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking));
  BAT_CUDA(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
  BAT_CUDA(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeRelaxed));
  cudaError_t ce = cudaEventRecord(b->fork, b->cap);
  const int sms = sm_count();
  for (Bucket& bk : b->buckets) {
    if (ce != cudaSuccess) break;
    ce = cudaStreamWaitEvent(bk.stream, b->fork, 0);
    if (ce != cudaSuccess) break;
    const int gblocks = std::min((bk.n + 7) / 8, sms * 16);
    gather_kernel<<<gblocks, 256, 0, bk.stream>>>(bk.n, bk.M, bk.src, bk.data);
    if (opts->rician && ce == cudaSuccess) ce = launch_prepare(bk.n, bk.M, bk.data, bk.stream);
    if (ce == cudaSuccess && !bk.mlp) ce = launch_fit(fit_args(*opts, bk), bk.K, opts->f0 != 0, bk.stream);
    if (ce == cudaSuccess && bk.mlp) {
      // learned start: features -> network (tcgen05) -> state, tau and proposal widths
      bpx_options oi = *opts;
      oi.model = bk.model;
      oi.nfibres = bk.K;
      bpx_volume pv{};
      pv.nvox = bk.n;
      pv.ndir = bk.M;
      pv.data = bk.data;
      pv.bvecs = bk.bvecs;
      pv.bvals = bk.bvals;
      bpx_status ls = bpx_mlp_features_dev(&pv, 0, bk.x, bk.s0hat, bk.stream);
      if (ls == BPX_OK)
        ls = mlp_forward_buffers(bk.M, bk.mlp, bk.n, bk.x, bk.netout, bk.wbf, bk.act0, bk.act1, bk.chunk, bk.stream);
      if (ls == BPX_OK)
        ls = bpx_mlp_decode_dev(&oi, bk.n, bk.netout, bk.s0hat, bk.params, bk.tau, bk.props, bk.status, bk.stream);
      if (ls != BPX_OK) {
        cudaGraph_t junk = nullptr;
        cudaStreamEndCapture(b->cap, &junk);
        if (junk) cudaGraphDestroy(junk);
        return ls;
      }
    }
    if (ce == cudaSuccess) ce = launch_mcmc(mcmc_args(*opts, bk), bk.model, bk.K, opts->rician != 0, bk.lay, bk.stream);
    if (ce == cudaSuccess) {
      FinishArgs fa{};
      fa.nvox = bk.n;
      fa.nsamples = ns;
      fa.nfib = bk.K;
      fa.records = bk.rec;
      fa.out = bk.packed;
      ce = launch_finish(fa, bk.stream);
    }
    if (ce == cudaSuccess) {
      scatter_kernel<<<std::min((bk.n + 255) / 256, sms * 8), 256, 0, bk.stream>>>(bk.n, bk.K, ns, bk.item_of,
                                                                                  bk.local_of, bk.item_tab, bk.packed);
      ce = cudaGetLastError();
    }
    if (ce == cudaSuccess) ce = cudaEventRecord(bk.done, bk.stream);
    if (ce == cudaSuccess) ce = cudaStreamWaitEvent(b->cap, bk.done, 0);
  }
  cudaGraph_t g = nullptr;
  const cudaError_t ee = cudaStreamEndCapture(b->cap, &g);
  if (ce != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return cuda_err(ce, "batch capture");
  }
  if (ee != cudaSuccess) return cuda_err(ee, "cudaStreamEndCapture");
  b->graph = g;
  BAT_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
  *out = b.release();
  return BPX_OK;
}

bpx_status bpx_batch_run(bpx_batch* b, void* stream) {
  NvtxRange nvtx_range("bpx.batch_run");
  if (!b || !b->exec) return api_fail(BPX_ERR_INVALID_ARG, "bpx_batch_run: no batch");
  BAT_CUDA(cudaGraphLaunch(b->exec, (cudaStream_t)stream));
  return BPX_OK;
}

int32_t bpx_batch_buckets(const bpx_batch* b, int32_t* desc, int32_t max) {
  if (!b) return -1;
  const int nb = (int)b->buckets.size();
  for (int i = 0; i < nb && i < max && desc; ++i) {
    const Bucket& bk = b->buckets[i];
    int32_t* d = desc + 7 * i;
    d[0] = bk.model;
    d[1] = bk.K;
    d[2] = bk.M;
    d[3] = bk.lay.tpv;
    d[4] = bk.lay.mpl;
    d[5] = bk.n;
    d[6] = (int32_t)bk.items.size();
  }
  return nb;
}

bpx_status bpx_batch_destroy(bpx_batch* b) {
  delete b;
  return BPX_OK;
}

}  // extern "C"
