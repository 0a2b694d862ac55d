// bpx_api.cu -- the C-ABI of libbpx.so (declared in include/bpx.h).
//
// Host code: option validation, launch dispatch, the per-device workspace cache and the
// host-buffer drop-in for xfibres_gpu() (CUDA/xfibres_gpu.cu:29-146).  No entry point calls
// exit(); failures return a bpx_status and leave a message for bpx_last_error().
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include <cuda.h>

#include "bpx.h"
#include "bpx_device.cuh"
#include "bpx_internal.h"

namespace bpx {

cudaError_t launch_mcmc_m1(const McmcArgs&, int, bool, McmcLayout, cudaStream_t);
cudaError_t launch_mcmc_m2(const McmcArgs&, int, bool, McmcLayout, cudaStream_t);
cudaError_t launch_mcmc_m3(const McmcArgs&, int, bool, McmcLayout, cudaStream_t);
cudaError_t launch_energy_m1(const EnergyArgs&, int, bool, McmcLayout, cudaStream_t);
cudaError_t launch_energy_m2(const EnergyArgs&, int, bool, McmcLayout, cudaStream_t);
cudaError_t launch_energy_m3(const EnergyArgs&, int, bool, McmcLayout, cudaStream_t);

namespace {
thread_local std::string g_last_error;

constexpr int kMaxDevices = 64;
int g_sm_count[kMaxDevices] = {0};

// compiled (tpv, mpl) layouts, in order of preference for a given capacity
const McmcLayout kLayouts[] = {{4, 9}, {8, 8}, {8, 9}, {16, 9}, {32, 9}, {32, 16}};
constexpr int kNumLayouts = sizeof(kLayouts) / sizeof(kLayouts[0]);
constexpr int kMaxNdir = 512;

bpx_status fail(bpx_status st, const std::string& msg) {
  g_last_error = msg;
  return st;
}

bpx_status cuda_fail(cudaError_t e, const char* where) {
  g_last_error = std::string(where) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
  return BPX_ERR_CUDA;
}

#define BPX_CUDA(call)                                   \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
  } while (0)

bpx_status check_device() {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(BPX_ERR_NO_DEVICE, std::string("no CUDA device: ") + cudaGetErrorString(e));
  int major = 0;
  e = cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute");
  if (major != 10) return fail(BPX_ERR_NO_DEVICE, "libbpx is built for sm_100a only (found compute capability " + std::to_string(major) + ".x)");
  return BPX_OK;
}

bpx_status check_opts(const bpx_options* o) {
  if (!o) return fail(BPX_ERR_INVALID_ARG, "opts is NULL");
  if (o->model < 1 || o->model > 3) return fail(BPX_ERR_INVALID_ARG, "model must be 1, 2 or 3");
  if (o->nfibres < 1 || o->nfibres > BPX_MAX_FIBRES) return fail(BPX_ERR_INVALID_ARG, "nfibres must be 1..3");
  if (o->njumps < 0 || o->nburn < 0) return fail(BPX_ERR_INVALID_ARG, "njumps and nburn must be >= 0");
  if (o->sampleevery < 1) return fail(BPX_ERR_INVALID_ARG, "sampleevery must be >= 1");
  if (o->updateproposalevery < 1) return fail(BPX_ERR_INVALID_ARG, "updateproposalevery must be >= 1");
  if (o->njumps / o->sampleevery > 255 * 256 * 256) return fail(BPX_ERR_INVALID_ARG, "too many samples");
  if (o->updateproposalevery > 255) return fail(BPX_ERR_UNSUPPORTED, "updateproposalevery > 255 is not supported (acceptance counters are 8-bit)");
  return BPX_OK;
}

bpx_status check_vol(const bpx_volume* v, bool need_data) {
  if (!v) return fail(BPX_ERR_INVALID_ARG, "vol is NULL");
  if (v->nvox < 0) return fail(BPX_ERR_INVALID_ARG, "nvox < 0");
  if (v->ndir < 7 || v->ndir > kMaxNdir) return fail(BPX_ERR_UNSUPPORTED, "ndir must be in 7.." + std::to_string(kMaxNdir));
  if (v->nvox > 0 && need_data && (!v->data || !v->bvecs || !v->bvals)) return fail(BPX_ERR_INVALID_ARG, "data/bvecs/bvals is NULL");
  return BPX_OK;
}

struct Workspace {
  void* ptr = nullptr;
  size_t cap = 0;
  uint64_t ctx = 0;  // context_id() the buffer was allocated in
};
std::mutex g_ws_mutex;
Workspace g_ws[kWorkspaceSlots][kMaxDevices];

}  // namespace
}  // namespace bpx

// A set of private workspaces (one per slot) on one device; see bpx_handle_create.
struct bpx_handle {
  int device = 0;
  bpx::Workspace ws[bpx::kWorkspaceSlots];
};

namespace bpx {
namespace {

// the handle bound to this host thread (bpx_handle_bind), or NULL: the per-device shared workspaces
thread_local bpx_handle* g_bound = nullptr;

// grow-only scratch of one slot: the bound handle's, else the device's shared one (which all
// unbound callers on the device share; see the concurrency note of bpx.h)
bpx_status workspace(size_t bytes, void** out, int slot = kWsPipeline) {
  int dev = 0;
  BPX_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_ws_mutex);
  if (g_bound && g_bound->device != dev)
    return fail(BPX_ERR_INVALID_ARG, "the handle bound to this thread belongs to device " +
                                         std::to_string(g_bound->device) + ", the current device is " +
                                         std::to_string(dev));
  Workspace& w = g_bound ? g_bound->ws[slot] : g_ws[slot][dev % kMaxDevices];
  if (w.ptr && w.ctx != context_id()) {  // allocated in a context that no longer exists: forget it
    w.ptr = nullptr;
    w.cap = 0;
  }
  if (w.cap < bytes) {
    if (w.ptr) BPX_CUDA(cudaFree(w.ptr));
    w.ptr = nullptr;
    w.cap = 0;
    BPX_CUDA(cudaMalloc(&w.ptr, bytes));
    w.cap = bytes;
    w.ctx = context_id();
  }
  *out = w.ptr;
  return BPX_OK;
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

McmcLayout pick_layout(const bpx_options* o, int ndir) {
  if (o->mcmc_tpv > 0 && o->mcmc_mpl > 0) return McmcLayout{o->mcmc_tpv, o->mcmc_mpl};
  return choose_layout(o->model, o->nfibres, o->rician != 0, ndir);
}

}  // namespace

void set_last_error(const char* msg) { g_last_error = msg ? msg : ""; }
bpx_status api_fail(bpx_status st, const std::string& msg) { return fail(st, msg); }
bpx_status api_cuda_fail(cudaError_t e, const char* where) { return cuda_fail(e, where); }
bpx_status api_check_device() { return check_device(); }
bpx_status api_check_opts(const bpx_options* o) { return check_opts(o); }
bpx_status api_check_vol(const bpx_volume* v) { return check_vol(v, true); }
bpx_status api_workspace(int slot, size_t bytes, void** out) { return workspace(bytes, out, slot); }

uint64_t context_id() {
  typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
  typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long*);
  static std::once_flag once;
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<CtxGetCurrentFn>(p);
    p = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<CtxGetIdFn>(p);
  });
  if (!get_current || !get_id) return 0;
  CUcontext c = nullptr;
  if (get_current(&c) != CUDA_SUCCESS || !c) return 0;
  unsigned long long id = 0;
  if (get_id(c, &id) != CUDA_SUCCESS) return 0;
  return (uint64_t)id;
}

int sm_count() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 1;
  dev %= kMaxDevices;
  if (g_sm_count[dev] == 0) {
    int n = 0;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    g_sm_count[dev] = n > 0 ? n : 1;
  }
  return g_sm_count[dev];
}

McmcLayout choose_layout(int model, int nfib, bool rician, int ndir) {
  (void)model;
  (void)nfib;
  (void)rician;
  for (int i = 0; i < kNumLayouts; ++i)
    if (kLayouts[i].tpv * kLayouts[i].mpl >= ndir) return kLayouts[i];
  return McmcLayout{0, 0};
}

bool layout_supported(int, int, bool, McmcLayout lay) {
  for (int i = 0; i < kNumLayouts; ++i)
    if (kLayouts[i].tpv == lay.tpv && kLayouts[i].mpl == lay.mpl) return true;
  return false;
}

cudaError_t launch_mcmc(const McmcArgs& a, int model, int nfib, bool rician, McmcLayout lay, cudaStream_t s) {
  if (a.nvox == 0) return cudaSuccess;
  switch (model) {
    case 1: return launch_mcmc_m1(a, nfib, rician, lay, s);
    case 2: return launch_mcmc_m2(a, nfib, rician, lay, s);
    case 3: return launch_mcmc_m3(a, nfib, rician, lay, s);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_energy(const EnergyArgs& a, int model, int nfib, bool rician, cudaStream_t s) {
  if (a.nvox == 0) return cudaSuccess;
  const McmcLayout lay = choose_layout(model, nfib, rician, a.ndir);
  switch (model) {
    case 1: return launch_energy_m1(a, nfib, rician, lay, s);
    case 2: return launch_energy_m2(a, nfib, rician, lay, s);
    case 3: return launch_energy_m3(a, nfib, rician, lay, s);
  }
  return cudaErrorInvalidValue;
}

// correct_bvals_bvecs (CUDA/xfibres_gpu.cu:151-170) for every (voxel, measurement)
__global__ void gradnonlin_kernel(int nvox, int ndir, const float* grad, const float* bvecs, const float* bvals,
                                  float* bvecs_out, float* bvals_out) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)nvox * ndir) return;
  const int v = (int)(i / ndir), m = (int)(i % ndir);
  const float* L = grad + (size_t)v * 9;  // column-major 3x3: L(r,c) = L[c*3 + r]
  float g[3] = {bvecs[m], bvecs[ndir + m], bvecs[2 * ndir + m]};
  float b = bvals[m];
  if (b > 0.f) {
    float h[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) h[r] = g[r] + L[0 * 3 + r] * g[0] + L[1 * 3 + r] * g[1] + L[2 * 3 + r] * g[2];
    const float mag = sqrtf(h[0] * h[0] + h[1] * h[1] + h[2] * h[2]);
    if (mag != 0.f) {
#pragma unroll
      for (int r = 0; r < 3; ++r) h[r] /= mag;
    }
#pragma unroll
    for (int r = 0; r < 3; ++r) g[r] = h[r];
    b = mag * mag * b;
  }
  float* go = bvecs_out + (size_t)v * 3 * ndir;
  go[m] = g[0];
  go[ndir + m] = g[1];
  go[2 * ndir + m] = g[2];
  bvals_out[(size_t)v * ndir + m] = b;
}

// Pipe calibration: 8 independent dependency chains per thread so issue rate, not latency,
// bounds both kernels; the grid fills every SM several times over.
__global__ void mufu_rate_kernel(float* out, int iters) {
  float a[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) a[j] = 1e-3f * (threadIdx.x + j);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int j = 0; j < 8; ++j) a[j] = ex2_approx(-a[j]);
  }
  float s = 0.f;
#pragma unroll
  for (int j = 0; j < 8; ++j) s += a[j];
  if (s == 12345.f) out[threadIdx.x] = s;
}

__global__ void fma_rate_kernel(float* out, int iters) {
  float a[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) a[j] = 1e-3f * (threadIdx.x + j);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int j = 0; j < 8; ++j) a[j] = fmaf(a[j], 0.9999f, 1e-4f);
  }
  float s = 0.f;
#pragma unroll
  for (int j = 0; j < 8; ++j) s += a[j];
  if (s == 12345.f) out[threadIdx.x] = s;
}

}  // namespace bpx

using namespace bpx;

extern "C" {

int32_t bpx_abi_version(void) { return BPX_ABI_VERSION; }

void bpx_options_default(bpx_options* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->model = 1;
  o->nfibres = 1;
  o->fudge = 1.0f;
  o->njumps = 1250;
  o->nburn = 1000;
  o->sampleevery = 25;
  o->updateproposalevery = 40;
  o->R_prior_mean = 0.13f;
  o->R_prior_std = 0.03f;
  o->R_prior_fudge = 0.0f;
  o->seed = 8665904ull;
}

int32_t bpx_nparams_fit(const bpx_options* o) {
  if (!o) return -1;
  return 2 + 3 * o->nfibres + (o->model >= 2 ? 1 : 0) + (o->f0 ? 1 : 0);
}

int32_t bpx_nsamples(const bpx_options* o) {
  if (!o || o->sampleevery < 1) return -1;
  return o->njumps / o->sampleevery;
}

int32_t bpx_max_ndir(void) { return kMaxNdir; }

const char* bpx_last_error(void) { return g_last_error.c_str(); }

int32_t bpx_mcmc_layouts(int32_t* tpv, int32_t* mpl, int32_t max) {
  for (int i = 0; i < kNumLayouts && i < max; ++i) {
    if (tpv) tpv[i] = kLayouts[i].tpv;
    if (mpl) mpl[i] = kLayouts[i].mpl;
  }
  return kNumLayouts;
}

bpx_status bpx_prepare_data_dev(int32_t nvox, int32_t ndir, float* data, void* stream) {
  NvtxRange nvtx_range("bpx.prepare");
  if (nvox < 0 || ndir < 1 || (nvox > 0 && !data)) return fail(BPX_ERR_INVALID_ARG, "bad arguments to bpx_prepare_data_dev");
  if (nvox == 0) return BPX_OK;
  bpx_status st = check_device();
  if (st != BPX_OK) return st;
  BPX_CUDA(launch_prepare(nvox, ndir, data, (cudaStream_t)stream));
  return BPX_OK;
}

bpx_status bpx_gradnonlin_dev(int32_t nvox, int32_t ndir, const float* grad, const float* bvecs, const float* bvals,
                              float* bvecs_out, float* bvals_out, void* stream) {
  if (nvox < 0 || ndir < 1) return fail(BPX_ERR_INVALID_ARG, "bad sizes to bpx_gradnonlin_dev");
  if (nvox == 0) return BPX_OK;
  if (!grad || !bvecs || !bvals || !bvecs_out || !bvals_out) return fail(BPX_ERR_INVALID_ARG, "NULL pointer to bpx_gradnonlin_dev");
  bpx_status st = check_device();
  if (st != BPX_OK) return st;
  const size_t n = (size_t)nvox * ndir;
  const int threads = 256;
  gradnonlin_kernel<<<(unsigned)((n + threads - 1) / threads), threads, 0, (cudaStream_t)stream>>>(nvox, ndir, grad, bvecs, bvals, bvecs_out, bvals_out);
  BPX_CUDA(cudaGetLastError());
  return BPX_OK;
}

}  // extern "C"

namespace bpx {

namespace {
// argument checks of the fit entries, made before any device call or allocation
bpx_status fit_validate(const bpx_options* opts, const bpx_volume* vol, const float* params, const float* tau) {
  bpx_status st = check_opts(opts);
  if (st == BPX_OK) st = check_vol(vol, true);
  if (st != BPX_OK) return st;
  if (vol->nvox == 0) return BPX_OK;
  if (!params) return fail(BPX_ERR_INVALID_ARG, "params is NULL");
  if (opts->rician && !tau) return fail(BPX_ERR_INVALID_ARG, "tau is NULL under rician");
  return check_device();
}
}  // namespace

bpx_status fit_dev_scratch(const bpx_options* opts, const bpx_volume* vol, float* params, float* tau, uint32_t* status,
                           void* scratch, void* stream) {
  NvtxRange nvtx_range("bpx.fit");
  bpx_status st = fit_validate(opts, vol, params, tau);
  if (st != BPX_OK || vol->nvox == 0) return st;
  if (!scratch) return fail(BPX_ERR_INVALID_ARG, "fit stage scratch is NULL");
  FitArgs a{};
  a.nvox = vol->nvox;
  a.ndir = vol->ndir;
  a.data = vol->data;
  a.bvecs = vol->bvecs;
  a.bvals = vol->bvals;
  a.gradnonlin = opts->gradnonlin;
  a.params = params;
  a.np_out = bpx_nparams_fit(opts);
  a.tau = tau;
  a.status = status;
  a.model = opts->model;
  a.rician = opts->rician;
  a.nonlin = opts->nonlin;
  a.R = opts->R_prior_mean;
  a.scratch = (double*)scratch;
  a.flags = (uint32_t*)((char*)scratch + (size_t)vol->nvox * 16 * sizeof(double));
  BPX_CUDA(launch_fit(a, opts->nfibres, opts->f0 != 0, (cudaStream_t)stream));
  return BPX_OK;
}

}  // namespace bpx

extern "C" {

bpx_status bpx_fit_dev(const bpx_options* opts, const bpx_volume* vol, float* params, float* tau, uint32_t* status,
                       void* stream) {
  bpx_status st = fit_validate(opts, vol, params, tau);
  if (st != BPX_OK || vol->nvox == 0) return st;
  void* scratch = nullptr;
  st = workspace((size_t)vol->nvox * kFitScratchBytes, &scratch, kWsFit);
  if (st != BPX_OK) return st;
  return fit_dev_scratch(opts, vol, params, tau, status, scratch, stream);
}

}  // extern "C"

namespace bpx {
namespace {

// One MCMC launch over a volume: the whole chain, or the stretch st describes (nullptr: all of it
// from the LM parameters).
struct Stretch {
  int it_begin, it_end;
  const float* state_in;
  float* state_out;
  const int32_t* acc_in;
  int32_t* acc_out;
};

bpx_status mcmc_run(const bpx_options* opts, const bpx_volume* vol, const float* params, const float* tau,
                    const float* props_in, float* props_out, int32_t freeze_props, float* records,
                    uint32_t* status, void* stream, const Stretch* sp) {
  NvtxRange nvtx_range("bpx.mcmc");
  bpx_status st = check_opts(opts);
  if (st == BPX_OK) st = check_vol(vol, true);
  if (st != BPX_OK) return st;
  if (vol->nvox == 0) return BPX_OK;
  const bool from_state = sp && sp->state_in;
  if ((!params && !from_state) || !records) return fail(BPX_ERR_INVALID_ARG, "params/records is NULL");
  if (opts->rician && !tau && !from_state) return fail(BPX_ERR_INVALID_ARG, "tau is NULL under rician");
  st = check_device();
  if (st != BPX_OK) return st;
  const McmcLayout lay = pick_layout(opts, vol->ndir);
  if (lay.tpv == 0 || !layout_supported(opts->model, opts->nfibres, opts->rician != 0, lay) || lay.tpv * lay.mpl < vol->ndir)
    return fail(BPX_ERR_UNSUPPORTED, "no compiled MCMC layout for ndir=" + std::to_string(vol->ndir));
  McmcArgs a{};
  a.nvox = vol->nvox;
  a.ndir = vol->ndir;
  a.data = vol->data;
  a.bvecs = vol->bvecs;
  a.bvals = vol->bvals;
  a.gradnonlin = opts->gradnonlin;
  a.params = params;
  a.np_fit = bpx_nparams_fit(opts);
  a.tau = tau;
  a.records = records;
  a.nsamples = bpx_nsamples(opts);
  a.status = status;
  a.nburn = opts->nburn;
  a.njumps = opts->njumps;
  a.sampleevery = opts->sampleevery;
  a.upe = opts->updateproposalevery;
  a.f0 = opts->f0;
  a.ardf0 = opts->ardf0;
  a.no_ard = opts->no_ard;
  a.all_ard = opts->all_ard;
  a.fudge = opts->fudge;
  a.R_mean = opts->R_prior_mean;
  a.R_std = opts->R_prior_std;
  a.R_fudge = opts->R_prior_fudge;
  a.seed = opts->seed;
  a.voxel_offset = vol->voxel_offset;
  a.props_in = props_in;
  a.props_out = props_out;
  if (freeze_props < 0 || freeze_props > 2) return fail(BPX_ERR_INVALID_ARG, "freeze_props must be 0, 1 or 2");
  a.freeze_props = freeze_props;
  if (sp) {
    a.it_begin = sp->it_begin;
    a.it_end = sp->it_end;
    a.state_in = sp->state_in;
    a.state_out = sp->state_out;
    a.acc_in = sp->acc_in;
    a.acc_out = sp->acc_out;
  }
  BPX_CUDA(launch_mcmc(a, opts->model, opts->nfibres, opts->rician != 0, lay, (cudaStream_t)stream));
  return BPX_OK;
}

}  // namespace
}  // namespace bpx

extern "C" {

bpx_status bpx_mcmc_ex_dev(const bpx_options* opts, const bpx_volume* vol, const float* params, const float* tau,
                           const float* props_in, float* props_out, int32_t freeze_props, float* records,
                           uint32_t* status, void* stream) {
  return mcmc_run(opts, vol, params, tau, props_in, props_out, freeze_props, records, status, stream, nullptr);
}

bpx_status bpx_mcmc_stretch_dev(const bpx_options* opts, const bpx_volume* vol, const float* params, const float* tau,
                                const float* state_in, const float* props_in, const int32_t* acc_in,
                                int32_t it_begin, int32_t it_end, int32_t freeze_props, float* records,
                                float* state_out, float* props_out, int32_t* acc_out, uint32_t* status,
                                void* stream) {
  bpx_status st = check_opts(opts);
  if (st != BPX_OK) return st;
  const int total = opts->nburn + opts->njumps;
  if (it_begin < 0 || it_end <= it_begin || it_end > total)
    return fail(BPX_ERR_INVALID_ARG, "need 0 <= it_begin < it_end <= nburn + njumps");
  if (it_begin > 0 && !state_in) return fail(BPX_ERR_INVALID_ARG, "a stretch that starts after iteration 0 needs state_in");
  Stretch sp{it_begin, it_end, state_in, state_out, acc_in, acc_out};
  return mcmc_run(opts, vol, params, tau, props_in, props_out, freeze_props, records, status, stream, &sp);
}

bpx_status bpx_mcmc_dev(const bpx_options* opts, const bpx_volume* vol, const float* params, const float* tau,
                        float* records, uint32_t* status, void* stream) {
  return bpx_mcmc_ex_dev(opts, vol, params, tau, nullptr, nullptr, 0, records, status, stream);
}

bpx_status bpx_finish_dev(const bpx_options* opts, int32_t nvox, const float* records, bpx_outputs* out, void* stream) {
  NvtxRange nvtx_range("bpx.finish");
  bpx_status st = check_opts(opts);
  if (st != BPX_OK) return st;
  if (nvox < 0 || !out) return fail(BPX_ERR_INVALID_ARG, "bad arguments to bpx_finish_dev");
  if (nvox == 0) return BPX_OK;
  if (!records) return fail(BPX_ERR_INVALID_ARG, "records is NULL");
  const int ns = bpx_nsamples(opts);
  if (ns < 1) return fail(BPX_ERR_INVALID_ARG, "no samples (njumps < sampleevery)");
  st = check_device();
  if (st != BPX_OK) return st;
  FinishArgs a{};
  a.nvox = nvox;
  a.nsamples = ns;
  a.nfib = opts->nfibres;
  a.records = records;
  a.out = *out;
  BPX_CUDA(launch_finish(a, (cudaStream_t)stream));
  return BPX_OK;
}

bpx_status bpx_postproc_dev(const bpx_options* opts, int32_t nvox, const bpx_outputs* out, float thr,
                            bpx_postproc* post, void* stream) {
  NvtxRange nvtx_range("bpx.postproc");
  bpx_status st = check_opts(opts);
  if (st != BPX_OK) return st;
  if (nvox < 0 || !out || !post) return fail(BPX_ERR_INVALID_ARG, "bad arguments to bpx_postproc_dev");
  if (nvox == 0) return BPX_OK;
  if (!out->th || !out->ph || !out->mean_f || !out->dyads)
    return fail(BPX_ERR_INVALID_ARG, "bpx_postproc_dev needs out->th, ph, mean_f and dyads");
  const int ns = bpx_nsamples(opts);
  if (ns < 1) return fail(BPX_ERR_INVALID_ARG, "no samples (njumps < sampleevery)");
  st = check_device();
  if (st != BPX_OK) return st;
  PostArgs a{};
  a.nvox = nvox;
  a.nsamples = ns;
  a.nfib = opts->nfibres;
  a.th = out->th;
  a.ph = out->ph;
  a.mean_f = out->mean_f;
  a.dyads = out->dyads;
  a.thr = thr;
  a.post = *post;
  BPX_CUDA(launch_postproc(a, (cudaStream_t)stream));
  return BPX_OK;
}

bpx_status bpx_energy_dev(const bpx_options* opts, const bpx_volume* vol, const float* states, float* lik, float* prior,
                          void* stream) {
  bpx_status st = check_opts(opts);
  if (st == BPX_OK) st = check_vol(vol, true);
  if (st != BPX_OK) return st;
  if (vol->nvox == 0) return BPX_OK;
  if (!states) return fail(BPX_ERR_INVALID_ARG, "states is NULL");
  st = check_device();
  if (st != BPX_OK) return st;
  EnergyArgs a{};
  a.nvox = vol->nvox;
  a.ndir = vol->ndir;
  a.data = vol->data;
  a.bvecs = vol->bvecs;
  a.bvals = vol->bvals;
  a.gradnonlin = opts->gradnonlin;
  a.states = states;
  a.lik = lik;
  a.prior = prior;
  a.f0 = opts->f0;
  a.ardf0 = opts->ardf0;
  a.no_ard = opts->no_ard;
  a.all_ard = opts->all_ard;
  a.fudge = opts->fudge;
  a.R_mean = opts->R_prior_mean;
  a.R_std = opts->R_prior_std;
  a.R_fudge = opts->R_prior_fudge;
  BPX_CUDA(launch_energy(a, opts->model, opts->nfibres, opts->rician != 0, (cudaStream_t)stream));
  return BPX_OK;
}

bpx_status bpx_xfibres_dev(const bpx_options* opts, const bpx_volume* vol, bpx_outputs* out, void* stream) {
  NvtxRange nvtx_range("bpx.xfibres");
  bpx_status st = check_opts(opts);
  if (st == BPX_OK) st = check_vol(vol, true);
  if (st != BPX_OK) return st;
  if (!out) return fail(BPX_ERR_INVALID_ARG, "out is NULL");
  if (vol->nvox == 0) return BPX_OK;
  const int ns = bpx_nsamples(opts);
  if (ns < 1) return fail(BPX_ERR_INVALID_ARG, "no samples (njumps < sampleevery)");
  st = check_device();
  if (st != BPX_OK) return st;
  const size_t nvox = vol->nvox;
  const size_t np = bpx_nparams_fit(opts);
  const size_t nrec = BPX_NREC(opts->nfibres);
  const size_t b_params = align256(nvox * np * sizeof(float));
  const size_t b_tau = align256(nvox * sizeof(float));
  const size_t b_rec = align256(nrec * ns * nvox * sizeof(float));
  const size_t b_status = align256(nvox * sizeof(uint32_t));
  void* ws = nullptr;
  st = workspace(b_params + b_tau + b_rec + b_status, &ws);
  if (st != BPX_OK) return st;
  char* p = (char*)ws;
  float* params = (float*)p;
  float* tau = (float*)(p + b_params);
  float* rec = (float*)(p + b_params + b_tau);
  uint32_t* status = out->status ? out->status : (uint32_t*)(p + b_params + b_tau + b_rec);
  if (opts->rician) {
    st = bpx_prepare_data_dev(vol->nvox, vol->ndir, const_cast<float*>(vol->data), stream);
    if (st != BPX_OK) return st;
  }
  st = bpx_fit_dev(opts, vol, params, tau, status, stream);
  if (st != BPX_OK) return st;
  st = bpx_mcmc_dev(opts, vol, params, tau, rec, status, stream);
  if (st != BPX_OK) return st;
  st = bpx_finish_dev(opts, vol->nvox, rec, out, stream);
  return st;
}

}  // extern "C"

namespace {

// Host-buffer pipeline: the plain (mlp == NULL) or the learned pipeline over the volume in
// sub-volumes of kHostChunk voxels, each through one of two device buffer sets, so that the copies
// of one sub-volume (host to device on one copy stream, device to host on another) overlap the
// computation of the next on the compute stream.  Every voxel's result is independent of the
// others and its chain is keyed by its global index (voxel_offset + position), so the outputs are
// those of one call over the whole volume, bit for bit.  Synchronous.  The sub-volume size is
// 65536 voxels (about 14 waves of the whole-brain chain on a B200), or BPX_HOST_CHUNK from the
// environment.
size_t host_chunk() {
  const char* e = std::getenv("BPX_HOST_CHUNK");
  const long long v = e ? std::atoll(e) : 0;
  return v > 0 ? (size_t)v : (size_t)65536;
}

bpx_status xfibres_host_impl(const bpx_options* opts, const bpx_volume* vol, bpx_outputs* host_out, const float* mlp,
                             int32_t freeze_props) {
  bpx_status st = check_opts(opts);
  if (st == BPX_OK) st = check_vol(vol, true);
  if (st != BPX_OK) return st;
  if (!host_out) return fail(BPX_ERR_INVALID_ARG, "host_out is NULL");
  if (vol->nvox == 0) return BPX_OK;
  if (opts->gradnonlin && !vol->grad) return fail(BPX_ERR_INVALID_ARG, "gradnonlin set but grad is NULL");
  const int ns = bpx_nsamples(opts);
  if (ns < 1) return fail(BPX_ERR_INVALID_ARG, "no samples (njumps < sampleevery)");
  st = check_device();
  if (st != BPX_OK) return st;
  const size_t nvox = vol->nvox, ndir = vol->ndir, K = opts->nfibres;
  const size_t chunk = host_chunk();
  const size_t C = nvox < chunk ? nvox : chunk;  // voxels per sub-volume
  const bool gn = opts->gradnonlin != 0;
  // device buffers: the shared b-table and weights, then two sets of per-sub-volume buffers
  const size_t b_bvec = align256(3 * ndir * 4), b_bval = align256(ndir * 4);
  const size_t b_mlp = mlp ? align256((size_t)bpx_mlp_nparams(vol->ndir) * 4) : 0;
  const size_t b_data = align256(C * ndir * 4);
  const size_t b_grad = gn ? align256(C * 9 * 4) : 0;
  const size_t b_bvec_v = gn ? align256(C * 3 * ndir * 4) : 0, b_bval_v = gn ? align256(C * ndir * 4) : 0;
  const size_t b_samp = align256(K * ns * C * 4);
  const size_t b_vox = align256(C * 4);
  const size_t b_vk = align256(K * C * 4), b_dy = align256(K * 3 * C * 4);
  const size_t per_set = b_data + b_grad + b_bvec_v + b_bval_v + 3 * b_samp + 7 * b_vox + b_vk + b_dy;
  const size_t total = b_bvec + b_bval + b_mlp + 2 * per_set;
  char* base = nullptr;
  BPX_CUDA(cudaMalloc(&base, total));
  cudaStream_t sc = nullptr, sin = nullptr, sout = nullptr;
  cudaEvent_t ev_in[2] = {nullptr, nullptr}, ev_done[2] = {nullptr, nullptr}, ev_free[2] = {nullptr, nullptr};
  cudaError_t ce = cudaStreamCreateWithFlags(&sc, cudaStreamNonBlocking);
  if (ce == cudaSuccess) ce = cudaStreamCreateWithFlags(&sin, cudaStreamNonBlocking);
  if (ce == cudaSuccess) ce = cudaStreamCreateWithFlags(&sout, cudaStreamNonBlocking);
  for (int b = 0; b < 2 && ce == cudaSuccess; ++b) {
    ce = cudaEventCreateWithFlags(&ev_in[b], cudaEventDisableTiming);
    if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&ev_done[b], cudaEventDisableTiming);
    if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&ev_free[b], cudaEventDisableTiming);
  }
  auto release = [&]() {
    if (sc) cudaStreamSynchronize(sc);
    if (sin) cudaStreamSynchronize(sin);
    if (sout) cudaStreamSynchronize(sout);
    for (int b = 0; b < 2; ++b) {
      if (ev_in[b]) cudaEventDestroy(ev_in[b]);
      if (ev_done[b]) cudaEventDestroy(ev_done[b]);
      if (ev_free[b]) cudaEventDestroy(ev_free[b]);
    }
    if (sc) cudaStreamDestroy(sc);
    if (sin) cudaStreamDestroy(sin);
    if (sout) cudaStreamDestroy(sout);
    cudaFree(base);
  };
  if (ce != cudaSuccess) {
    release();
    return cuda_fail(ce, "xfibres_host: streams and events");
  }
  char* p = base;
  auto take = [&](size_t b) {
    char* r = p;
    p += b;
    return r;
  };
  float* d_bvec = (float*)take(b_bvec);
  float* d_bval = (float*)take(b_bval);
  float* d_mlp = mlp ? (float*)take(b_mlp) : nullptr;
  struct Set {
    float *data, *grad, *bvec_v, *bval_v;
    bpx_outputs out;
  } set[2];
  for (int b = 0; b < 2; ++b) {
    Set& q = set[b];
    q.data = (float*)take(b_data);
    q.grad = gn ? (float*)take(b_grad) : nullptr;
    q.bvec_v = gn ? (float*)take(b_bvec_v) : nullptr;
    q.bval_v = gn ? (float*)take(b_bval_v) : nullptr;
    std::memset(&q.out, 0, sizeof(q.out));
    q.out.th = (float*)take(b_samp);
    q.out.ph = (float*)take(b_samp);
    q.out.f = (float*)take(b_samp);
    q.out.mean_d = (float*)take(b_vox);
    q.out.mean_dstd = (float*)take(b_vox);
    q.out.mean_R = (float*)take(b_vox);
    q.out.mean_f0 = (float*)take(b_vox);
    q.out.mean_tau = (float*)take(b_vox);
    q.out.mean_S0 = (float*)take(b_vox);
    q.out.status = (uint32_t*)take(b_vox);
    q.out.mean_f = (float*)take(b_vk);
    q.out.dyads = (float*)take(b_dy);
  }
  auto run = [&]() -> bpx_status {
    if (mlp) BPX_CUDA(cudaMemcpyAsync(d_mlp, mlp, (size_t)bpx_mlp_nparams(vol->ndir) * 4, cudaMemcpyHostToDevice, sin));
    BPX_CUDA(cudaMemcpyAsync(d_bvec, vol->bvecs, 3 * ndir * 4, cudaMemcpyHostToDevice, sin));
    BPX_CUDA(cudaMemcpyAsync(d_bval, vol->bvals, ndir * 4, cudaMemcpyHostToDevice, sin));
    const bpx_outputs& h = *host_out;
    int k = 0;
    for (size_t v0 = 0; v0 < nvox; v0 += C, ++k) {
      const size_t c = nvox - v0 < C ? nvox - v0 : C;
      Set& q = set[k & 1];
      // inputs of this sub-volume, once its buffer set's previous outputs have been copied out
      if (k >= 2) BPX_CUDA(cudaStreamWaitEvent(sin, ev_free[k & 1], 0));
      BPX_CUDA(cudaMemcpyAsync(q.data, vol->data + v0 * ndir, c * ndir * 4, cudaMemcpyHostToDevice, sin));
      if (gn) BPX_CUDA(cudaMemcpyAsync(q.grad, vol->grad + v0 * 9, c * 9 * 4, cudaMemcpyHostToDevice, sin));
      BPX_CUDA(cudaEventRecord(ev_in[k & 1], sin));
      // the pipeline on the compute stream
      BPX_CUDA(cudaStreamWaitEvent(sc, ev_in[k & 1], 0));
      bpx_volume dv = *vol;
      dv.nvox = (int32_t)c;
      dv.voxel_offset = vol->voxel_offset + v0;
      dv.data = q.data;
      dv.bvecs = d_bvec;
      dv.bvals = d_bval;
      dv.grad = nullptr;
      if (gn) {
        bpx_status s2 = bpx_gradnonlin_dev((int32_t)c, vol->ndir, q.grad, d_bvec, d_bval, q.bvec_v, q.bval_v, sc);
        if (s2 != BPX_OK) return s2;
        dv.bvecs = q.bvec_v;
        dv.bvals = q.bval_v;
      }
      bpx_status s3 = mlp ? bpx_xfibres_learned_dev(opts, &dv, d_mlp, freeze_props, &q.out, sc)
                          : bpx_xfibres_dev(opts, &dv, &q.out, sc);
      if (s3 != BPX_OK) return s3;
      BPX_CUDA(cudaEventRecord(ev_done[k & 1], sc));
      // the outputs back, into the host arrays' columns v0 .. v0 + c (pitched copies of the rows)
      BPX_CUDA(cudaStreamWaitEvent(sout, ev_done[k & 1], 0));
      auto rows_back = [&](void* dst, const void* src, size_t rows) -> cudaError_t {
        if (!dst) return cudaSuccess;
        return cudaMemcpy2DAsync((char*)dst + v0 * 4, nvox * 4, src, c * 4, c * 4, rows, cudaMemcpyDeviceToHost, sout);
      };
      BPX_CUDA(rows_back(h.th, q.out.th, K * ns));
      BPX_CUDA(rows_back(h.ph, q.out.ph, K * ns));
      BPX_CUDA(rows_back(h.f, q.out.f, K * ns));
      BPX_CUDA(rows_back(h.mean_d, q.out.mean_d, 1));
      BPX_CUDA(rows_back(h.mean_dstd, q.out.mean_dstd, 1));
      BPX_CUDA(rows_back(h.mean_R, q.out.mean_R, 1));
      BPX_CUDA(rows_back(h.mean_f0, q.out.mean_f0, 1));
      BPX_CUDA(rows_back(h.mean_tau, q.out.mean_tau, 1));
      BPX_CUDA(rows_back(h.mean_S0, q.out.mean_S0, 1));
      BPX_CUDA(rows_back(h.status, q.out.status, 1));
      BPX_CUDA(rows_back(h.mean_f, q.out.mean_f, K));
      BPX_CUDA(rows_back(h.dyads, q.out.dyads, 3 * K));
      BPX_CUDA(cudaEventRecord(ev_free[k & 1], sout));
    }
    BPX_CUDA(cudaStreamSynchronize(sout));
    BPX_CUDA(cudaStreamSynchronize(sc));
    return BPX_OK;
  };
  st = run();
  release();
  return st;
}

}  // namespace

extern "C" {

bpx_status bpx_xfibres_host(const bpx_options* opts, const bpx_volume* vol, bpx_outputs* host_out) {
  NvtxRange nvtx_range("bpx.xfibres_host");
  return xfibres_host_impl(opts, vol, host_out, nullptr, 0);
}

bpx_status bpx_xfibres_learned_host(const bpx_options* opts, const bpx_volume* vol, const float* mlp_params,
                                    int32_t freeze_props, bpx_outputs* host_out) {
  if (!mlp_params) return fail(BPX_ERR_INVALID_ARG, "mlp_params is NULL");
  return xfibres_host_impl(opts, vol, host_out, mlp_params, freeze_props);
}

bpx_status bpx_measure_pipes(double* mufu_ops_per_s, double* fma_ops_per_s) {
  bpx_status st = check_device();
  if (st != BPX_OK) return st;
  const int threads = 256, blocks = sm_count() * 8;
  float* dummy = nullptr;
  BPX_CUDA(cudaMalloc(&dummy, threads * sizeof(float)));
  cudaEvent_t e0, e1;
  BPX_CUDA(cudaEventCreate(&e0));
  BPX_CUDA(cudaEventCreate(&e1));
  auto time_it = [&](bool mufu, int iters, float* ms) -> cudaError_t {
    for (int rep = 0; rep < 2; ++rep) {  // first repetition warms up clocks and caches
      cudaEventRecord(e0, 0);
      if (mufu)
        mufu_rate_kernel<<<blocks, threads>>>(dummy, iters);
      else
        fma_rate_kernel<<<blocks, threads>>>(dummy, iters);
      cudaEventRecord(e1, 0);
      cudaError_t e = cudaEventSynchronize(e1);
      if (e != cudaSuccess) return e;
    }
    return cudaEventElapsedTime(ms, e0, e1);
  };
  float ms_m = 0.f, ms_f = 0.f;
  const int it_m = 4096, it_f = 32768;
  cudaError_t e = time_it(true, it_m, &ms_m);
  if (e == cudaSuccess) e = time_it(false, it_f, &ms_f);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(dummy);
  if (e != cudaSuccess) return cuda_fail(e, "bpx_measure_pipes");
  const double lanes = (double)blocks * threads * 8.0;
  if (mufu_ops_per_s) *mufu_ops_per_s = lanes * it_m / (ms_m * 1e-3);
  if (fma_ops_per_s) *fma_ops_per_s = lanes * it_f / (ms_f * 1e-3);
  return BPX_OK;
}

bpx_status bpx_handle_create(bpx_handle** h) {
  if (!h) return fail(BPX_ERR_INVALID_ARG, "bpx_handle_create: h is NULL");
  *h = nullptr;
  bpx_status st = check_device();
  if (st != BPX_OK) return st;
  int dev = 0;
  BPX_CUDA(cudaGetDevice(&dev));
  bpx_handle* p = new (std::nothrow) bpx_handle;
  if (!p) return fail(BPX_ERR_CUDA, "bpx_handle_create: out of host memory");
  p->device = dev;
  *h = p;
  return BPX_OK;
}

bpx_status bpx_handle_bind(bpx_handle* h) {
  g_bound = h;
  return BPX_OK;
}

bpx_status bpx_handle_destroy(bpx_handle* h) {
  if (!h) return BPX_OK;
  if (g_bound == h) g_bound = nullptr;
  int cur = 0;
  BPX_CUDA(cudaGetDevice(&cur));
  if (cur != h->device) BPX_CUDA(cudaSetDevice(h->device));
  bpx_status st = BPX_OK;
  {
    std::lock_guard<std::mutex> lk(g_ws_mutex);
    for (int slot = 0; slot < kWorkspaceSlots; ++slot) {
      Workspace& w = h->ws[slot];
      // cudaFree waits for the device's work, so kernels still using the buffer finish first
      if (w.ptr && w.ctx == context_id()) {
        const cudaError_t e = cudaFree(w.ptr);
        if (e != cudaSuccess && st == BPX_OK) st = cuda_fail(e, "bpx_handle_destroy: cudaFree");
      }
      w.ptr = nullptr;
      w.cap = 0;
    }
  }
  if (cur != h->device) cudaSetDevice(cur);
  delete h;
  return st;
}

bpx_status bpx_release_workspace(void) {
  int dev = 0;
  BPX_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_ws_mutex);
  for (int slot = 0; slot < kWorkspaceSlots; ++slot) {
    Workspace& w = g_ws[slot][dev % kMaxDevices];
    if (w.ptr && w.ctx == context_id()) BPX_CUDA(cudaFree(w.ptr));
    w.ptr = nullptr;
    w.cap = 0;
  }
  return BPX_OK;
}

}  // extern "C"
