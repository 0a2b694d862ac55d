// bpx_noalloc.cu -- the allocation-free pipeline entry (bpx_xfibres_noalloc_dev).
//
// Same stages as bpx_xfibres_dev (bpx_api.cu), but the intermediates live in a file-scope
// __device__ array instead of the grow-only workspace, so the call never allocates device memory.
// Host code must not pass the array's name to a kernel (in host code it names a host-side stand-in);
// its device address is resolved once per device with cudaGetSymbolAddress.
#include <mutex>
#include <string>

#include "bpx.h"
#include "bpx_internal.h"

namespace {

constexpr size_t kScratchBytes = BPX_NOALLOC_SCRATCH_BYTES;
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_mutex;
void* g_scratch_dev[kMaxDevices] = {nullptr};
uint64_t g_scratch_ctx[kMaxDevices] = {0};  // bpx::context_id() the address was resolved in

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

size_t scratch_bytes(const bpx_options* o, size_t nvox, bool own_status) {
  const size_t np = (size_t)bpx_nparams_fit(o), ns = (size_t)bpx_nsamples(o);
  return align256(nvox * np * 4) + align256(nvox * 4) + align256((size_t)BPX_NREC(o->nfibres) * ns * nvox * 4) +
         (own_status ? align256(nvox * 4) : 0) + align256(nvox * bpx::kFitScratchBytes);
}

// The array's device address on the current device, resolved on first use (cudaGetSymbolAddress
// loads the module that holds the array, which is when the device memory behind it is taken).
bpx_status scratch_address(void** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    bpx::set_last_error("bpx_xfibres_noalloc_dev: no usable CUDA device");
    return BPX_ERR_NO_DEVICE;
  }
  std::lock_guard<std::mutex> lk(g_mutex);
  // an address resolved in an earlier context (before a cudaDeviceReset) is re-resolved
  if (!g_scratch_dev[dev] || g_scratch_ctx[dev] != bpx::context_id()) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      const std::string msg = std::string("bpx_xfibres_noalloc_dev: cudaGetSymbolAddress failed: ") +
                              cudaGetErrorString(e);
      bpx::set_last_error(msg.c_str());
      return BPX_ERR_CUDA;
    }
    g_scratch_dev[dev] = p;
    g_scratch_ctx[dev] = bpx::context_id();
  }
  *out = g_scratch_dev[dev];
  return BPX_OK;
}

}  // namespace

extern "C" bpx_status bpx_xfibres_noalloc_dev(const bpx_options* opts, const bpx_volume* vol, bpx_outputs* out,
                                              void* stream) {
  // every argument check of bpx_xfibres_dev, before anything touches the device or the caller's data
  bpx_status st = bpx::api_check_opts(opts);
  if (st == BPX_OK) st = bpx::api_check_vol(vol);
  if (st != BPX_OK) return st;
  if (!out) return bpx::api_fail(BPX_ERR_INVALID_ARG, "out is NULL");
  if (bpx_nsamples(opts) < 1) return bpx::api_fail(BPX_ERR_INVALID_ARG, "no samples (njumps < sampleevery)");
  st = bpx::api_check_device();
  if (st != BPX_OK) return st;
  // a call with nvox == 0 still resolves the array: it is the warm-up call that makes the library
  // take the array's device memory before the caller reserves its own pool
  void* base = nullptr;
  st = scratch_address(&base);
  if (st != BPX_OK || vol->nvox == 0) return st;
  const bool own_status = out->status == nullptr;
  const size_t need = scratch_bytes(opts, (size_t)vol->nvox, own_status);
  if (need > kScratchBytes) {
    size_t lo = 0, hi = (size_t)vol->nvox;  // largest voxel count that fits
    while (lo < hi) {
      const size_t mid = (lo + hi + 1) / 2;
      if (scratch_bytes(opts, mid, own_status) <= kScratchBytes)
        lo = mid;
      else
        hi = mid - 1;
    }
    const std::string msg = "bpx_xfibres_noalloc_dev: " + std::to_string(vol->nvox) + " voxels need " +
                            std::to_string(need) + " bytes of scratch; the allocation-free entry holds " +
                            std::to_string(kScratchBytes) + " bytes, i.e. at most " + std::to_string(lo) +
                            " voxels for these options";
    bpx::set_last_error(msg.c_str());
    return BPX_ERR_UNSUPPORTED;
  }
  const size_t nvox = (size_t)vol->nvox;
  const size_t np = (size_t)bpx_nparams_fit(opts), ns = (size_t)bpx_nsamples(opts);
  char* p = (char*)base;
  float* params = (float*)p;
  p += align256(nvox * np * 4);
  float* tau = (float*)p;
  p += align256(nvox * 4);
  float* rec = (float*)p;
  p += align256((size_t)BPX_NREC(opts->nfibres) * ns * nvox * 4);
  uint32_t* status = own_status ? (uint32_t*)p : out->status;
  if (own_status) p += align256(nvox * 4);
  void* fit_scratch = p;
  if (opts->rician) st = bpx_prepare_data_dev(vol->nvox, vol->ndir, const_cast<float*>(vol->data), stream);
  if (st == BPX_OK) st = bpx::fit_dev_scratch(opts, vol, params, tau, status, fit_scratch, stream);
  if (st == BPX_OK) st = bpx_mcmc_dev(opts, vol, params, tau, rec, status, stream);
  if (st == BPX_OK) st = bpx_finish_dev(opts, vol->nvox, rec, out, stream);
  return st;
}
