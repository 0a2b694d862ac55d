// bpx_internal.h -- launch descriptors shared by the kernels and the C-ABI layer.
#pragma once

#include <cstdint>
#include <string>
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include "bpx.h"

namespace bpx {

// Names a host-side stage for profilers (Nsight Systems shows the range and the kernels launched
// inside it); NVTX v3 is header-only and costs a few instructions when no tool is attached.
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

constexpr int kFitThreads = 128;   // 4 warps, one voxel per warp at a time
constexpr int kFitVoxPerBlock = 32;  // voxels a fit block shares out among its warps
#ifndef BPX_FIT_MIN_BLOCKS
#define BPX_FIT_MIN_BLOCKS 4
#endif
constexpr int kFitMinBlocks = BPX_FIT_MIN_BLOCKS;  // register cap: 65536 / (128 * 4) = 128 per thread
constexpr int kMcmcThreads = 128;  // 4 warps
// Register cap of the MCMC kernel as resident blocks per SM: 4 (128 registers, 16 warps) for up to
// 9 measurements per lane, 3 (168 registers, 12 warps) for more, where 128 registers spill in the
// proposal loop.  BPX_MCMC_MIN_BLOCKS overrides both.
template <int MPL>
constexpr int mcmc_min_blocks() {
#ifdef BPX_MCMC_MIN_BLOCKS
  return BPX_MCMC_MIN_BLOCKS;
#else
  return MPL <= 9 ? 4 : 3;
#endif
}

int sm_count();  // multiprocessors of the current device (cached per device)
// Unique id of the CUDA context current on this thread (cuCtxGetId), 0 if none is current or the
// driver lacks the call.  Per-device caches of device addresses (workspaces, the error word, the
// allocation-free array) store it and treat a different id as a new context (after
// cudaDeviceReset the old addresses are gone and must be neither used nor freed).
uint64_t context_id();
void set_last_error(const char* msg);  // message returned by bpx_last_error() on this thread

// C-ABI helpers shared by the entry-point files (bpx_api.cu): status with message, device and
// argument checks, and the grow-only per-device workspaces (one per slot, so that a pipeline
// stage can hold one while calling a stage that uses another).
constexpr int kWorkspaceSlots = 5;
constexpr int kWsPipeline = 0;  // fit parameters, tau, records, status of bpx_xfibres_dev
constexpr int kWsNetwork = 1;   // the network's weights and activations
constexpr int kWsLearned = 2;   // intermediates of the learned pipeline
constexpr int kWsFit = 3;       // FP64 parameters between the fit stages
constexpr int kWsTrack = 4;     // the tracking kernel's per-thread visit tables
bpx_status api_fail(bpx_status st, const std::string& msg);
bpx_status api_cuda_fail(cudaError_t e, const char* where);
bpx_status api_check_device();
bpx_status api_check_opts(const bpx_options* o);
bpx_status api_check_vol(const bpx_volume* v);
bpx_status api_workspace(int slot, size_t bytes, void** out);
// bpx_fit_dev with caller-provided stage scratch (nvox * kFitScratchBytes, 8-byte aligned)
bpx_status fit_dev_scratch(const bpx_options* opts, const bpx_volume* vol, float* params, float* tau, uint32_t* status,
                           void* scratch, void* stream);

struct FitArgs {
  int nvox, ndir;
  const float* data;
  const float* bvecs;
  const float* bvals;
  int gradnonlin;
  float* params;
  int np_out;
  float* tau;
  uint32_t* status;
  int model, rician, nonlin;
  float R;
  double* scratch;   // [nvox][16] FP64 parameters between the fit stages (kFitScratchBytes per voxel)
  uint32_t* flags;   // [nvox] stage flags (within kFitScratchBytes)
};
constexpr size_t kFitScratchBytes = 16 * sizeof(double) + sizeof(uint32_t);  // per voxel

struct McmcArgs {
  int nvox, ndir;
  const float* data;
  const float* bvecs;
  const float* bvals;
  int gradnonlin;
  const float* params;
  int np_fit;
  const float* tau;
  float* records;  // [nrec][nsamples][nvox]
  int nsamples;
  uint32_t* status;
  int nburn, njumps, sampleevery, upe;
  int f0, ardf0, no_ard, all_ard;
  float fudge, R_mean, R_std, R_fudge;
  uint64_t seed, voxel_offset;
  const float* props_in;  // [6+3K][nvox] initial proposal widths, or NULL for initialise_props
  float* props_out;       // [6+3K][nvox] proposal widths after the last iteration, or NULL
  int freeze_props;       // 0: adapt (reference); 1: never adapt; 2: adapt during burn-in only
  const uint64_t* voxel_keys;  // [nvox] RNG voxel keys (packed batches), or NULL: voxel_offset + v
  // a stretch of the chain: iterations [it_begin, it_end) (it_end 0: to the end), started from
  // state_in [6+3K][nvox] (record rows) and acc_in [6+3K][nvox] when given; the state, acceptance
  // counts since the last width update and widths at it_end go to state_out / acc_out / props_out
  int it_begin, it_end;
  const float* state_in;
  float* state_out;
  const int32_t* acc_in;
  int32_t* acc_out;
};

struct EnergyArgs {
  int nvox, ndir;
  const float* data;
  const float* bvecs;
  const float* bvals;
  int gradnonlin;
  const float* states;  // [nvox][BPX_NSTATE]
  float* lik;
  float* prior;
  int f0, ardf0, no_ard, all_ard;
  float fudge, R_mean, R_std, R_fudge;
};

struct FinishArgs {
  int nvox, nsamples, nfib;
  const float* records;
  bpx_outputs out;
};

struct PostArgs {
  int nvox, nsamples, nfib;
  const float* th;      // [K][ns][nvox] (finished, fibres sorted)
  const float* ph;
  const float* mean_f;  // [K][nvox]
  const float* dyads;   // [K][3][nvox]
  float thr;
  bpx_postproc post;
};

// Launch layout of the MCMC kernel: TPV lanes per voxel, at most MPL measurements per lane.
struct McmcLayout {
  int tpv, mpl;
};

// the initialiser network's forward pass on caller buffers (weights copy of mlp_weight_elems
// bf16 values, two activation buffers of chunk_rows x 256 bf16); bpx_mlp.cu
size_t mlp_weight_elems(int ndir);
bpx_status mlp_forward_buffers(int ndir, const float* params, int nvox, const uint16_t* x, float* out, uint16_t* wbf,
                               uint16_t* buf0, uint16_t* buf1, int chunk_rows, cudaStream_t s);

cudaError_t launch_fit(const FitArgs& a, int nfib, bool f0, cudaStream_t s);
cudaError_t launch_prepare(int nvox, int ndir, float* data, cudaStream_t s);
cudaError_t launch_mcmc(const McmcArgs& a, int model, int nfib, bool rician, McmcLayout lay, cudaStream_t s);
McmcLayout choose_layout(int model, int nfib, bool rician, int ndir);
bool layout_supported(int model, int nfib, bool rician, McmcLayout lay);
cudaError_t launch_energy(const EnergyArgs& a, int model, int nfib, bool rician, cudaStream_t s);
cudaError_t launch_finish(const FinishArgs& a, cudaStream_t s);
cudaError_t launch_postproc(const PostArgs& a, cudaStream_t s);

}  // namespace bpx
