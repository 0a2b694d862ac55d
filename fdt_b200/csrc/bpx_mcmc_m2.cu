// bpx_mcmc_m2.cu -- instantiations of the MCMC and energy kernels for model 2.
#include "bpx_mcmc_impl.cuh"

namespace bpx {

cudaError_t launch_mcmc_m2(const McmcArgs& a, int nfib, bool ric, McmcLayout lay, cudaStream_t s) {
  return launch_mcmc_model<2>(a, nfib, ric, lay, s);
}

cudaError_t launch_energy_m2(const EnergyArgs& a, int nfib, bool ric, McmcLayout lay, cudaStream_t s) {
  return launch_energy_model<2>(a, nfib, ric, lay, s);
}

}  // namespace bpx
