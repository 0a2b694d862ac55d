// bpx_mcmc_m1.cu -- instantiations of the MCMC and energy kernels for model 1.
#include "bpx_mcmc_impl.cuh"

namespace bpx {

cudaError_t launch_mcmc_m1(const McmcArgs& a, int nfib, bool ric, McmcLayout lay, cudaStream_t s) {
  return launch_mcmc_model<1>(a, nfib, ric, lay, s);
}

cudaError_t launch_energy_m1(const EnergyArgs& a, int nfib, bool ric, McmcLayout lay, cudaStream_t s) {
  return launch_energy_model<1>(a, nfib, ric, lay, s);
}

}  // namespace bpx
