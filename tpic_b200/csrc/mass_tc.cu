// Tensor-core (tcgen05) mass-matrix assembly forms. Placeholder until the
// tcgen05 kernels land: the TF32 and BF16x3 selections are rejected.
#include "kernels.cuh"

namespace tpicb200 {

cudaError_t launch_deposit_tc(int, const Geom&, double, double, double, const tpicb200_particles*,
                              const uint32_t*, const uint32_t*, const void*, void*, void*, uint32_t*,
                              cudaStream_t) {
  return cudaErrorNotSupported;
}

}  // namespace tpicb200
