// Instantiations of the line-FFT pass kernel: the first inverse pass gathering Gut rows from k-space.
#include "mlg_fft_kernels.cuh"

namespace mlg {

int fft_dispatch_gut_in(const FftAxisPlan& a, const PassDesc& d, int L, cudaStream_t s) {
  return dispatch_size<1, PassMode::kGutIn>(a, d, L, s);
}

}  // namespace mlg
