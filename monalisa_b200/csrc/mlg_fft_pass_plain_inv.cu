// Instantiations of the line-FFT pass kernel: inverse plain passes.
#include "mlg_fft_kernels.cuh"

namespace mlg {

int fft_dispatch_plain_inv(const FftAxisPlan& a, const PassDesc& d, int L, cudaStream_t s) {
  return dispatch_size<1, PassMode::kPlain>(a, d, L, s);
}

}  // namespace mlg
