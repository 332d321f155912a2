// Instantiations of the line-FFT pass kernel: the forward x pass fused with x .* KFC.
#include "mlg_fft_kernels.cuh"

namespace mlg {

int fft_dispatch_shanna_in(const FftAxisPlan& a, const PassDesc& d, int L, cudaStream_t s) {
  return dispatch_size<-1, PassMode::kShannaIn>(a, d, L, s);
}

}  // namespace mlg
