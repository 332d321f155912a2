// Instantiations of the line-FFT pass kernel: the inverse x pass fused with .* KFC_conj and the coil sum.
#include "mlg_fft_kernels.cuh"

namespace mlg {

int fft_dispatch_nakatsha_out(const FftAxisPlan& a, const PassDesc& d, int L, cudaStream_t s) {
  return dispatch_size<1, PassMode::kNakatshaOut>(a, d, L, s);
}

}  // namespace mlg
