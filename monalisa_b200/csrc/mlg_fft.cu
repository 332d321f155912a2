// Pruned, fused line-FFT passes (see mlg_fft.cuh): host side -- axis tables
// and the per-pass dispatch into the instantiations of mlg_fft_pass_*.cu.
#include <algorithm>
#include <cmath>
#include <vector>

#include "mlg_fft_kernels.cuh"

namespace mlg {

int fft_axis_init(int N, FftAxisPlan& a) {
  a = FftAxisPlan();
  MLG_CHECK(N >= 1 && N <= 1024, "FFT length %d outside [1, 1024]", N);
  // N = N1 * N2 with N1 <= N2 <= 32, N1 as large as possible
  int best1 = 0;
  for (int n1 = 1; n1 <= 32; ++n1)
    if (N % n1 == 0 && N / n1 <= 32 && n1 <= N / n1) best1 = n1;
  if (best1 == 0) return fail(MLG_ERR_UNSUPPORTED, "FFT length %d has no factorisation N1*N2 with N1,N2 <= 32", N);
  a.N = N;
  a.N1 = best1;
  a.N2 = N / best1;
  // unrolled register transforms exist for these factor pairs (lengths 2^k
  // and 3 * 2^k from 16 to 1024); other lengths use the runtime DFT
  static const int kFast[] = {404, 408, 808, 816, 1616, 1632, 3232, 608, 812, 1216, 1624, 2432};
  a.fast = false;
  for (int f : kFast) a.fast = a.fast || f == a.N1 * 100 + a.N2;
  std::vector<float2> t(N);
  for (int j = 0; j < N; ++j) {
    const double ang = -2.0 * M_PI * (double)j / (double)N;
    t[j] = make_float2((float)std::cos(ang), (float)std::sin(ang));
  }
  MLG_CUDA(cudaMalloc(&a.tw, sizeof(float2) * N));
  MLG_CUDA(cudaMemcpy(a.tw, t.data(), sizeof(float2) * N, cudaMemcpyHostToDevice));
  return MLG_OK;
}

void fft_axis_free(FftAxisPlan& a) {
  cudaFree(a.tw);
  a = FftAxisPlan();
}

int fft_pass_blocks(const FftAxisPlan& a, const PassDesc& d) {
  return blocks_for(d, lines_per_cta(a, d.C, PassMode::kNakatshaOut));
}

int fft_pass(const FftAxisPlan& a, PassMode mode, const PassDesc& d, int* n_partial, cudaStream_t s) {
  MLG_CHECK(a.N >= 1 && a.tw, "FFT axis not initialised");
  MLG_CHECK(d.C >= 1, "C must be >= 1");
  const int L = lines_per_cta(a, d.C, mode);
  MLG_CHECK((size_t)a.N * L * d.C * sizeof(float2) <= 200 * 1024,
            "FFT line of %d points x %d coils exceeds shared memory", a.N, d.C);
  if (n_partial) *n_partial = mode == PassMode::kNakatshaOut && d.partial ? blocks_for(d, L) : 0;
  switch (mode) {
    case PassMode::kShannaIn:
      MLG_CHECK(d.ax == 0 && d.dir < 0, "kShannaIn is a forward x pass");
      return fft_dispatch_shanna_in(a, d, L, s);
    case PassMode::kNakatshaOut:
      MLG_CHECK(d.ax == 0 && d.dir > 0, "kNakatshaOut is an inverse x pass");
      return fft_dispatch_nakatsha_out(a, d, L, s);
    case PassMode::kGutIn:
      MLG_CHECK(d.dir > 0 && d.g_rowptr && d.g_y, "kGutIn is an inverse pass over Gut");
      return fft_dispatch_gut_in(a, d, L, s);
    default:
      return d.dir < 0 ? fft_dispatch_plain_fwd(a, d, L, s) : fft_dispatch_plain_inv(a, d, L, s);
  }
}

}  // namespace mlg
