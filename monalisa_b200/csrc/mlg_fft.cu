// Pruned, fused line-FFT passes (see mlg_fft.cuh): host side -- axis tables
// and the per-pass dispatch into the instantiations of mlg_fft_pass_*.cu.
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "mlg_fft_kernels.cuh"

namespace mlg {

bool tma_passes_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("MLG_FFT_TMA");
    return !(e && std::strcmp(e, "0") == 0);
  }();
  return on;
}

bool tma_test_stall() {
  static const bool on = [] {
    const char* e = std::getenv("MLG_TEST_WAIT_TIMEOUT");
    return e && std::strcmp(e, "1") == 0;
  }();
  return on;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library)
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

int* fft_wait_word() {
  static std::mutex mu;
  static int* words[128] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 128) return nullptr;
  std::lock_guard<std::mutex> lk(mu);
  if (!words[dev]) {
    int* w = nullptr;
    if (cudaMalloc(&w, sizeof(int)) != cudaSuccess || cudaMemset(w, 0, sizeof(int)) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    words[dev] = w;
  }
  return words[dev];
}

int fft_wait_status(int* word, cudaStream_t s) {
  if (!word) return MLG_OK;
  int h = 0;
  MLG_CUDA(cudaMemcpyAsync(&h, word, sizeof(int), cudaMemcpyDeviceToHost, s));
  MLG_CUDA(cudaStreamSynchronize(s));
  if (h == 0) return MLG_OK;
  MLG_CUDA(cudaMemsetAsync(word, 0, sizeof(int), s));
  MLG_CUDA(cudaStreamSynchronize(s));
  return fail(MLG_ERR_TIMEOUT, "a bounded wait inside a line-FFT pass ran out; results of the work since the last "
                               "check are invalid");
}

int tma_line_map(CUtensorMap* map, const void* base, int C, int dim_u, long long st_u, int len, long long st_ax,
                 int dim_v, long long st_v, int box_L, int box_rows, bool half) {
  auto enc = tensor_map_encoder();
  MLG_CHECK(enc != nullptr, "cuTensorMapEncodeTiled is not available");
  MLG_CHECK(((uintptr_t)base & 15) == 0, "TMA volume base not 16-byte aligned");
  MLG_CHECK(C >= 1 && 2 * C <= 256 && box_L >= 1 && box_L <= 256 && box_rows >= 1 && box_rows <= 256,
            "TMA box out of range");
  const cuuint64_t dims[4] = {(cuuint64_t)2 * C, (cuuint64_t)dim_u, (cuuint64_t)len, (cuuint64_t)dim_v};
  const cuuint64_t es = half ? 4 : 8;  // bytes per complex value
  const cuuint64_t strides[3] = {(cuuint64_t)st_u * es, (cuuint64_t)st_ax * es, (cuuint64_t)st_v * es};
  for (int i = 0; i < 3; ++i)
    MLG_CHECK(strides[i] % 16 == 0 && strides[i] < (1ull << 40), "TMA stride %llu not a multiple of 16 bytes",
              (unsigned long long)strides[i]);
  const cuuint32_t box[4] = {(cuuint32_t)(2 * C), (cuuint32_t)box_L, (cuuint32_t)box_rows, 1};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  MLG_CHECK(!half || (4 * C) % 16 == 0, "FP16 boxes need a multiple of 4 coils");
  const CUresult r = enc(map, half ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4,
                         const_cast<void*>(base), dims, strides, box, estr,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  MLG_CHECK(r == CUDA_SUCCESS, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return MLG_OK;
}

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
