// Pruned, fused line-FFT passes over coil-fastest volumes (mlg_fft.cu).
//
// A volume is float2 [z][y][x][c] (coils fastest).  One pass transforms every
// line along one axis; the line lives on the full axis [0, N) but the input
// buffer only holds [in_lo, in_lo + in_len) of it (the rest is zero) and
// the output buffer only keeps [out_lo, out_lo + out_len).  Zero-filling and
// cropping therefore cost nothing, and the centred-DFT modulation, the coil
// maps (x .* KFC on the way in, .* KFC_conj + coil sum on the way out) are
// fused into the first / last pass.
#pragma once

#include "mlg_internal.cuh"

namespace mlg {

enum class PassMode : int {
  kPlain = 0,        // zero-filled load, cropped store
  kShannaIn = 1,     // load x .* KFC .* (-1)^(x+y+z) from the image (axis x)
  kNakatshaOut = 2,  // store sum_c s .* KFC_conj (coil sum) into the image (axis x)
  kGutIn = 3,        // load grid cells as Gut rows gathered from k-space (first inverse pass)
};

struct FftAxisPlan {
  int N = 0, N1 = 0, N2 = 0;  // N = N1 * N2, both <= 32
  bool fast = false;          // templated power-of-two path
  float2* tw = nullptr;       // exp(-2 pi i j / N), j < N (device)
};

struct PassDesc {
  int ax = 0;                     // FFT axis
  int dir = -1;                   // -1 forward (e^-i), +1 inverse (unnormalised)
  int C = 1;                      // coils
  int dims[3] = {1, 1, 1};        // line grid: extents of the non-FFT axes (dims[ax] unused)
  const float2* in = nullptr;
  float2* out = nullptr;
  long long in_stride[3] = {0, 0, 0};   // in float2 units, coil stride 1
  long long out_stride[3] = {0, 0, 0};
  int in_lo = 0, in_len = 0, out_lo = 0, out_len = 0;
  // fusion (kShannaIn / kNakatshaOut); image is [n_z][n_y][n_x], KFC [pix][c]
  const float2* img = nullptr;
  int img_per_coil = 0;
  const float2* kfc = nullptr;
  float2* img_out = nullptr;
  int coord_off[3] = {0, 0, 0};   // full-grid coordinate of line-grid index 0 (sign)
  float sfac = 1.0f;              // kNakatshaOut scale (sign applied per element)
  double* partial = nullptr;      // kNakatshaOut: FP64 |x|^2 per CTA
  // kGutIn: cell (u, v, n) of the full grid is row u*cs[u] + v*cs[v] + n*cs[ax]
  // of Gut (rows already carry the (-1)^cell modulation); rows longer than
  // kLongRow were computed beforehand into g_long ([cell][c], the grid buffer)
  const uint32_t* g_rowptr = nullptr;
  const int* g_col = nullptr;
  const float* g_val = nullptr;
  const float* g_hy = nullptr;    // row weights of y (NULL = 1)
  const float2* g_y = nullptr;    // k-space [nPt][C]
  const float2* g_long = nullptr;
  long long cell_stride[3] = {0, 0, 0};
  // kPlain: when set, input cell (u, v, n) (index via cell_stride) is read
  // only if its bit is set and is zero otherwise (cells a sparse product left
  // unwritten)
  const uint32_t* in_mask = nullptr;
  // the same bits regrouped per line (optional, with in_mask): bit n of word
  // n / 32 of line ui + dims[u] * vi, lmask_words words per line (a multiple
  // of 4); the pipelined pass fetches them ahead of the line copies
  const uint32_t* in_lmask = nullptr;
  int lmask_words = 0;
  // device word set to 1 when a bounded wait inside a pass runs out (passes
  // with such waits: the TMA passes), or NULL
  int* wait_err = nullptr;
  // bundle buffers of the TMA passes (2 or 3; the plan's variant), or 0:
  // the cp.async passes even where a TMA pass exists
  int tma_slots = 2;
  // FP16 storage of a pass intermediate (mixed precision): the input
  // (in_half, TMA passes) or output (out_half, TMA and cp.async plain passes)
  // volume holds __half2 values times a power of two from h_amax / h_len
  // (half_store_scale); out_absmax (optional, the pipelined forward x pass):
  // raised to the largest component the pass stores (FP32 output).  A pass
  // shape whose kernel lacks a requested one fails with MLG_ERR_UNSUPPORTED.
  int in_half = 0, out_half = 0;
  const unsigned* h_amax = nullptr;
  int h_len = 1;
  int h_len_out = 0;  // with both in_half and out_half: the output's h_len (0: h_len)
  unsigned* out_absmax = nullptr;
  // check only: MLG_OK when a kernel would run the pass with every field
  // above honoured, MLG_ERR_UNSUPPORTED otherwise; nothing is launched
  int dry = 0;
  // optional, the last forward pass: line masks (the geometry of in_lmask,
  // lmask_words words per line) of the output cells that will be read; a TMA
  // pass then stores only the 32-row chunks that hold such a cell, other
  // kernels store everything
  const uint32_t* out_lmask = nullptr;
};

// The current device's wait flag (set by a pass whose bounded wait ran out),
// allocated on first use -- call it outside stream capture.
int* fft_wait_word();
// Synchronises s, then reads and clears *word: MLG_OK, or MLG_ERR_TIMEOUT
// when a pass's wait ran out since the last check.
int fft_wait_status(int* word, cudaStream_t s);

// Whether the TMA passes may run at all (MLG_FFT_TMA=0 turns them off for
// every plan; otherwise PassDesc::tma_slots decides per pass).
bool tma_passes_enabled();

int fft_axis_init(int N, FftAxisPlan& a);
void fft_axis_free(FftAxisPlan& a);
// Launches one pass; *n_partial receives the CTA count when partial sums are
// written (kNakatshaOut).
int fft_pass(const FftAxisPlan& a, PassMode mode, const PassDesc& d, int* n_partial, cudaStream_t s);
// CTA count of a pass (for partial-sum buffer sizing).
int fft_pass_blocks(const FftAxisPlan& a, const PassDesc& d);

}  // namespace mlg
