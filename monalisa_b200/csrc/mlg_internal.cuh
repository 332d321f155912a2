// Internal declarations shared by the libmonalisa_gpu translation units.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <cufft.h>

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/monalisa_gpu.h"

namespace mlg {

// NVTX range over a host scope: profilers (Nsight Systems, ncu --nvtx) show
// the operator stages and solver phases by name; without a tool attached the
// calls return at once.
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};


// ---- status / error plumbing ----------------------------------------------
void set_error(const char* fmt, ...);
int fail(int status, const char* fmt, ...);
const char* cuda_name(cudaError_t e);

extern std::atomic<long long> g_launches;
inline void count_launch(long long n = 1) { g_launches.fetch_add(n, std::memory_order_relaxed); }

#define MLG_CUDA(call)                                                                  \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess) {                                                            \
      return ::mlg::fail(e_ == cudaErrorMemoryAllocation ? MLG_ERR_OOM : MLG_ERR_CUDA,  \
                         "%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_)); \
    }                                                                                   \
  } while (0)

#define MLG_CUFFT(call)                                                                 \
  do {                                                                                  \
    cufftResult r_ = (call);                                                            \
    if (r_ != CUFFT_SUCCESS) {                                                          \
      return ::mlg::fail(r_ == CUFFT_ALLOC_FAILED ? MLG_ERR_OOM : MLG_ERR_CUDA,         \
                         "%s:%d %s: cufft status %d", __FILE__, __LINE__, #call, (int)r_); \
    }                                                                                   \
  } while (0)

#define MLG_CHECK(cond, ...)                              \
  do {                                                    \
    if (!(cond)) return ::mlg::fail(MLG_ERR_ARG, __VA_ARGS__); \
  } while (0)

#define MLG_TRY(expr)            \
  do {                           \
    int s_ = (expr);             \
    if (s_ != MLG_OK) return s_; \
  } while (0)

// After a launch: records a launch and checks the launch configuration.
#define MLG_LAUNCHED()                                                   \
  do {                                                                   \
    ::mlg::count_launch();                                               \
    cudaError_t e_ = cudaGetLastError();                                 \
    if (e_ != cudaSuccess)                                               \
      return ::mlg::fail(MLG_ERR_CUDA, "%s:%d launch: %s", __FILE__, __LINE__, \
                         cudaGetErrorString(e_));                        \
  } while (0)

int ensure_device();  // MLG_ERR_NO_DEVICE if no usable GPU

// ---- device buffers -------------------------------------------------------
// Stream-ordered allocation from the device's default memory pool (kept
// warm: the release threshold is raised once per device).
int dev_alloc(void** p, size_t bytes, cudaStream_t s);
void dev_free(void* p, cudaStream_t s);

template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  cudaStream_t s = nullptr;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { reset(); }
  int alloc(size_t count, cudaStream_t stream) {
    reset();
    s = stream;
    n = count;
    if (count == 0) return MLG_OK;
    return dev_alloc(reinterpret_cast<void**>(&p), count * sizeof(T), stream);
  }
  void reset() {
    if (p) dev_free(p, s);
    p = nullptr;
    n = 0;
  }
  T* release() {
    T* q = p;
    p = nullptr;
    n = 0;
    return q;
  }
};

// ---- device CSR -----------------------------------------------------------
// Absolute-index CSR with a dense row pointer over all l_size rows (rows the
// jump format squeezes out are empty).  Long rows (more than kLongRow
// entries) are listed separately so that one CTA can split them.
constexpr int kLongRow = 256;
// rows with more than kMidRow (and at most kLongRow) entries are gathered by
// a warp each inside the operators (measured on Gut: 16, 32, 64, 128 entries
// gave 0.797 / 0.769 / 0.757 / 0.749 ms on the 4096-spoke 16-coil koosh
// case and 0.243 / 0.233 / 0.228 / 0.266 ms on a 1500-spoke 12-coil one)
constexpr int kMidRow = 64;

struct Csr {
  int r_size = 0;         // number of columns
  int l_size = 0;         // number of rows
  long long nnz = 0;
  uint32_t* row_ptr = nullptr;  // [l_size + 1]
  int* col = nullptr;           // [nnz]
  float* val = nullptr;         // [nnz]
  int* long_rows = nullptr;     // rows with > kLongRow entries
  int n_long = 0;
  int n_nonempty = 0;
  // long rows cut into segments of at most kSegLen entries: segment i covers
  // entries [seg_lo[i], seg_hi[i]); long row j owns segments
  // [long_seg0[j], long_seg0[j+1])
  uint32_t* seg_lo = nullptr;
  uint32_t* seg_hi = nullptr;
  int* long_seg0 = nullptr;
  int n_seg = 0;
  // non-empty rows in ascending order and a bitmask over all rows (bit r of
  // word r/32 set when row r has entries); built on demand by
  // csr_build_nonempty
  int* nz_rows = nullptr;
  uint32_t* nz_mask = nullptr;
  // a processing order of the rows for the coil-pair products: row
  // ord_rows[i] holds entries [ord_bounds[i].x, ord_bounds[i].y); the rows
  // are the non-empty ones (ord_nonempty) or all rows, sorted so that
  // consecutive rows touch a compact block of grid cells (csr_build_order)
  int* ord_rows = nullptr;
  uint2* ord_bounds = nullptr;
  int n_ord = 0;
  bool ord_nonempty = false;
  // non-empty order only: the first ord_short rows have at most kMidRow
  // entries, the rest more (each part in block order); -1: not split
  int ord_short = -1;
  // FP16 copy of val for the mixed-precision solver (built on demand)
  __half* val_h = nullptr;
  // Row records of the first ord_short ordered rows (sign-folded copies
  // inside plans, csr_build_records): 8 words per row -- cell, entry count,
  // then up to kRecInline (column, value bits) pairs; a longer row stores
  // its first entry index in word 2 and keeps its entries in the CSR
  uint32_t* ord_rec = nullptr;
};
constexpr int kRecInline = 3;

#ifdef __CUDACC__
// Scale of a mixed-precision intermediate stored in FP16: a power of two s
// with bound * s < 2^15 (< 65504), bound = 2 len amax >= any component of a
// length-len transform (or of a product of transforms whose lengths
// multiply to len) of values whose components are at most amax (the writer
// of those values recorded amax; writer and reader compute the same s).
__device__ __forceinline__ float half_store_scale(const unsigned* amax, int len) {
  const float bound = __uint_as_float(__ldg(amax)) * (float)len * 2.0f;
  if (!(bound > 0.f) || !(bound < 1e38f)) return 1.f;
  int e;
  frexpf(bound, &e);  // bound < 2^e
  return ldexpf(1.f, 15 - e);
}
#endif
constexpr int kSegLen = 512;

void csr_free(Csr& c);
// Builds ord_rec from ord_rows / ord_bounds and this matrix's values
// (idempotent; needs the split non-empty order).
int csr_build_records(Csr& c, cudaStream_t s);

// Builds the segment tables of the long rows (call once the long-row list is
// on the device).
int csr_build_segments(Csr& c, cudaStream_t s);
// Builds nz_rows / nz_mask (idempotent).
int csr_build_nonempty(Csr& c, cudaStream_t s);
// Builds ord_rows / ord_bounds (idempotent): the non-empty rows (nonempty;
// rows are cells of the grid N) or all rows (rows keyed by the cell of their
// first entry; empty rows last), in order of 8 x 8 x 8 bricks of cells, x
// fastest within a brick; ties keep row order.  Needs nz_rows for nonempty.
int csr_build_order(Csr& c, const int* N, bool nonempty, cudaStream_t s);

}  // namespace mlg

struct mlg_matrix_s {
  mlg::Csr csr;
  int device = 0;
};

namespace mlg {

// Builds a Csr from host jump-format arrays (validated).  With nBlock > 0
// the matrix is in the multi-block form of bmSparseMat.m:100-188: the running
// column sum restarts at each block's first entry m_block_start[b] and the
// running row sum at each block's first stored row l_block_start[b]
// (block_length[b] rows each); nBlock = 0 is the one-block form.
int csr_from_jump(int r_size, const int* r_jump, const int* r_nJump, const float* m_val, int l_size,
                  const int* l_jump, int l_nJump, Csr& out, cudaStream_t s, int nBlock = 0,
                  const int* block_length = nullptr, const int* l_block_start = nullptr,
                  const long long* m_block_start = nullptr);
// Finishes a Csr whose row_ptr/col/val are already on the device: lists the
// long rows and counts the non-empty ones.
int csr_index_long_rows(Csr& c, cudaStream_t s);
// Copies `src` with each value multiplied by +1/-1 per row (row_sign) or per
// column (col_sign), sign(i) = (-1)^(x+y+z) of linear cell index i on grid N.
int csr_sign_copy(const Csr& src, bool by_row, int imDim, const int* N, float global_sign, Csr& dst,
                  cudaStream_t s);
// Frees a copy made by csr_sign_copy (only its values are owned).
void csr_free_sign_copy(Csr& c);
// Adds the FP16 copy of the values (val_h) if absent.
int csr_make_half(Csr& c, cudaStream_t s);

// ---- SpMM kernels (mlg_sparsemat.cu) ---------------------------------------
// Element layouts of the dense operands.
enum class Layout : int {
  kPointC64 = 0,   // float2 [rows][nCh]          (coil fastest, interleaved)
  kCoilC64 = 1,    // float2 [nCh][rows]          (coil major, interleaved)
  kCoilSplit = 2,  // float re[nCh][rows], im[...] (MATLAB column layout)
  kPointSplit = 3, // float re[rows][nCh], im[...] (MATLAB point layout)
  kCoilReal = 4,   // float [nCh][rows]           (real, column layout)
  kPointReal = 5,  // float [rows][nCh]           (real, row layout)
};

struct Operand {
  Layout layout = Layout::kPointC64;
  void* a = nullptr;        // float2* or float* (re)
  void* b = nullptr;        // im (split layouts)
  long long rows = 0;       // leading dimension for coil-major layouts
};

struct SpmmArgs {
  const Csr* m = nullptr;
  int nCh = 1;
  Operand in;
  Operand out;
  const float* in_row_scale = nullptr;  // multiplies input row j (e.g. HY)
  float out_scale = 1.0f;
  // Optional per-row normalisation (bmGridder_n2u): divides each output row
  // by the sum of its weights, 1 if that sum is < 1e-5.
  bool normalize = false;
  // Optional FP64 partial sums of sum_rows w_row * |out|^2 (w = row weight,
  // NULL = 1): one double per CTA written to partial[], count in *n_partial.
  const float* sqn_row_weight = nullptr;
  double* partial = nullptr;
  // Only the rows longer than kLongRow (the CTA-split kernel); the others are
  // left untouched (a fused consumer gathers them itself).
  bool long_only = false;
  // Per-segment partial sums of the long rows: >= spmm_scratch_floats()
  // floats.  NULL: spmm allocates them (not allowed during stream capture).
  float* seg_scratch = nullptr;
  // Only the non-empty rows (m->nz_rows, which must exist) are computed and
  // written; the others are left untouched.
  bool nonempty_only = false;
  // Read the matrix values from m->val_h (FP16) instead of m->val; the sums
  // stay FP32.
  bool half_values = false;
  // Short rows of an ordered non-empty product from the matrix's row
  // records (ord_rec), when built (FP32 values, rounded to FP16 as read with
  // half_values)
  bool records = false;
  // Optional: raised (atomicMax on the bits) to the largest |re| or |im| of
  // the values written, before any FP16 rounding (device, non-negative float)
  unsigned* absmax = nullptr;
  // Optional: the input (point layout, even nCh) holds __half2 values times
  // half_store_scale(in_half_amax, in_half_len) (the mixed-precision forward
  // grid); coil-pair products of rows without long rows only
  const unsigned* in_half_amax = nullptr;
  int in_half_len = 0;
  // Contracted arithmetic for the coil-pair rows (operators inside plans):
  // the row scale folded into the matrix value (m * HY_j) and fused
  // multiply-adds.  Off (the default): separate round-to-nearest multiply and
  // add in stored order, bit-identical to the reference's CPU products.
  bool contract = false;
};

// Scratch floats spmm needs for the long-row segments of `m` at nCh coils.
size_t spmm_scratch_floats(const Csr& m, int nCh);

int spmm(const SpmmArgs& a, cudaStream_t s);
// Number of FP64 partial sums spmm writes for this matrix / mapping.
int spmm_partial_count(const SpmmArgs& a);

// Deterministic final reduction of partial sums: out[0] = sum partial[0..n).
int reduce_partials(const double* partial, int n, double* out, cudaStream_t s);

// Tables of the deapodisation (bmK.m:6-156) shared by the host and device
// computations (mlg_deapod.cpp): support weights w[az][ay][ax] (S, Sy, Sz
// samples per axis) and cosine tables c_d[j][a] (all ones along absent
// axes), grid N, clip K_max.
struct DeapodTables {
  int imDim = 1;
  int N[3] = {1, 1, 1};
  int S = 1, Sy = 1, Sz = 1;
  double K_max = 0.0;
  std::vector<double> w, cx, cy, cz;
};
int deapod_tables(int imDim, const int* N_u, int kernelType, int nWin, const double* kernelParam, DeapodTables& T);

}  // namespace mlg
