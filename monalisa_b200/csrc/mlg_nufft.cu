// Fused NUFFT operators.
//
// bmShanna (src/fourier123/map_function/nonCartesian/bmShanna_MATLAB.m:28-54):
//   x .* KFC -> zero-fill n_u -> N_u -> fftshift(fft(ifftshift)) -> Gu
// bmNakatsha (bmNakatsha_MATLAB.m:32-56):
//   Gut -> fftshift(ifft(ifftshift)) -> crop -> .* KFC_conj -> coil sum
//
// Gridded data are coil-fastest [cell][coil]: a grid cell's coils share one
// 128-byte line, which is what the Gu / Gut gathers read or write per matrix
// entry.  The transforms are this library's pruned line-FFT passes
// (mlg_fft.cu): the forward runs x, y, z passes where each pass only
// transforms the lines that can be non-zero and zero-fills on load (the
// zero-filled n_u block never exists in memory); the inverse runs z, y, x
// passes that keep only the lines of the cropped n_u block.  x .* KFC and the
// input modulation are fused into the first forward pass, .* KFC_conj, the
// output modulation, the 1/prod(N) scaling and the coil sum into the last
// inverse pass.
//
// For even N the centred transform is a modulated plain DFT:
//   fftshift(F(ifftshift(v)))[k] = (-1)^k (-1)^(N/2) F((-1)^n v)[k]
// (same for the inverse).  The input modulation of the forward is fused into
// the x pass and its output modulation folded into the column signs of Gu;
// the inverse's input modulation is folded into the row signs of Gut and its
// output modulation fused into the last pass.
#include <algorithm>
#include <vector>

#include "mlg_plan.cuh"

namespace mlg {

constexpr int kEwThreads = 256;

static int ew_grid(long long n) {
  return (int)std::max<long long>(1, std::min<long long>((n + kEwThreads - 1) / kEwThreads, 148LL * 16));
}

// element strides (float2 units) of a coil-fastest box with extents e[3]
static void box_strides(const int e[3], int C, long long st[3]) {
  st[0] = C;
  st[1] = (long long)C * e[0];
  st[2] = (long long)C * e[0] * e[1];
}

// The last forward pass may store only the chunks of grid lines that hold
// cells Gu reads (plan variant fwd_masked_store; the line masks of the
// masked adjoint cover every Gu column when gu_covered).
static void set_masked_store(const mlg_plan_s* p, PassDesc& pd) {
  if (p->fwd_masked_store && p->gu_covered && p->line_mask) {
    pd.out_lmask = p->line_mask;
    pd.lmask_words = p->line_mask_words;
  }
}

// Forward passes: x (image -> A), y (A -> B), z (B -> grid).  The last pass
// of the transform writes the grid.  half (3-D): B in scaled FP16 -- the x
// pass records max|A| in mix_amax[0], the y pass stores B times the power of
// two that bounds a length-n[1] transform of it below 2^15, the z pass reads
// it back; dry: check only (PassDesc::dry).
static int forward_pass(mlg_plan_s* p, int ax, const float2* x, bool x_per_coil, cudaStream_t s, bool half = false,
                        bool dry = false, bool half_grid = false) {
  const int C = p->nCh, d = p->imDim;
  const int* N = p->N;
  const int* n = p->n;
  const int eA[3] = {N[0], n[1], n[2]};
  const int eB[3] = {N[0], N[1], n[2]};
  const int eG[3] = {N[0], N[1], N[2]};
  PassDesc pd;
  pd.ax = ax;
  pd.dir = -1;
  pd.C = C;
  pd.wait_err = p->wait_err;
  pd.tma_slots = p->pass_buffers;
  pd.dry = dry ? 1 : 0;
  if (half) {
    pd.h_amax = p->mix_amax;
    pd.h_len = n[1];
  }
  if (ax == 0) {
    if (half) pd.out_absmax = p->mix_amax;
    pd.dims[1] = n[1];
    pd.dims[2] = n[2];
    pd.in_lo = p->off[0];
    pd.in_len = n[0];
    pd.img = x;
    pd.img_per_coil = x_per_coil ? 1 : 0;
    pd.kfc = p->KFC;
    for (int k = 0; k < 3; ++k) pd.coord_off[k] = p->off[k];
    pd.out = d == 1 ? p->grid : p->bufA;
    box_strides(d == 1 ? eG : eA, C, pd.out_stride);
    pd.out_lo = 0;
    pd.out_len = N[0];
    return fft_pass(p->ax[0], PassMode::kShannaIn, pd, nullptr, s);
  }
  if (ax == 1) {
    pd.dims[0] = N[0];
    pd.dims[2] = n[2];
    pd.in = p->bufA;
    box_strides(eA, C, pd.in_stride);
    pd.in_lo = p->off[1];
    pd.in_len = n[1];
    pd.out = d == 2 ? p->grid : p->bufB;
    box_strides(d == 2 ? eG : eB, C, pd.out_stride);
    pd.out_lo = 0;
    pd.out_len = N[1];
    pd.out_half = half ? 1 : 0;
    if (d == 2) set_masked_store(p, pd);
    return fft_pass(p->ax[1], PassMode::kPlain, pd, nullptr, s);
  }
  pd.dims[0] = N[0];
  pd.dims[1] = N[1];
  pd.in_half = half ? 1 : 0;
  if (half_grid) {  // the grid in FP16 too: |grid| <= 2 n_y n_z max|A|
    pd.out_half = 1;
    pd.h_len_out = n[1] * n[2];
  }
  pd.in = p->bufB;
  box_strides(eB, C, pd.in_stride);
  pd.in_lo = p->off[2];
  pd.in_len = n[2];
  pd.out = p->grid;
  box_strides(eG, C, pd.out_stride);
  pd.out_lo = 0;
  pd.out_len = N[2];
  set_masked_store(p, pd);
  return fft_pass(p->ax[2], PassMode::kPlain, pd, nullptr, s);
}

// Inverse passes: z (grid -> B), y (B -> A), x (A -> image, coil sum).  In 2-D
// and 3-D the first pass does not read a grid at all: it gathers the Gut rows
// of its cells from k-space itself (kGutIn), so the adjoint never writes or
// reads the full grid; only rows longer than kLongRow were computed into the
// grid buffer beforehand.  In 1-D the first pass is also the last one and
// reads the grid written by the Gut product.
enum : int { kAdjFullGrid = 0, kAdjFused = 1, kAdjMasked = 2 };

static bool fused_gut(const mlg_plan_s* p) { return p->adjoint_mode == kAdjFused; }

// adjoint variants a plan can run
bool adjoint_mode_valid(const mlg_plan_s* p, int mode) {
  if (mode == kAdjFullGrid) return true;
  // the fused gather reads FP32 k-space and FP32 values inside the FFT pass:
  // FP32 plans only
  if (mode == kAdjFused) return p->imDim >= 2 && p->precision == MLG_PRECISION_FP32;
  if (mode == kAdjMasked)
    return (p->nCh % 2) == 0 && p->Gut_s.nz_mask != nullptr && p->Gut_s.ord_rows != nullptr && p->Gut_s.ord_nonempty;
  return false;
}

static void set_gut_input(mlg_plan_s* p, PassDesc& pd, const float2* y, const float* HY) {
  pd.g_rowptr = p->Gut_s.row_ptr;
  pd.g_col = p->Gut_s.col;
  pd.g_val = p->Gut_s.val;
  pd.g_hy = HY;
  pd.g_y = y;
  pd.g_long = p->grid;
  pd.cell_stride[0] = 1;
  pd.cell_stride[1] = p->N[0];
  pd.cell_stride[2] = (long long)p->N[0] * p->N[1];
}

// half (3-D): B in scaled FP16 -- the Gut product records max|grid| in
// mix_amax[1], the z pass stores B times the power of two that bounds a
// length-N[2] transform of it below 2^15, the y pass reads it back; dry:
// check only (PassDesc::dry).
static int inverse_pass(mlg_plan_s* p, int ax, const float2* y, const float* HY, float scale, float2* x,
                        double* partial, int* n_partial, cudaStream_t s, bool half = false, bool dry = false) {
  const int C = p->nCh, d = p->imDim;
  const int* N = p->N;
  const int* n = p->n;
  const int eA[3] = {N[0], n[1], n[2]};
  const int eB[3] = {N[0], N[1], n[2]};
  const int eG[3] = {N[0], N[1], N[2]};
  PassDesc pd;
  pd.ax = ax;
  pd.dir = 1;
  pd.C = C;
  pd.wait_err = p->wait_err;
  pd.tma_slots = p->pass_buffers;
  pd.dry = dry ? 1 : 0;
  if (half) {
    pd.h_amax = p->mix_amax + 1;
    pd.h_len = N[2];
  }
  const bool gut_in = fused_gut(p) && ax == d - 1;
  if (gut_in) set_gut_input(p, pd, y, HY);
  if (p->adjoint_mode == kAdjMasked && ax == d - 1) {
    pd.in_mask = p->Gut_s.nz_mask;
    pd.in_lmask = p->line_mask;
    pd.lmask_words = p->line_mask_words;
    pd.cell_stride[0] = 1;
    pd.cell_stride[1] = p->N[0];
    pd.cell_stride[2] = (long long)p->N[0] * p->N[1];
  }
  const PassMode plain = gut_in ? PassMode::kGutIn : PassMode::kPlain;
  if (ax == 2) {
    pd.dims[0] = N[0];
    pd.dims[1] = N[1];
    pd.in = p->grid;
    box_strides(eG, C, pd.in_stride);
    pd.in_lo = 0;
    pd.in_len = N[2];
    pd.out = p->bufB;
    box_strides(eB, C, pd.out_stride);
    pd.out_lo = p->off[2];
    pd.out_len = n[2];
    pd.out_half = half ? 1 : 0;
    return fft_pass(p->ax[2], plain, pd, nullptr, s);
  }
  if (ax == 1) {
    pd.dims[0] = N[0];
    pd.dims[2] = n[2];
    pd.in = d == 2 ? p->grid : p->bufB;
    box_strides(d == 2 ? eG : eB, C, pd.in_stride);
    pd.in_half = half ? 1 : 0;
    pd.in_lo = 0;
    pd.in_len = N[1];
    pd.out = p->bufA;
    box_strides(eA, C, pd.out_stride);
    pd.out_lo = p->off[1];
    pd.out_len = n[1];
    return fft_pass(p->ax[1], plain, pd, nullptr, s);
  }
  pd.dims[1] = n[1];
  pd.dims[2] = n[2];
  pd.in = d == 1 ? p->grid : p->bufA;
  box_strides(d == 1 ? eG : eA, C, pd.in_stride);
  pd.in_lo = 0;
  pd.in_len = N[0];
  pd.out_lo = p->off[0];
  pd.out_len = n[0];
  pd.img_out = x;
  pd.kfc = p->KFCc;
  for (int k = 0; k < 3; ++k) pd.coord_off[k] = p->off[k];
  pd.sfac = (float)((double)p->shift_const / (double)p->Nu_tot * (double)scale);
  pd.partial = partial;
  return fft_pass(p->ax[0], PassMode::kNakatshaOut, pd, n_partial, s);
}

// Whether the CG steps of a mixed solve keep bufB in FP16: a 3-D plan, a
// coil count whose FP16 cells fill 16-byte TMA rows, no fused Gut gather (it
// reads FP32), and a dry run of the four passes accepted by their kernels.
// Cached per (pass_buffers, adjoint_mode), the plan state the pass kernels
// depend on.
bool half_intermediate_possible(mlg_plan_s* p) {
  if (p->imDim != 3 || (p->nCh % 4) != 0 || fused_gut(p)) return false;
  const int key = p->pass_buffers * 8 + p->adjoint_mode;
  if (p->half_b_key == key) return p->half_b_ok;
  // the maxima's words are not read by a dry run; any non-null address will do
  unsigned* const words = p->mix_amax;
  unsigned dummy[2];
  if (!words) p->mix_amax = dummy;
  bool ok = true;
  for (int ax = 0; ax < 3 && ok; ++ax) ok = forward_pass(p, ax, nullptr, false, nullptr, true, true) == MLG_OK;
  for (int ax = 2; ax >= 1 && ok; --ax)
    ok = inverse_pass(p, ax, nullptr, nullptr, 1.f, nullptr, nullptr, nullptr, nullptr, true, true) == MLG_OK;
  // the forward grid in FP16 as well: the z pass storing FP16, Gu's coil-pair
  // gathers reading it (even coil count, no long rows)
  const bool ok_g = ok && (p->nCh % 2) == 0 && p->Gu && p->Gu_s.n_long == 0 &&
                    forward_pass(p, 2, nullptr, false, nullptr, true, true, true) == MLG_OK;
  p->mix_amax = words;
  p->half_b_key = key;
  p->half_b_ok = ok;
  p->half_g_ok = ok_g;
  return ok;
}

static bool half_b(mlg_plan_s* p) { return p->cg_half && p->mix_amax && half_intermediate_possible(p); }

int shanna_stage(mlg_plan_s* p, int stage, const float2* x, bool x_per_coil, float2* y, const float* sqn_w,
                 double* partial, int* n_partial, cudaStream_t s) {
  if (stage < 3) {
    if (stage >= p->imDim) return MLG_OK;
    const bool half = half_b(p);
    if (half && stage == 0) MLG_CUDA(cudaMemsetAsync(p->mix_amax, 0, sizeof(unsigned), s));
    return forward_pass(p, stage, x, x_per_coil, s, half, false, half && p->half_g_ok);
  }
  SpmmArgs a;
  a.m = &p->Gu_s;
  a.nCh = p->nCh;
  a.in.layout = Layout::kPointC64;
  a.in.a = p->grid;
  a.in.rows = p->Nu_tot;
  a.out.layout = Layout::kPointC64;
  if (half_b(p) && p->half_g_ok) {  // the forward grid stored in FP16 by the z pass
    a.in_half_amax = p->mix_amax;
    a.in_half_len = p->n[1] * p->n[2];
  }
  a.half_values = p->precision != MLG_PRECISION_FP32;
  a.contract = true;  // operator-internal product: fused multiply-adds
  a.out.a = y;
  a.out.rows = p->nPt;
  a.sqn_row_weight = sqn_w;
  a.partial = partial;
  a.seg_scratch = p->seg_scratch;
  if (n_partial) *n_partial = partial ? spmm_partial_count(a) : 0;
  return spmm(a, s);
}

// stage 0: the Gut product into the grid buffer -- all rows (kAdjFullGrid),
// the non-empty rows (kAdjMasked) or only the long rows (kAdjFused, whose
// first pass gathers the rest itself); stages 1..imDim: inverse passes over
// the last, ..., first dimension
int nakatsha_stage(mlg_plan_s* p, int stage, const float2* y, const float* HY, float scale, float2* x,
                   double* partial, int* n_partial, cudaStream_t s) {
  if (stage == 0) {
    if (fused_gut(p) && p->Gut_s.n_long == 0) return MLG_OK;
    // the masked variant leaves empty rows stale: the pass never reads them
    SpmmArgs a;
    a.m = &p->Gut_s;
    a.nCh = p->nCh;
    a.in.layout = Layout::kPointC64;  // the solver's residual stays FP32 in every precision
    a.half_values = p->precision != MLG_PRECISION_FP32;
    a.contract = true;  // HY folded into the matrix values, fused multiply-adds
    a.in.a = const_cast<float2*>(y);
    a.in.rows = p->nPt;
    a.in_row_scale = HY;
    a.out.layout = Layout::kPointC64;
    a.out.a = p->grid;
    a.out.rows = p->Nu_tot;
    a.long_only = fused_gut(p);
    a.nonempty_only = p->adjoint_mode == kAdjMasked;
    a.records = p->gut_records != 0;
    a.seg_scratch = p->seg_scratch;
    if (half_b(p)) {
      MLG_CUDA(cudaMemsetAsync(p->mix_amax + 1, 0, sizeof(unsigned), s));
      a.absmax = p->mix_amax + 1;
    }
    return spmm(a, s);
  }
  const int ax = p->imDim - stage;
  if (ax < 0) return MLG_OK;
  return inverse_pass(p, ax, y, HY, scale, x, partial, n_partial, s, ax >= 1 && half_b(p));
}

int shanna_run(mlg_plan_s* p, const float2* x, bool x_per_coil, float2* y, const float* sqn_w, double* partial,
               int* n_partial, cudaStream_t s) {
  static const char* kNames[kShannaStages] = {"shanna: x pass (x.*KFC)", "shanna: y pass", "shanna: z pass",
                                              "shanna: Gu"};
  NvtxRange r("shanna");
  for (int st = 0; st < kShannaStages; ++st) {
    NvtxRange rs(kNames[st]);
    MLG_TRY(shanna_stage(p, st, x, x_per_coil, y, sqn_w, partial, n_partial, s));
  }
  return MLG_OK;
}

int nakatsha_run(mlg_plan_s* p, const float2* y, const float* HY, float scale, float2* x, double* partial,
                 int* n_partial, cudaStream_t s) {
  static const char* kNames[kNakatshaStages] = {"nakatsha: Gut", "nakatsha: last-axis pass", "nakatsha: middle pass",
                                                "nakatsha: x pass (.*KFC_conj, coil sum)"};
  NvtxRange r("nakatsha");
  for (int st = 0; st < kNakatshaStages; ++st) {
    NvtxRange rs(kNames[st]);
    MLG_TRY(nakatsha_stage(p, st, y, HY, scale, x, partial, n_partial, s));
  }
  return MLG_OK;
}

// ---- layout conversion kernels ----------------------------------------------
// split [rows, nCh] column layout <-> float2 point layout [rows][nCh]
__global__ void pack_col_to_point_kernel(const float* __restrict__ re, const float* __restrict__ im, long long rows,
                                         int nCh, float2* __restrict__ out) {
  const long long n = rows * nCh;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const long long r = i / nCh;
    const int c = (int)(i - r * nCh);
    out[i] = make_float2(re[(long long)c * rows + r], im ? im[(long long)c * rows + r] : 0.f);
  }
}

__global__ void unpack_point_to_col_kernel(const float2* __restrict__ in, long long rows, int nCh,
                                           float* __restrict__ re, float* __restrict__ im) {
  const long long n = rows * nCh;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(i / rows);
    const long long r = i - (long long)c * rows;
    const float2 v = in[r * nCh + c];
    re[i] = v.x;
    im[i] = v.y;
  }
}

// split -> interleaved (same element order)
__global__ void interleave_kernel(const float* __restrict__ re, const float* __restrict__ im, long long n,
                                  float2* __restrict__ out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = make_float2(re[i], im ? im[i] : 0.f);
}

__global__ void deinterleave_kernel(const float2* __restrict__ in, long long n, float* __restrict__ re,
                                    float* __restrict__ im) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float2 v = in[i];
    re[i] = v.x;
    im[i] = v.y;
  }
}

int pack_col_to_point(const float* re, const float* im, long long rows, int nCh, float2* out, cudaStream_t s) {
  pack_col_to_point_kernel<<<ew_grid(rows * nCh), kEwThreads, 0, s>>>(re, im, rows, nCh, out);
  MLG_LAUNCHED();
  return MLG_OK;
}
int unpack_point_to_col(const float2* in, long long rows, int nCh, float* re, float* im, cudaStream_t s) {
  unpack_point_to_col_kernel<<<ew_grid(rows * nCh), kEwThreads, 0, s>>>(in, rows, nCh, re, im);
  MLG_LAUNCHED();
  return MLG_OK;
}
int interleave(const float* re, const float* im, long long n, float2* out, cudaStream_t s) {
  interleave_kernel<<<ew_grid(n), kEwThreads, 0, s>>>(re, im, n, out);
  MLG_LAUNCHED();
  return MLG_OK;
}
int deinterleave(const float2* in, long long n, float* re, float* im, cudaStream_t s) {
  deinterleave_kernel<<<ew_grid(n), kEwThreads, 0, s>>>(in, n, re, im);
  MLG_LAUNCHED();
  return MLG_OK;
}

// Line masks of the masked first inverse pass: word w of line (ui, vi) holds
// the occupancy bits of cells ui*cu + vi*cv + n*cax, n = 32w .. 32w+31.
__global__ void line_mask_kernel(const uint32_t* __restrict__ nz, int du, int dv, long long cu, long long cv,
                                 long long cax, int Nax, int LW, uint32_t* __restrict__ lm) {
  const long long total = (long long)du * dv * LW;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long line = i / LW;
    const int w = (int)(i - line * LW);
    const long long base = (line % du) * cu + (line / du) * cv;
    uint32_t m = 0;
    for (int j = 0; j < 32 && w * 32 + j < Nax; ++j) {
      const long long cell = base + (long long)(w * 32 + j) * cax;
      m |= ((nz[cell >> 5] >> (cell & 31)) & 1u) << j;
    }
    lm[i] = m;
  }
}

// 1 in *miss when a Gu column (a grid cell Gu reads) is not an occupied cell
// of Gut's occupancy bits.
__global__ void cover_check_kernel(const int* __restrict__ col, long long nnz, const uint32_t* __restrict__ nz,
                                   int* miss) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nnz; k += (long long)gridDim.x * blockDim.x) {
    const int c = __ldg(col + k);
    if (!((__ldg(nz + (c >> 5)) >> (c & 31)) & 1u)) *miss = 1;
  }
}

// Whether the line masks cover every cell Gu reads (Gu and Gut of one
// trajectory are transposes, so they do; matrices from elsewhere may not).
static int check_gu_covered(mlg_plan_s* p, cudaStream_t s) {
  p->gu_covered = false;
  if (!p->line_mask || !p->Gu || !p->Gut_s.nz_mask || p->Gu_s.nnz == 0) return MLG_OK;
  DevBuf<int> miss;
  MLG_TRY(miss.alloc(1, s));
  MLG_CUDA(cudaMemsetAsync(miss.p, 0, sizeof(int), s));
  cover_check_kernel<<<ew_grid(p->Gu_s.nnz), kEwThreads, 0, s>>>(p->Gu_s.col, p->Gu_s.nnz, p->Gut_s.nz_mask, miss.p);
  MLG_LAUNCHED();
  int h = 1;
  MLG_CUDA(cudaMemcpyAsync(&h, miss.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  MLG_CUDA(cudaStreamSynchronize(s));
  p->gu_covered = h == 0;
  return MLG_OK;
}

// Geometry as inverse_pass sets it for axis imDim - 1 (2-D and 3-D; in 1-D
// that pass is the fused x pass, which reads the occupancy mask itself).
static int build_line_mask(mlg_plan_s* p, cudaStream_t s) {
  if (!p->Gut_s.nz_mask || p->imDim < 2) return MLG_OK;
  const int ax = p->imDim - 1;
  const int du = p->N[0];
  const int dv = ax == 2 ? p->N[1] : p->n[2];
  const long long cs[3] = {1, p->N[0], (long long)p->N[0] * p->N[1]};
  const int v = ax == 2 ? 1 : 2;
  const int LW = ((p->N[ax] + 31) / 32 + 3) / 4 * 4;
  const long long total = (long long)du * dv * LW;
  MLG_CUDA(cudaMalloc(&p->line_mask, sizeof(uint32_t) * (size_t)total));
  p->line_mask_words = LW;
  line_mask_kernel<<<ew_grid(total), kEwThreads, 0, s>>>(p->Gut_s.nz_mask, du, dv, cs[0], cs[v], cs[ax], p->N[ax], LW,
                                                         p->line_mask);
  MLG_LAUNCHED();
  return MLG_OK;
}

// ---- plan lifecycle ---------------------------------------------------------
static void plan_free(mlg_plan_s* p) {
  if (!p) return;
  cudaSetDevice(p->device);
  if (p->borrowed && p->stream) cudaStreamSynchronize(p->stream);  // the owner's stream stays alive
  if (p->owner) --p->owner->n_borrowers;
  if (p->cg_graph) cudaGraphExecDestroy(p->cg_graph);
  csr_free_sign_copy(p->Gu_s);
  csr_free_sign_copy(p->Gut_s);
  if (!p->borrowed) {
    for (int d = 0; d < 3; ++d) fft_axis_free(p->ax[d]);
    cudaFree(p->KFC);
    cudaFree(p->KFCc);
    cudaFree(p->grid);
    cudaFree(p->bufA);
    cudaFree(p->bufB);
    if (p->ev_in) cudaEventDestroy(p->ev_in);
    if (p->ev_out) cudaEventDestroy(p->ev_out);
    if (p->stream) cudaStreamDestroy(p->stream);
  }
  cudaFree(p->partial);
  cudaFree(p->seg_scratch);
  cudaFree(p->line_mask);
  cudaFree(p->mix_amax);
  cudaFree(p->scalars);
  cudaFree(p->x_p);
  cudaFree(p->x_dagM);
  cudaFree(p->k_res);
  cudaFree(p->k_Mp);
  cudaFree(p->HY);
  delete p;
}

void plan_destroy(mlg_plan_s* p) { plan_free(p); }

// KFC / KFC_conj arrive as [prod(n_u), nCh] column layout (separate real and
// imaginary parts, host memory) and are stored coil-fastest.
static int upload_kfc(const float* re, const float* im, long long nu, int nCh, float2* dst, cudaStream_t s) {
  const long long nk = nu * nCh;
  if (!re) {
    MLG_CUDA(cudaMemsetAsync(dst, 0, sizeof(float2) * (size_t)nk, s));
    return MLG_OK;
  }
  DevBuf<float> tmp;
  MLG_TRY(tmp.alloc(2 * (size_t)nk, s));
  MLG_CUDA(cudaMemcpyAsync(tmp.p, re, sizeof(float) * nk, cudaMemcpyHostToDevice, s));
  if (im) MLG_CUDA(cudaMemcpyAsync(tmp.p + nk, im, sizeof(float) * nk, cudaMemcpyHostToDevice, s));
  MLG_TRY(pack_col_to_point(tmp.p, im ? tmp.p + nk : nullptr, nu, nCh, dst, s));
  MLG_CUDA(cudaStreamSynchronize(s));
  return MLG_OK;
}

static int plan_create_impl(int imDim, const int* N_u, const int* n_u, int nCh, const Csr* Gu, const Csr* Gut,
                            const float* KFC_re, const float* KFC_im, const float* KFCc_re, const float* KFCc_im,
                            mlg_plan_s** out, const mlg_plan_s* share = nullptr) {
  MLG_CHECK(out, "NULL output");
  *out = nullptr;
  MLG_CHECK(imDim >= 1 && imDim <= 3, "imDim must be 1, 2 or 3");
  MLG_CHECK(N_u && nCh >= 1, "invalid N_u / nCh");
  MLG_CHECK(Gu || Gut, "at least one of Gu / Gut is needed");
  MLG_TRY(ensure_device());
  mlg_plan_s* p = new mlg_plan_s();
  p->borrowed = share != nullptr;
  auto bail = [&](int status) {
    plan_free(p);
    return status;
  };
  cudaGetDevice(&p->device);
  if (share && share->device != p->device)
    return bail(fail(MLG_ERR_ARG, "the shared plan lives on device %d, the current device is %d", share->device,
                     p->device));
  p->imDim = imDim;
  p->nCh = nCh;
  long long Nu = 1, nu = 1;
  float sc = 1.0f;
  for (int d = 0; d < 3; ++d) {
    p->N[d] = d < imDim ? N_u[d] : 1;
    p->n[d] = d < imDim ? (n_u ? n_u[d] : N_u[d]) : 1;
    if (d < imDim) {
      if (p->N[d] < 2 || (p->N[d] & 1) || p->n[d] < 2 || (p->n[d] & 1) || p->n[d] > p->N[d])
        return bail(fail(MLG_ERR_ARG, "N_u and n_u must be even, >= 2, with n_u <= N_u (dim %d: N=%d n=%d)", d,
                         N_u[d], n_u ? n_u[d] : N_u[d]));
      if ((p->N[d] / 2) & 1) sc = -sc;
    }
    p->off[d] = p->N[d] / 2 - p->n[d] / 2;
    Nu *= p->N[d];
    nu *= p->n[d];
  }
  p->Nu_tot = Nu;
  p->nu_tot = nu;
  p->shift_const = sc;
  p->HX = 1.0;  // dK_u = 1 until mlg_plan_set_dk
  for (int d = 0; d < imDim; ++d) {
    p->dX[d] = 1.0f / (float)p->N[d];
    p->HX = (double)((float)p->HX * p->dX[d]);
  }
  if (Gu && Gu->r_size != Nu) return bail(fail(MLG_ERR_ARG, "Gu has %d columns, prod(N_u) = %lld", Gu->r_size, Nu));
  if (Gut && Gut->l_size != Nu) return bail(fail(MLG_ERR_ARG, "Gut has %d rows, prod(N_u) = %lld", Gut->l_size, Nu));
  if (Gu && Gut && Gu->l_size != Gut->r_size)
    return bail(fail(MLG_ERR_ARG, "Gu rows (%d) and Gut columns (%d) differ", Gu->l_size, Gut->r_size));
  p->nPt = Gu ? Gu->l_size : Gut->r_size;
  p->Gu = Gu;
  p->Gut = Gut;
  int st = MLG_OK;
  if (share) {
    for (int d = 0; d < 3; ++d) p->ax[d] = share->ax[d];
    p->stream = share->stream;
    p->ev_in = share->ev_in;
    p->ev_out = share->ev_out;
    p->HX = share->HX;
    for (int d = 0; d < 3; ++d) p->dX[d] = share->dX[d];
  } else {
    for (int d = 0; d < imDim; ++d)
      if ((st = fft_axis_init(p->N[d], p->ax[d])) != MLG_OK) return bail(st);
    if (cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&p->ev_in, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&p->ev_out, cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      return bail(fail(MLG_ERR_CUDA, "stream/event creation failed"));
    }
  }
  cudaStream_t s = p->stream;
  p->wait_err = fft_wait_word();
  if (!p->wait_err) return bail(fail(MLG_ERR_OOM, "plan: the device wait flag could not be allocated"));
  // occupancy tables and the list of Gut's non-empty cells (in blocks of
  // nearby cells) live with the caller's matrix (built once, shared by the
  // sign-folded copy)
  if (Gu && (st = csr_sign_copy(*Gu, false, imDim, p->N, sc, p->Gu_s, s)) != MLG_OK) return bail(st);
  if (Gut && (nCh % 2) == 0 && (st = csr_build_nonempty(const_cast<Csr&>(*Gut), s)) != MLG_OK) return bail(st);
  if (Gut && (nCh % 2) == 0 && (st = csr_build_order(const_cast<Csr&>(*Gut), p->N, true, s)) != MLG_OK)
    return bail(st);
  if (Gut && (st = csr_sign_copy(*Gut, true, imDim, p->N, 1.0f, p->Gut_s, s)) != MLG_OK) return bail(st);
  if (Gut && (nCh % 2) == 0 && nCh / 2 <= 16 && (st = csr_build_records(p->Gut_s, s)) != MLG_OK) return bail(st);
  p->gut_records = p->Gut_s.ord_rec ? 1 : 0;  // measured faster on c2 (0.607 vs 0.671 ms)
  if ((st = build_line_mask(p, s)) != MLG_OK) return bail(st);
  if ((st = check_gu_covered(p, s)) != MLG_OK) return bail(st);
  p->fwd_masked_store = p->gu_covered ? 1 : 0;
  p->adjoint_mode = adjoint_mode_valid(p, kAdjMasked) ? kAdjMasked : (imDim >= 2 ? kAdjFused : kAdjFullGrid);
  const size_t kbytes = sizeof(float2) * (size_t)nu * nCh;
  const size_t gbytes = sizeof(float2) * (size_t)Nu * nCh;
  const size_t abytes = sizeof(float2) * (size_t)p->N[0] * p->n[1] * p->n[2] * nCh;
  const size_t bbytes = sizeof(float2) * (size_t)p->N[0] * p->N[1] * p->n[2] * nCh;
  if (share) {
    p->KFC = share->KFC;
    p->KFCc = share->KFCc;
    p->grid = share->grid;
    p->bufA = share->bufA;
    p->bufB = share->bufB;
  } else {
    if (cudaMalloc(&p->KFC, kbytes) != cudaSuccess || cudaMalloc(&p->KFCc, kbytes) != cudaSuccess ||
        cudaMalloc(&p->grid, gbytes) != cudaSuccess || cudaMalloc(&p->bufA, abytes) != cudaSuccess ||
        cudaMalloc(&p->bufB, bbytes) != cudaSuccess) {
      cudaGetLastError();
      return bail(fail(MLG_ERR_OOM, "plan: device allocation failed"));
    }
    if ((st = upload_kfc(KFC_re, KFC_im, nu, nCh, p->KFC, s)) != MLG_OK) return bail(st);
    if ((st = upload_kfc(KFCc_re, KFCc_im, nu, nCh, p->KFCc, s)) != MLG_OK) return bail(st);
  }
  // partial-sum buffer: the largest CTA count any fused reduction uses
  PassDesc last;
  last.ax = 0;
  last.C = nCh;
  last.dims[1] = p->n[1];
  last.dims[2] = p->n[2];
  int cap = fft_pass_blocks(p->ax[0], last) + 8;
  if (Gu) {
    SpmmArgs a;
    a.m = &p->Gu_s;
    a.nCh = nCh;
    cap = std::max(cap, spmm_partial_count(a));
  }
  cap = std::max(cap, ew_grid((long long)p->nPt * nCh) + 8);
  cap = std::max(cap, 256);  // the solver's two-stage max over ve uses 128 floats
  p->partial_cap = cap;
  const size_t seg_floats = std::max<size_t>(
      1, std::max(Gu ? spmm_scratch_floats(*Gu, nCh) : 0, Gut ? spmm_scratch_floats(*Gut, nCh) : 0));
  if (cudaMalloc(&p->partial, sizeof(double) * (size_t)cap) != cudaSuccess ||
      cudaMalloc(&p->seg_scratch, sizeof(float) * seg_floats) != cudaSuccess ||
      cudaMalloc(&p->scalars, sizeof(double) * 64) != cudaSuccess) {
    cudaGetLastError();
    return bail(fail(MLG_ERR_OOM, "plan: partial buffer allocation failed"));
  }
  if (cudaStreamSynchronize(s) != cudaSuccess) return bail(fail(MLG_ERR_CUDA, "plan creation failed"));
  p->bytes = (share ? 0 : 2 * kbytes + gbytes + abytes + bbytes) +
             sizeof(float) * (size_t)((Gu ? Gu->nnz : 0) + (Gut ? Gut->nnz : 0)) + sizeof(double) * (cap + 64) +
             sizeof(float) * seg_floats + (p->Gut_s.ord_rec ? 32 * (size_t)p->Gut_s.ord_short : 0);
  *out = p;
  return MLG_OK;
}

int plan_create_sharing(const mlg_plan_s* base, const Csr* Gu, const Csr* Gut, mlg_plan_s** out) {
  MLG_CHECK(base && out, "NULL argument");
  MLG_CHECK(!base->borrowed, "share the plan that owns the buffers, not a plan that borrows them");
  MLG_TRY(plan_create_impl(base->imDim, base->N, base->n, base->nCh, Gu, Gut, nullptr, nullptr, nullptr, nullptr, out,
                           base));
  (*out)->owner = const_cast<mlg_plan_s*>(base);
  ++(*out)->owner->n_borrowers;
  return MLG_OK;
}

// Orders the plan's stream after the caller's stream and back.
struct StreamJoin {
  mlg_plan_s* p;
  cudaStream_t user;
  StreamJoin(mlg_plan_s* plan, cudaStream_t u) : p(plan), user(u) {
    cudaEventRecord(p->ev_in, user);
    cudaStreamWaitEvent(p->stream, p->ev_in, 0);
  }
  ~StreamJoin() {
    cudaEventRecord(p->ev_out, p->stream);
    cudaStreamWaitEvent(user, p->ev_out, 0);
  }
};

}  // namespace mlg

using namespace mlg;

extern "C" {

int mlg_plan_create(int imDim, const int* N_u, const int* n_u, int nCh, mlg_matrix_t Gu, mlg_matrix_t Gut,
                    const float* KFC_re, const float* KFC_im, const float* KFCc_re, const float* KFCc_im,
                    mlg_plan_t* out) {
  MLG_CHECK(Gu || Gut, "at least one of Gu / Gut is needed");
  return plan_create_impl(imDim, N_u, n_u, nCh, Gu ? &Gu->csr : nullptr, Gut ? &Gut->csr : nullptr, KFC_re, KFC_im,
                          KFCc_re, KFCc_im, out);
}

int mlg_plan_destroy(mlg_plan_t p) {
  if (p && p->n_borrowers > 0)
    return fail(MLG_ERR_STATE, "%d plan(s) still borrow this plan's buffers: destroy them first", p->n_borrowers);
  plan_free(p);
  return MLG_OK;
}

int mlg_plan_create_sharing(mlg_plan_t base, mlg_matrix_t Gu, mlg_matrix_t Gut, mlg_plan_t* out) {
  MLG_CHECK(base && out, "NULL argument");
  MLG_CHECK(Gu || Gut, "at least one of Gu / Gut is needed");
  MLG_CUDA(cudaSetDevice(base->device));
  return plan_create_sharing(base, Gu ? &Gu->csr : nullptr, Gut ? &Gut->csr : nullptr, out);
}

int mlg_plan_status(mlg_plan_t p) {
  MLG_CHECK(p, "NULL plan");
  MLG_CUDA(cudaSetDevice(p->device));
  return fft_wait_status(p->wait_err, p->stream);
}

int mlg_plan_device_bytes(mlg_plan_t p, long long* bytes) {
  MLG_CHECK(p && bytes, "NULL argument");
  *bytes = (long long)p->bytes;
  return MLG_OK;
}

int mlg_shanna_dev(mlg_plan_t p, const void* x, int x_per_coil, void* y, void* stream) {
  MLG_CHECK(p && x && y, "NULL argument");
  MLG_CHECK(p->Gu, "plan has no Gu");
  MLG_CUDA(cudaSetDevice(p->device));
  StreamJoin j(p, (cudaStream_t)stream);
  return shanna_run(p, (const float2*)x, x_per_coil != 0, (float2*)y, nullptr, nullptr, nullptr, p->stream);
}

int mlg_nakatsha_dev(mlg_plan_t p, const void* y, const float* HY, float scale, void* x, void* stream) {
  MLG_CHECK(p && x && y, "NULL argument");
  MLG_CHECK(p->Gut, "plan has no Gut");
  MLG_CUDA(cudaSetDevice(p->device));
  StreamJoin j(p, (cudaStream_t)stream);
  return nakatsha_run(p, (const float2*)y, HY, scale, (float2*)x, nullptr, nullptr, p->stream);
}

// Stateless host-buffer operators (drop-ins for the CUFFT MEX files).
int mlg_shanna(int imDim, const int* N_u, const int* n_u, int nCh, const float* xR, const float* xI, int x_nCol,
               const float* KFC_R, const float* KFC_I, int r_size, const int* r_jump, const int* r_nJump,
               const float* m_val, int l_size, const int* l_jump, int l_nJump, float* yR, float* yI) {
  MLG_TRY(ensure_device());
  MLG_CHECK(xR && KFC_R && yR && yI, "NULL buffer");
  MLG_CHECK(x_nCol == 1 || x_nCol == nCh, "x must have 1 or nCh columns (got %d, nCh=%d)", x_nCol, nCh);
  mlg_matrix_t G = nullptr;
  MLG_TRY(mlg_matrix_create(r_size, r_jump, r_nJump, m_val, l_size, l_jump, l_nJump, &G));
  mlg_plan_s* p = nullptr;
  int st = plan_create_impl(imDim, N_u, n_u, nCh, &G->csr, nullptr, KFC_R, KFC_I, nullptr, nullptr, &p);
  if (st != MLG_OK) {
    mlg_matrix_destroy(G);
    return st;
  }
  cudaStream_t s = p->stream;
  const long long nx = p->nu_tot * x_nCol, ny = (long long)p->nPt * nCh;
  DevBuf<float> dx, dy;
  DevBuf<float2> x2, y2;
  if (st == MLG_OK) st = dx.alloc(2 * nx, s);
  if (st == MLG_OK) st = x2.alloc(nx, s);
  if (st == MLG_OK) st = y2.alloc(ny, s);
  if (st == MLG_OK) st = dy.alloc(2 * ny, s);
  if (st == MLG_OK) {
    cudaMemcpyAsync(dx.p, xR, sizeof(float) * nx, cudaMemcpyHostToDevice, s);
    if (xI) cudaMemcpyAsync(dx.p + nx, xI, sizeof(float) * nx, cudaMemcpyHostToDevice, s);
    // [prod(n_u), x_nCol] column layout -> [pixel][coil]
    st = pack_col_to_point(dx.p, xI ? dx.p + nx : nullptr, p->nu_tot, x_nCol, x2.p, s);
  }
  if (st == MLG_OK) st = shanna_run(p, x2.p, x_nCol > 1, y2.p, nullptr, nullptr, nullptr, s);
  if (st == MLG_OK) st = unpack_point_to_col(y2.p, p->nPt, nCh, dy.p, dy.p + ny, s);
  if (st == MLG_OK) {
    cudaMemcpyAsync(yR, dy.p, sizeof(float) * ny, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(yI, dy.p + ny, sizeof(float) * ny, cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess)
      st = fail(MLG_ERR_CUDA, "shanna failed: %s", cudaGetErrorString(cudaGetLastError()));
  }
  if (st == MLG_OK) st = fft_wait_status(p->wait_err, s);
  dx.reset();
  dy.reset();
  x2.reset();
  y2.reset();
  cudaStreamSynchronize(s);
  plan_free(p);
  mlg_matrix_destroy(G);
  return st;
}

int mlg_nakatsha(int imDim, const int* N_u, const int* n_u, int nCh, const float* yR, const float* yI,
                 const float* KFCc_R, const float* KFCc_I, int r_size, const int* r_jump, const int* r_nJump,
                 const float* m_val, int l_size, const int* l_jump, int l_nJump, float* xR, float* xI) {
  MLG_TRY(ensure_device());
  MLG_CHECK(yR && yI && KFCc_R && xR && xI, "NULL buffer");
  mlg_matrix_t G = nullptr;
  MLG_TRY(mlg_matrix_create(r_size, r_jump, r_nJump, m_val, l_size, l_jump, l_nJump, &G));
  mlg_plan_s* p = nullptr;
  int st = plan_create_impl(imDim, N_u, n_u, nCh, nullptr, &G->csr, nullptr, nullptr, KFCc_R, KFCc_I, &p);
  if (st != MLG_OK) {
    mlg_matrix_destroy(G);
    return st;
  }
  cudaStream_t s = p->stream;
  const long long ny = (long long)p->nPt * nCh, nx = p->nu_tot;
  DevBuf<float> dy, dx;
  DevBuf<float2> y2, x2;
  if (st == MLG_OK) st = dy.alloc(2 * ny, s);
  if (st == MLG_OK) st = y2.alloc(ny, s);
  if (st == MLG_OK) st = x2.alloc(nx, s);
  if (st == MLG_OK) st = dx.alloc(2 * nx, s);
  if (st == MLG_OK) {
    cudaMemcpyAsync(dy.p, yR, sizeof(float) * ny, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dy.p + ny, yI, sizeof(float) * ny, cudaMemcpyHostToDevice, s);
    st = pack_col_to_point(dy.p, dy.p + ny, p->nPt, nCh, y2.p, s);
  }
  if (st == MLG_OK) st = nakatsha_run(p, y2.p, nullptr, 1.0f, x2.p, nullptr, nullptr, s);
  if (st == MLG_OK) st = deinterleave(x2.p, nx, dx.p, dx.p + nx, s);
  if (st == MLG_OK) {
    cudaMemcpyAsync(xR, dx.p, sizeof(float) * nx, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(xI, dx.p + nx, sizeof(float) * nx, cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess)
      st = fail(MLG_ERR_CUDA, "nakatsha failed: %s", cudaGetErrorString(cudaGetLastError()));
  }
  if (st == MLG_OK) st = fft_wait_status(p->wait_err, s);
  dx.reset();
  dy.reset();
  x2.reset();
  y2.reset();
  cudaStreamSynchronize(s);
  plan_free(p);
  mlg_matrix_destroy(G);
  return st;
}

}  // extern "C"

// ---- inverse DFT (bmIDF{1,2,3}) ----------------------------------------------
namespace mlg {

__global__ void idf_modulate_kernel(const float* __restrict__ re, const float* __restrict__ im, long long Nu,
                                    long long total, int imDim, int Nx, int Ny, float2* __restrict__ out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long cell = i % Nu;
    long long s = cell % Nx;
    if (imDim > 1) {
      const long long q = cell / Nx;
      s += q % Ny;
      if (imDim > 2) s += q / Ny;
    }
    const float sg = (s & 1) ? -1.f : 1.f;
    out[i] = make_float2(re[i] * sg, (im ? im[i] : 0.f) * sg);
  }
}

__global__ void idf_demodulate_kernel(const float2* __restrict__ in, long long Nu, long long total, int imDim, int Nx,
                                      int Ny, float fac, float* __restrict__ re, float* __restrict__ im) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long cell = i % Nu;
    long long s = cell % Nx;
    if (imDim > 1) {
      const long long q = cell / Nx;
      s += q % Ny;
      if (imDim > 2) s += q / Ny;
    }
    const float f = (s & 1) ? -fac : fac;
    re[i] = in[i].x * f;
    im[i] = in[i].y * f;
  }
}

}  // namespace mlg

extern "C" int mlg_idf(int imDim, const int* N_u, const float* dK_u, int nCol, const float* xR, const float* xI,
                       float* yR, float* yI) {
  MLG_TRY(ensure_device());
  MLG_CHECK(imDim >= 1 && imDim <= 3 && N_u && dK_u && nCol >= 1, "invalid argument");
  MLG_CHECK(xR && yR && yI, "NULL buffer");
  long long Nu = 1;
  float sc = 1.f;
  double dk = 1.0;
  int N[3] = {1, 1, 1};
  for (int d = 0; d < imDim; ++d) {
    MLG_CHECK(N_u[d] >= 2 && !(N_u[d] & 1), "N_u must be even and >= 2");
    N[d] = N_u[d];
    Nu *= N_u[d];
    dk *= dK_u[d];
    if ((N_u[d] / 2) & 1) sc = -sc;
  }
  const long long total = Nu * nCol;
  cudaStream_t s = nullptr;
  DevBuf<float> dxs, dys;
  DevBuf<float2> buf;
  MLG_TRY(dxs.alloc(2 * total, s));
  MLG_TRY(buf.alloc(total, s));
  MLG_TRY(dys.alloc(2 * total, s));
  MLG_CUDA(cudaMemcpyAsync(dxs.p, xR, sizeof(float) * total, cudaMemcpyHostToDevice, s));
  if (xI) MLG_CUDA(cudaMemcpyAsync(dxs.p + total, xI, sizeof(float) * total, cudaMemcpyHostToDevice, s));
  idf_modulate_kernel<<<ew_grid(total), kEwThreads, 0, s>>>(dxs.p, xI ? dxs.p + total : nullptr, Nu, total, imDim,
                                                            N[0], N[1], buf.p);
  MLG_LAUNCHED();
  cufftHandle h;
  int n[3];
  for (int d = 0; d < imDim; ++d) n[d] = N[imDim - 1 - d];
  MLG_CUFFT(cufftPlanMany(&h, imDim, n, nullptr, 1, (int)Nu, nullptr, 1, (int)Nu, CUFFT_C2C, nCol));
  cufftSetStream(h, s);
  cufftResult r = cufftExecC2C(h, (cufftComplex*)buf.p, (cufftComplex*)buf.p, CUFFT_INVERSE);
  count_launch();
  if (r != CUFFT_SUCCESS) {
    cufftDestroy(h);
    return fail(MLG_ERR_CUDA, "idf: cufftExecC2C failed (%d)", (int)r);
  }
  // ifft's 1/prod(N) times the reference's single(prod(N_u)*prod(dK_u))
  const float F = (float)((double)Nu * dk);
  const float fac = (float)(sc * (double)F / (double)Nu);
  idf_demodulate_kernel<<<ew_grid(total), kEwThreads, 0, s>>>(buf.p, Nu, total, imDim, N[0], N[1], fac, dys.p,
                                                              dys.p + total);
  MLG_LAUNCHED();
  MLG_CUDA(cudaMemcpyAsync(yR, dys.p, sizeof(float) * total, cudaMemcpyDeviceToHost, s));
  MLG_CUDA(cudaMemcpyAsync(yI, dys.p + total, sizeof(float) * total, cudaMemcpyDeviceToHost, s));
  MLG_CUDA(cudaStreamSynchronize(s));
  cufftDestroy(h);
  return MLG_OK;
}
