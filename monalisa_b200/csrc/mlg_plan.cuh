// Internal NUFFT plan shared by the operator (mlg_nufft.cu) and solver
// (mlg_solver.cu) translation units.
#pragma once

#include "mlg_fft.cuh"
#include "mlg_internal.cuh"

struct mlg_plan_s {
  int device = 0;
  int imDim = 3;
  int N[3] = {1, 1, 1};    // grid (N_u)
  int n[3] = {1, 1, 1};    // image (n_u)
  int off[3] = {0, 0, 0};  // N/2 - n/2: where the image block sits in the grid
  int nCh = 1;
  long long Nu_tot = 1, nu_tot = 1;
  int nPt = 0;             // rows of Gu
  // fftshift as modulation: the centred DFT equals (-1)^k * c * DFT((-1)^n x)
  // with c = prod_d (-1)^(N_d/2)
  float shift_const = 1.0f;
  const mlg::Csr* Gu = nullptr;   // caller's matrices
  const mlg::Csr* Gut = nullptr;
  mlg::Csr Gu_s;                  // values x (-1)^(col cell) x shift_const
  mlg::Csr Gut_s;                 // values x (-1)^(row cell)
  float2* KFC = nullptr;          // [nu][nCh]
  float2* KFCc = nullptr;         // [nu][nCh]
  float2* grid = nullptr;         // [Nu][nCh] (coil fastest)
  float2* bufA = nullptr;         // [n_z][n_y][N_x][nCh]
  float2* bufB = nullptr;         // [n_z][N_y][N_x][nCh]
  mlg::FftAxisPlan ax[3];
  double* partial = nullptr;      // FP64 partial sums (CTA results)
  int partial_cap = 0;
  float* seg_scratch = nullptr;   // long-row segment partials of Gu / Gut
  // How the adjoint feeds its first inverse pass:
  //  0 kAdjFullGrid: Gut writes every grid cell, the pass streams the grid;
  //  1 kAdjFused:    the pass gathers Gut rows from k-space itself (2-D/3-D);
  //  2 kAdjMasked:   Gut writes only its non-empty rows, the pass reads a
  //                  cell only when its occupancy bit is set (even nCh).
  int adjoint_mode = 0;
  // Gut's occupancy bits regrouped per line of the first inverse pass (axis
  // imDim - 1): line_mask_words words per line (built with the occupancy
  // tables, for kAdjMasked)
  uint32_t* line_mask = nullptr;
  int line_mask_words = 0;
  double* scalars = nullptr;      // solver scalars (device)
  int* wait_err = nullptr;        // the device's pass wait flag (fft_wait_word, not owned)
  // kernel variants chosen per plan (mlg_plan_autotune_variants): line-FFT
  // bundles moved by the TMA unit through 2 or 3 shared buffers per CTA
  // (pass_buffers = 2, 3) or by per-thread cp.async copies (0); Gut's short
  // rows from row records (1, when built) or from the CSR (0); the last
  // forward pass storing only the 32-row chunks that hold cells Gu reads
  // (fwd_masked_store = 1; allowed when gu_covered: every Gu column is an
  // occupied cell of the line masks, checked once at plan creation)
  int pass_buffers = 2;
  int gut_records = 0;
  int fwd_masked_store = 0;
  bool gu_covered = false;
  cudaStream_t stream = nullptr;  // internal non-blocking stream
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  size_t bytes = 0;
  // solver work vectors, allocated on first use
  float2 *x_p = nullptr, *x_dagM = nullptr, *k_res = nullptr, *k_Mp = nullptr;
  float* HY = nullptr;
  int solver_nPt = 0;
  // HX = prod(dX_u), dX_u = (1/dK_u)/N_u (bmSensa.m:26-27), single precision
  double HX = 1.0;
  float dX[3] = {1.f, 1.f, 1.f};
  // captured inner CG step (replayed nCGD-1 times per outer iteration)
  cudaGraphExec_t cg_graph = nullptr;
  const void* cg_graph_x = nullptr;  // solution buffer baked into the graph
  long long cg_graph_kernels = 0;
  // A plan created from another one (same grid, image, coils and KFC, other
  // matrices) borrows that plan's KFC, KFCc, grid, bufA, bufB, FFT tables,
  // stream and events; both then run in the order of that one stream.
  bool borrowed = false;
  // MLG_PRECISION_FP32, _MIXED (FP16 matrix values and, inside the CG
  // steps, the FP16 transform intermediate) or _FP16_VALUES; mixed_run is set
  // while a mixed solve runs, cg_half while its CG steps run
  int precision = 0;
  bool mixed_run = false;
  bool cg_half = false;
  // FP16 storage of bufB (the y / z pass intermediate of a 3-D transform)
  // while cg_half is set, where every pass involved supports it: mix_amax[0]
  // = largest component of the forward x pass's output, mix_amax[1] = of the
  // Gut product (two device words, allocated with the solver buffers), the
  // bounds of the FP16 scales; half_b_key / half_b_ok cache the dry-run check
  // of the four passes per (pass_buffers, adjoint_mode)
  unsigned* mix_amax = nullptr;
  int half_b_key = -1;
  bool half_b_ok = false;
  // with half_b_ok: the forward grid in FP16 too (the last forward pass
  // stores it, Gu reads it; the same key)
  bool half_g_ok = false;
  int cg_graph_prec = -1;  // precision the captured CG step was built for
  mlg_plan_s* owner = nullptr;  // the plan whose buffers are borrowed
  int n_borrowers = 0;          // plans borrowing this one's buffers
};

namespace mlg {

// stages of the two operators (stage timing helper uses them one by one)
constexpr int kShannaStages = 4;    // x, y, z passes, Gu
constexpr int kNakatshaStages = 4;  // Gut, z, y, x passes
int shanna_stage(mlg_plan_s* p, int stage, const float2* x, bool x_per_coil, float2* y, const float* sqn_w,
                 double* partial, int* n_partial, cudaStream_t s);
int nakatsha_stage(mlg_plan_s* p, int stage, const float2* y, const float* HY, float scale, float2* x,
                   double* partial, int* n_partial, cudaStream_t s);
bool adjoint_mode_valid(const mlg_plan_s* p, int mode);
// whether the plan's passes take bufB in FP16 (mixed CG steps; host check)
bool half_intermediate_possible(mlg_plan_s* p);
int shanna_run(mlg_plan_s* p, const float2* x, bool x_per_coil, float2* y, const float* sqn_w, double* partial,
               int* n_partial, cudaStream_t s);
int nakatsha_run(mlg_plan_s* p, const float2* y, const float* HY, float scale, float2* x, double* partial,
                 int* n_partial, cudaStream_t s);
int sensa_run(mlg_plan_s* p, const float2* y, const float* ve, float ve_max, int nIter, int nCGD, float2* x,
              double* residual, bool use_graph, cudaStream_t s);
// a plan over other matrices that borrows base's buffers (see `borrowed`)
int plan_create_sharing(const mlg_plan_s* base, const Csr* Gu, const Csr* Gut, mlg_plan_s** out);
void plan_destroy(mlg_plan_s* p);

// layout conversions (mlg_nufft.cu)
int pack_col_to_point(const float* re, const float* im, long long rows, int nCh, float2* out, cudaStream_t s);
int unpack_point_to_col(const float2* in, long long rows, int nCh, float* re, float* im, cudaStream_t s);
int interleave(const float* re, const float* im, long long n, float2* out, cudaStream_t s);
int deinterleave(const float2* in, long long n, float* re, float* im, cudaStream_t s);

}  // namespace mlg
