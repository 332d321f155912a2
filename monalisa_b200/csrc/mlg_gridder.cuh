// Internal interface of the tile-binned adjoint gridder (mlg_gridder.cu).
#pragma once

#include "mlg_internal.cuh"

namespace mlg {

struct LeightGeom {
  int imDim = 1, nCh = 1, nWin = 3, half = 1;
  int N[3] = {1, 1, 1};
  int T[3] = {1, 1, 1};   // tile extent per dimension
  int nt[3] = {1, 1, 1};  // tiles per dimension
  long long ntiles = 1;
  long long Nu_tot = 1;
  int tile_cells = 1;
  size_t smem_bytes = 0;
  float t_shift = 0.5f;
  float g1 = 0.f, g2 = 0.f;  // Gaussian constants
  // register-accumulating tiles (8, 12 or 16 coils): at most 512 cells, two
  // per thread; otherwise shared-memory accumulators sized by smem_bytes
  bool gather = false;
};

struct LeightInputs {
  Layout layout = Layout::kPointSplit;  // kPointSplit or kPointC64, [nPt][nCh]
  const float* re = nullptr;
  const float* im = nullptr;
  const float2* c64 = nullptr;
  const float* tx = nullptr;  // 1-based grid coordinates
  const float* ty = nullptr;
  const float* tz = nullptr;
  const float* Dn = nullptr;
};

struct LeightOutput {
  Layout layout = Layout::kPointSplit;  // kPointSplit [Nu][nCh] or kCoilC64 [nCh][Nu]
  float* re = nullptr;
  float* im = nullptr;
  float2* c64 = nullptr;
  float scale = 1.0f;  // applied to kCoilC64 output only
};

// Two workspace regions: `counters` holds per-tile counters and scan
// temporaries (size depends on the tile count only, counters_bytes()); `bins`
// holds the (tile, sample) pairs, the chunk list and the partial tiles of
// split bins, whose size is known only after counting (bins_bytes()).  When
// `bins` is too small and `grow_bins` is set it is called to provide a larger
// region; otherwise the call fails with MLG_ERR_ARG.
struct LeightWorkspace {
  void* counters = nullptr;
  size_t counters_cap = 0;
  void* bins = nullptr;
  size_t bins_cap = 0;
  int (*grow_bins)(LeightWorkspace& ws, size_t bytes, cudaStream_t s) = nullptr;
  // sizes found by the last run
  long long last_pairs = 0, last_chunks = 0, last_slots = 0;

  static size_t align(size_t b) { return (b + 255) & ~size_t(255); }
  static size_t counters_bytes(const LeightGeom& g);
  static size_t bins_bytes(const LeightGeom& g, long long pairs, long long chunks, long long slots);
};

int leight_geometry(int imDim, int nCh, const int* N, int nWin, float sigma, LeightGeom& g);
// Upper bound of the (tile, sample) pairs nPt samples can produce.
long long leight_max_pairs(const LeightGeom& g, long long nPt);
// Loads every kernel the tile-binned form launches into the current device's
// context (under CUDA's lazy module loading a kernel is otherwise loaded, and
// its memory taken, at its first launch).
int leight_preload();
// Tile-binned form.  It waits on the host once per call: after the counting
// kernels it synchronises `s` to read the bin totals, then queues the rest.
int leight_run(const LeightGeom& g, const LeightInputs& in, int nPt, const LeightOutput& out, LeightWorkspace& ws,
               cudaStream_t s);

// Cell-binned form (the entry points that may allocate): the samples are
// sorted by the lower-corner cell of their window in a corner grid of
// N + nWin - 1 cells per image axis, and every grid cell gathers the samples
// of the corner cells whose windows cover it (no tiles, no atomics on the
// grid, no host synchronisation).  Its workspace, leight_cells_bytes(g, nPt)
// bytes, is known before the call.  Split complex input and output only.
size_t leight_cells_bytes(const LeightGeom& g, int nPt);
int leight_run_cells(const LeightGeom& g, const LeightInputs& in, int nPt, const LeightOutput& out, void* ws,
                     size_t ws_bytes, cudaStream_t s);

// Builds the "cell x sample" CSR of a precomputed-weight gridding call.
int n2u_build_csr(const float* d_w, const int* d_nJump, int nNb, int nPt, int Nu_tot, Csr& m, cudaStream_t s);

}  // namespace mlg
