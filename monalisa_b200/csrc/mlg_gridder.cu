// Adjoint (nonuniform -> uniform) gridding.
//
// 1. leight form (on-the-fly Gaussian window, clipped at the grid border,
//    per-cell normalisation): the semantics of
//    src/gridding123/mex/bmGridder_n2u_leight{1,2,3}/..._mex.cpp.
//    The reference scatters serially into the whole grid.  Here the grid is
//    cut into tiles that fit in shared memory; every sample is binned into
//    each tile its window touches (a counting sort: count, scan, fill), and
//    one CTA accumulates a tile's samples with shared-memory atomics, then
//    normalises and writes the tile once.  No global float atomics: each
//    output cell is written by exactly one CTA.  Tiles whose bin is larger
//    than kChunkPairs are split into chunks; each chunk writes its partial
//    tile to a scratch area and a combine kernel sums the chunks of a tile in
//    chunk order, then normalises.
// 2. precomputed-weight form (bmGridder_n2u_mex.cpp:72-201): the jump-coded
//    targets are decoded, the (cell, entry) pairs are stably sorted by cell
//    and the result is a CSR "cell x sample" matrix evaluated by the SpMM
//    kernels with row normalisation -- per cell the entries keep the
//    reference's accumulation order, so short rows are bit-exact.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>

#include "mlg_gridder.cuh"

namespace mlg {

constexpr int kChunkPairs = 1024;   // samples (pairs) per accumulate CTA
constexpr int kGridThreads = 256;
constexpr size_t kTileSmemBudget = 110 * 1024;

// ---- geometry -------------------------------------------------------------
int leight_geometry(int imDim, int nCh, const int* N, int nWin, float sigma, LeightGeom& g) {
  MLG_CHECK(imDim >= 1 && imDim <= 3, "imDim must be 1, 2 or 3");
  MLG_CHECK(nCh >= 1, "nCh must be >= 1");
  MLG_CHECK(nWin >= 1 && nWin <= 16, "nWin=%d outside [1,16]", nWin);
  MLG_CHECK(sigma > 0.f, "sigma must be > 0");
  g = LeightGeom();
  g.imDim = imDim;
  g.nCh = nCh;
  g.nWin = nWin;
  long long cells = 1;
  for (int d = 0; d < 3; ++d) {
    g.N[d] = d < imDim ? N[d] : 1;
    MLG_CHECK(g.N[d] >= 1, "grid size must be >= 1");
    cells *= g.N[d];
  }
  g.Nu_tot = cells;
  MLG_CHECK(cells < (1LL << 31), "grid of %lld cells too large", cells);
  // window geometry, bmGridder_n2u_leight3_mex.cpp:189-199
  if (nWin % 2) {
    g.t_shift = 0.5f;
    g.half = (nWin - 1) / 2;
  } else {
    g.t_shift = 0.0f;
    g.half = nWin / 2 - 1;
  }
  // Gaussian constants with the reference's float arithmetic (:202-205)
  g.g1 = 1 / ((float)std::sqrt(2 * 3.141592) * sigma);
  g.g2 = -1 / (2 * (sigma * sigma));
  // tile shape: start large, halve the largest extent until a tile's
  // accumulators fit the shared-memory budget
  const int G = 2 * nCh + 1;
  g.gather = nCh == 8 || nCh == 12 || nCh == 16;
  int T[3];
  if (g.gather) {  // 512 cells: two per thread of a 256-thread CTA
    if (imDim == 1) { T[0] = 512; T[1] = 1; T[2] = 1; }
    else if (imDim == 2) { T[0] = 32; T[1] = 16; T[2] = 1; }
    else { T[0] = 8; T[1] = 8; T[2] = 8; }
  } else if (imDim == 1) { T[0] = 4096; T[1] = 1; T[2] = 1; }
  else if (imDim == 2) { T[0] = 64; T[1] = 32; T[2] = 1; }
  else { T[0] = 16; T[1] = 8; T[2] = 8; }
  for (int d = 0; d < 3; ++d) T[d] = std::min(T[d], g.N[d]);
  while ((size_t)T[0] * T[1] * T[2] * G * sizeof(float) > kTileSmemBudget) {
    int dm = 0;
    for (int d = 1; d < 3; ++d) if (T[d] > T[dm]) dm = d;
    MLG_CHECK(T[dm] > 1, "nCh=%d too large for a shared-memory tile", nCh);
    T[dm] = (T[dm] + 1) / 2;
  }
  g.ntiles = 1;
  for (int d = 0; d < 3; ++d) {
    g.T[d] = T[d];
    g.nt[d] = (g.N[d] + T[d] - 1) / T[d];
    g.ntiles *= g.nt[d];
  }
  g.tile_cells = T[0] * T[1] * T[2];
  g.smem_bytes = (size_t)g.tile_cells * G * sizeof(float);
  return MLG_OK;
}

// Window of sample s: fractional offsets r[] and 0-based lower corner lo[].
// Returns false when the window misses the grid.
__device__ __forceinline__ bool sample_window(const LeightGeom& g, const LeightInputs& in, int s, float r[3],
                                              int lo[3]) {
  const float* t[3] = {in.tx, in.ty, in.tz};
  bool hit = true;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    if (d < g.imDim) {
      const float td = __ldg(t[d] + s);
      const float node = truncf(td + g.t_shift);  // modff's integral part
      if (!(fabsf(node) < 1.0e9f)) return false;   // NaN / huge: no cell
      r[d] = td - node;
      lo[d] = (int)node - 1 - g.half;
      hit = hit && (lo[d] + g.nWin - 1 >= 0) && (lo[d] <= g.N[d] - 1);
    } else {
      r[d] = 0.f;
      lo[d] = 0;
    }
  }
  return hit;
}

__device__ __forceinline__ void tile_range(const LeightGeom& g, const int lo[3], int t0[3], int t1[3]) {
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    if (d < g.imDim) {
      const int a = max(lo[d], 0), b = min(lo[d] + g.nWin - 1, g.N[d] - 1);
      t0[d] = a / g.T[d];
      t1[d] = b / g.T[d];
    } else {
      t0[d] = t1[d] = 0;
    }
  }
}

__global__ void leight_count_kernel(LeightGeom g, LeightInputs in, int nPt, int* __restrict__ count) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nPt; s += gridDim.x * blockDim.x) {
    float r[3];
    int lo[3], t0[3], t1[3];
    if (!sample_window(g, in, s, r, lo)) continue;
    tile_range(g, lo, t0, t1);
    for (int z = t0[2]; z <= t1[2]; ++z)
      for (int y = t0[1]; y <= t1[1]; ++y)
        for (int x = t0[0]; x <= t1[0]; ++x) atomicAdd(count + (x + g.nt[0] * (y + (long long)g.nt[1] * z)), 1);
  }
}

__global__ void leight_fill_kernel(LeightGeom g, LeightInputs in, int nPt, const int* __restrict__ offset,
                                   int* __restrict__ cursor, int* __restrict__ pairs) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nPt; s += gridDim.x * blockDim.x) {
    float r[3];
    int lo[3], t0[3], t1[3];
    if (!sample_window(g, in, s, r, lo)) continue;
    tile_range(g, lo, t0, t1);
    for (int z = t0[2]; z <= t1[2]; ++z)
      for (int y = t0[1]; y <= t1[1]; ++y)
        for (int x = t0[0]; x <= t1[0]; ++x) {
          const long long t = x + g.nt[0] * (y + (long long)g.nt[1] * z);
          pairs[offset[t] + atomicAdd(cursor + t, 1)] = s;
        }
  }
}

// chunks per tile (>= 1 so that empty tiles are still written) and partial
// slots (only tiles split over several chunks need them; those tiles are
// listed in split, in no particular order, for the combine kernel)
__global__ void leight_chunk_count_kernel(long long ntiles, const int* __restrict__ count, int* __restrict__ nchunk,
                                          int* __restrict__ nslot, int* __restrict__ split, int* __restrict__ nsplit) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < ntiles; t += (long long)gridDim.x * blockDim.x) {
    const int c = max(1, (count[t] + kChunkPairs - 1) / kChunkPairs);
    nchunk[t] = c;
    nslot[t] = c > 1 ? c : 0;
    if (c > 1) split[atomicAdd(nsplit, 1)] = (int)t;
  }
}

// Chunk list: the chunks of split tiles first, at their slot index (the
// longest-running CTAs start first), then the single-chunk tiles in no
// particular order.  chunk = (tile, first pair, end pair, slot or -1).
__global__ void leight_chunk_build_kernel(long long ntiles, const int* __restrict__ count,
                                          const int* __restrict__ offset, const int* __restrict__ nchunk,
                                          const int* __restrict__ slot_off, int nslots, int* __restrict__ nsingle,
                                          int4* __restrict__ chunks) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < ntiles; t += (long long)gridDim.x * blockDim.x) {
    const int n = nchunk[t];
    if (n == 1) {
      chunks[nslots + atomicAdd(nsingle, 1)] = make_int4((int)t, offset[t], offset[t] + count[t], -1);
      continue;
    }
    for (int i = 0; i < n; ++i) {
      const int b = offset[t] + i * kChunkPairs;
      const int e = min(b + kChunkPairs, offset[t] + count[t]);
      chunks[slot_off[t] + i] = make_int4((int)t, b, e, slot_off[t] + i);
    }
  }
}

__device__ __forceinline__ void tile_origin(const LeightGeom& g, long long t, int o[3]) {
  const long long q = t / g.nt[0];
  o[0] = (int)(t % g.nt[0]) * g.T[0];
  o[1] = (int)(q % g.nt[1]) * g.T[1];
  o[2] = (int)(q / g.nt[1]) * g.T[2];
}

// Normalises and stores a tile's accumulators (sm [tile_cells][G], acc =
// [norm, re0, im0, ...]): one (cell, coil) per thread and step.
__device__ __forceinline__ void store_tile(const LeightGeom& g, const LeightOutput& out, const float* sm,
                                          const int org[3]) {
  const int G = 2 * g.nCh + 1;
  const int ncell_items = g.tile_cells * g.nCh;
  for (int i = threadIdx.x; i < ncell_items; i += blockDim.x) {
    const int c = i % g.nCh, lc = i / g.nCh;
    const int lx = lc % g.T[0], ly = (lc / g.T[0]) % g.T[1], lz = lc / (g.T[0] * g.T[1]);
    const int x = org[0] + lx, y = org[1] + ly, z = org[2] + lz;
    if (x >= g.N[0] || y >= g.N[1] || z >= g.N[2]) continue;
    const long long cell = x + (long long)g.N[0] * (y + (long long)g.N[1] * z);
    const float* acc = sm + (size_t)lc * G;
    float s = acc[0];
    if (s < 1e-5f) s = 1.0f;  // bmGridder_n2u_leight3_mex.cpp:341-344
    const float re = __fdiv_rn(acc[1 + 2 * c], s), im = __fdiv_rn(acc[2 + 2 * c], s);
    if (out.layout == Layout::kPointSplit) {
      out.re[cell * g.nCh + c] = re;
      out.im[cell * g.nCh + c] = im;
    } else {  // kCoilC64
      out.c64[(long long)c * g.Nu_tot + cell] = make_float2(re * out.scale, im * out.scale);
    }
  }
}

__global__ void __launch_bounds__(kGridThreads) leight_accumulate_kernel(LeightGeom g, LeightInputs in,
                                                                         const int* __restrict__ pairs,
                                                                         const int4* __restrict__ chunks,
                                                                         float* __restrict__ partial,
                                                                         LeightOutput out) {
  extern __shared__ float sm[];
  const int G = 2 * g.nCh + 1;
  const int4 ch = chunks[blockIdx.x];
  const long long tile = ch.x;
  int org[3];
  tile_origin(g, tile, org);
  for (int i = threadIdx.x; i < g.tile_cells * G; i += blockDim.x) sm[i] = 0.f;
  __syncthreads();

  int W = g.nWin;
  if (g.imDim > 1) W *= g.nWin;
  if (g.imDim > 2) W *= g.nWin;
  const long long items = (long long)(ch.z - ch.y) * W;
  for (long long it = threadIdx.x; it < items; it += blockDim.x) {
    const int s = __ldg(pairs + ch.y + (int)(it / W));
    const int wc = (int)(it % W);
    float r[3];
    int lo[3];
    sample_window(g, in, s, r, lo);
    const int iw[3] = {wc % g.nWin, (wc / g.nWin) % g.nWin, wc / (g.nWin * g.nWin)};
    int cl[3];
    bool ok = true;
    float d2 = 0.f;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      if (d < g.imDim) {
        const int n = lo[d] + iw[d];
        cl[d] = n - org[d];
        ok = ok && n >= 0 && n < g.N[d] && cl[d] >= 0 && cl[d] < g.T[d];
        const float u = (float)(iw[d] - g.half);
        const float dd = r[d] - u;
        d2 = d == 0 ? __fmul_rn(dd, dd) : __fadd_rn(d2, __fmul_rn(dd, dd));
      } else {
        cl[d] = 0;
      }
    }
    if (!ok) continue;
    const float dn = __ldg(in.Dn + s);
    const float w = __fmul_rn(__fmul_rn(g.g1, expf(__fmul_rn(g.g2, d2))), dn);
    float* acc = sm + (cl[0] + g.T[0] * (cl[1] + g.T[1] * cl[2])) * G;
    atomicAdd(acc, w);
    const long long base = (long long)s * g.nCh;
    for (int c = 0; c < g.nCh; ++c) {
      float ar, ai;
      if (in.layout == Layout::kPointSplit) {
        ar = __ldg(in.re + base + c);
        ai = __ldg(in.im + base + c);
      } else {
        const float2 v = __ldg(in.c64 + base + c);
        ar = v.x;
        ai = v.y;
      }
      atomicAdd(acc + 1 + 2 * c, __fmul_rn(w, ar));
      atomicAdd(acc + 2 + 2 * c, __fmul_rn(w, ai));
    }
  }
  __syncthreads();

  if (ch.w >= 0) {  // partial tile of a split bin: raw accumulators to scratch
    float* dst = partial + (long long)ch.w * g.tile_cells * G;
    for (int i = threadIdx.x; i < g.tile_cells * G; i += blockDim.x) dst[i] = sm[i];
    return;
  }
  store_tile(g, out, sm, org);
}

// The same accumulation with a warp per sample, for many channels (G = 2 nCh
// + 1 >= 17) and windows of at most 32 cells: lane k < W forms window cell
// k's weight and tile-local cell once; every lane owns accumulator channels
// lane, lane + 32, ... (norm, re0, im0, re1, ...) and loads its values of the
// sample once; a loop over the window broadcasts (cell, weight) and each
// lane adds its channel -- one shared-memory atomic per lane and cell, no
// bank conflicts, instead of a coil loop per window cell.  Same values as
// leight_accumulate_kernel; only the (already unordered) atomic order
// differs.
constexpr int kWarpMaxK = 3;  // channel chunks of 32: G <= 96

__global__ void __launch_bounds__(kGridThreads) leight_accumulate_warp_kernel(LeightGeom g, LeightInputs in,
                                                                              const int* __restrict__ pairs,
                                                                              const int4* __restrict__ chunks,
                                                                              float* __restrict__ partial,
                                                                              LeightOutput out) {
  extern __shared__ float sm[];
  const int G = 2 * g.nCh + 1;
  const int4 ch = chunks[blockIdx.x];
  const long long tile = ch.x;
  int org[3];
  tile_origin(g, tile, org);
  for (int i = threadIdx.x; i < g.tile_cells * G; i += blockDim.x) sm[i] = 0.f;
  __syncthreads();

  int W = g.nWin;
  if (g.imDim > 1) W *= g.nWin;
  if (g.imDim > 2) W *= g.nWin;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int nk = (G + 31) / 32;
  for (int q = ch.y + warp; q < ch.z; q += nwarps) {
    const int s = __ldg(pairs + q);
    float r[3];
    int lo[3];
    sample_window(g, in, s, r, lo);
    // lane k < W: weight and tile-local cell (-1: outside the tile or grid)
    float wk = 0.f;
    int cellk = -1;
    if (lane < W) {
      const int iw[3] = {lane % g.nWin, (lane / g.nWin) % g.nWin, lane / (g.nWin * g.nWin)};
      int cl[3];
      bool ok = true;
      float d2 = 0.f;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        if (d < g.imDim) {
          const int n = lo[d] + iw[d];
          cl[d] = n - org[d];
          ok = ok && n >= 0 && n < g.N[d] && cl[d] >= 0 && cl[d] < g.T[d];
          const float u = (float)(iw[d] - g.half);
          const float dd = r[d] - u;
          d2 = d == 0 ? __fmul_rn(dd, dd) : __fadd_rn(d2, __fmul_rn(dd, dd));
        } else {
          cl[d] = 0;
        }
      }
      if (ok) {
        wk = __fmul_rn(__fmul_rn(g.g1, expf(__fmul_rn(g.g2, d2))), __ldg(in.Dn + s));
        cellk = cl[0] + g.T[0] * (cl[1] + g.T[1] * cl[2]);
      }
    }
    // this lane's channel values of the sample (channel 0 is the norm)
    float a[kWarpMaxK];
    const long long base = (long long)s * g.nCh;
#pragma unroll
    for (int j = 0; j < kWarpMaxK; ++j) {
      const int chn = lane + 32 * j;
      float v = 0.f;
      if (j < nk && chn >= 1 && chn < G) {
        const int c = (chn - 1) >> 1;
        const bool imag = (chn - 1) & 1;
        if (in.layout == Layout::kPointSplit) {
          v = __ldg((imag ? in.im : in.re) + base + c);
        } else {
          const float2 z = __ldg(in.c64 + base + c);
          v = imag ? z.y : z.x;
        }
      }
      a[j] = v;
    }
    for (int k = 0; k < W; ++k) {
      const int cell = __shfl_sync(0xffffffffu, cellk, k);
      const float w = __shfl_sync(0xffffffffu, wk, k);
      if (cell < 0) continue;  // uniform in the warp
      float* acc = sm + cell * G;
#pragma unroll
      for (int j = 0; j < kWarpMaxK; ++j) {
        const int chn = lane + 32 * j;
        if (j < nk && chn < G) atomicAdd(acc + chn, chn == 0 ? w : __fmul_rn(w, a[j]));
      }
    }
  }
  __syncthreads();

  if (ch.w >= 0) {  // partial tile of a split bin: raw accumulators to scratch
    float* dst = partial + (long long)ch.w * g.tile_cells * G;
    for (int i = threadIdx.x; i < g.tile_cells * G; i += blockDim.x) dst[i] = sm[i];
    return;
  }
  store_tile(g, out, sm, org);
}

// Register-accumulating form for NCH = 8, 12, 16 coils (tiles of at most
// 512 cells): thread t owns tile cells t and t + 256 with their 2 NCH + 1
// accumulators in registers.  The chunk's samples pass through shared
// memory in batches of kBatch (window corner and offsets, Dn, the NCH
// complex values); every thread tests its cells against each sample's
// window and accumulates the cells it covers -- no atomics, and per cell
// the samples are summed in list order.  Weights as in
// leight_accumulate_kernel.
constexpr int kBatch = 128;

template <int NCH>
__global__ void __launch_bounds__(kGridThreads, 2) leight_gather_kernel(LeightGeom g, LeightInputs in,
                                                                        const int* __restrict__ pairs,
                                                                        const int4* __restrict__ chunks,
                                                                        float* __restrict__ partial,
                                                                        LeightOutput out) {
  constexpr int G = 2 * NCH + 1, CPT = 2;
  __shared__ int s_lo[3][kBatch];
  __shared__ float s_r[3][kBatch];
  __shared__ float s_dn[kBatch];
  __shared__ int s_s[kBatch];
  __shared__ __align__(16) float s_a[kBatch][2 * NCH];
  const int4 ch = chunks[blockIdx.x];
  int org[3];
  tile_origin(g, ch.x, org);
  int cx[CPT], cy[CPT], cz[CPT], lcs[CPT];
  bool cin[CPT];
#pragma unroll
  for (int k = 0; k < CPT; ++k) {
    const int lc = threadIdx.x + k * kGridThreads;
    lcs[k] = lc;
    const int lx = lc % g.T[0], ly = (lc / g.T[0]) % g.T[1], lz = lc / (g.T[0] * g.T[1]);
    cx[k] = org[0] + lx;
    cy[k] = org[1] + ly;
    cz[k] = org[2] + lz;
    cin[k] = lc < g.tile_cells && cx[k] < g.N[0] && cy[k] < g.N[1] && cz[k] < g.N[2];
  }
  float acc[CPT][G];
#pragma unroll
  for (int k = 0; k < CPT; ++k)
#pragma unroll
    for (int q = 0; q < G; ++q) acc[k][q] = 0.f;

  const unsigned nW = (unsigned)g.nWin;
  for (int b0 = ch.y; b0 < ch.z; b0 += kBatch) {
    const int nb = min(kBatch, ch.z - b0);
    __syncthreads();  // the previous batch is consumed
    if ((int)threadIdx.x < nb) {
      const int s = __ldg(pairs + b0 + threadIdx.x);
      float r[3];
      int lo[3];
      const bool hit = sample_window(g, in, s, r, lo);
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        s_lo[d][threadIdx.x] = hit ? lo[d] : -(1 << 29);  // a missed window covers no cell
        s_r[d][threadIdx.x] = r[d];
      }
      s_dn[threadIdx.x] = __ldg(in.Dn + s);
      s_s[threadIdx.x] = s;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nb * NCH; i += kGridThreads) {
      const int j = i / NCH, c = i - j * NCH;
      const long long e = (long long)s_s[j] * NCH + c;
      float2 v;
      if (in.layout == Layout::kPointSplit)
        v = make_float2(__ldg(in.re + e), __ldg(in.im + e));
      else
        v = __ldg(in.c64 + e);
      s_a[j][2 * c] = v.x;
      s_a[j][2 * c + 1] = v.y;
    }
    __syncthreads();
    for (int j = 0; j < nb; ++j) {
      const int l0 = s_lo[0][j], l1 = s_lo[1][j], l2 = s_lo[2][j];
#pragma unroll
      for (int k = 0; k < CPT; ++k) {
        if (!cin[k]) continue;
        const int i0 = cx[k] - l0, i1 = cy[k] - l1, i2 = cz[k] - l2;
        if ((unsigned)i0 >= nW) continue;
        if (g.imDim > 1 && (unsigned)i1 >= nW) continue;
        if (g.imDim > 2 && (unsigned)i2 >= nW) continue;
        const float dd0 = s_r[0][j] - (float)(i0 - g.half);
        float d2 = __fmul_rn(dd0, dd0);
        if (g.imDim > 1) {
          const float dd1 = s_r[1][j] - (float)(i1 - g.half);
          d2 = __fadd_rn(d2, __fmul_rn(dd1, dd1));
        }
        if (g.imDim > 2) {
          const float dd2 = s_r[2][j] - (float)(i2 - g.half);
          d2 = __fadd_rn(d2, __fmul_rn(dd2, dd2));
        }
        const float w = __fmul_rn(__fmul_rn(g.g1, expf(__fmul_rn(g.g2, d2))), s_dn[j]);
        acc[k][0] = __fadd_rn(acc[k][0], w);
        const float4* a4 = reinterpret_cast<const float4*>(s_a[j]);
#pragma unroll
        for (int q = 0; q < NCH / 2; ++q) {  // fused multiply-adds: the order of the sums differs anyway
          const float4 a = a4[q];
          acc[k][1 + 4 * q] = __fmaf_rn(w, a.x, acc[k][1 + 4 * q]);
          acc[k][2 + 4 * q] = __fmaf_rn(w, a.y, acc[k][2 + 4 * q]);
          acc[k][3 + 4 * q] = __fmaf_rn(w, a.z, acc[k][3 + 4 * q]);
          acc[k][4 + 4 * q] = __fmaf_rn(w, a.w, acc[k][4 + 4 * q]);
        }
      }
    }
  }

#pragma unroll
  for (int k = 0; k < CPT; ++k) {
    if (lcs[k] >= g.tile_cells) continue;
    if (ch.w >= 0) {  // partial tile of a split bin: raw accumulators to scratch
      float* dst = partial + ((long long)ch.w * g.tile_cells + lcs[k]) * G;
#pragma unroll
      for (int q = 0; q < G; ++q) dst[q] = acc[k][q];
      continue;
    }
    if (!cin[k]) continue;
    const long long cell = cx[k] + (long long)g.N[0] * (cy[k] + (long long)g.N[1] * cz[k]);
    float s = acc[k][0];
    if (s < 1e-5f) s = 1.0f;  // bmGridder_n2u_leight3_mex.cpp:341-344
#pragma unroll
    for (int c = 0; c < NCH; ++c) {
      const float re = __fdiv_rn(acc[k][1 + 2 * c], s), im = __fdiv_rn(acc[k][2 + 2 * c], s);
      if (out.layout == Layout::kPointSplit) {
        out.re[cell * NCH + c] = re;
        out.im[cell * NCH + c] = im;
      } else {  // kCoilC64
        out.c64[(long long)c * g.Nu_tot + cell] = make_float2(re * out.scale, im * out.scale);
      }
    }
  }
}

// one CTA per split tile (split[blockIdx.x])
__global__ void __launch_bounds__(kGridThreads) leight_combine_kernel(LeightGeom g, const int* __restrict__ split,
                                                                      const int* __restrict__ nchunk,
                                                                      const int* __restrict__ slot_off,
                                                                      const float* __restrict__ partial,
                                                                      LeightOutput out) {
  extern __shared__ float sm[];
  const long long tile = split[blockIdx.x];
  const int n = nchunk[tile];
  if (n <= 1) return;
  const int G = 2 * g.nCh + 1;
  const float* src = partial + (long long)slot_off[tile] * g.tile_cells * G;
  const long long stride = (long long)g.tile_cells * G;
  for (int i = threadIdx.x; i < g.tile_cells * G; i += blockDim.x) {
    float a = 0.f;
    for (int k = 0; k < n; ++k) a = __fadd_rn(a, src[k * stride + i]);  // chunk order
    sm[i] = a;
  }
  __syncthreads();
  int org[3];
  tile_origin(g, tile, org);
  store_tile(g, out, sm, org);
}

static int grid_for(long long n, int threads = 256) {
  return (int)std::max<long long>(1, std::min<long long>((n + threads - 1) / threads, 148LL * 32));
}

// ---- workspace ------------------------------------------------------------
size_t LeightWorkspace::counters_bytes(const LeightGeom& g) {
  size_t scan_tmp = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, scan_tmp, (int*)nullptr, (int*)nullptr, (int)g.ntiles);
  return align((size_t)g.ntiles * 4) * 8 + align(8) + align(scan_tmp);
}

size_t LeightWorkspace::bins_bytes(const LeightGeom& g, long long pairs, long long chunks, long long slots) {
  const size_t G = 2 * (size_t)g.nCh + 1;
  return align((size_t)pairs * 4) + align((size_t)chunks * 16) + align((size_t)slots * g.tile_cells * G * 4);
}

long long leight_max_pairs(const LeightGeom& g, long long nPt) {
  // a window of nWin cells meets at most ceil((nWin - 1) / T) + 1 tiles per axis
  long long per = 1;
  for (int d = 0; d < g.imDim; ++d) per *= (g.nWin - 1 + g.T[d] - 1) / g.T[d] + 1;
  return nPt * per;
}

int leight_preload() {
  cudaFuncAttributes a;
  MLG_CUDA(cudaFuncGetAttributes(&a, leight_count_kernel));
  MLG_CUDA(cudaFuncGetAttributes(&a, leight_fill_kernel));
  MLG_CUDA(cudaFuncGetAttributes(&a, leight_chunk_count_kernel));
  MLG_CUDA(cudaFuncGetAttributes(&a, leight_chunk_build_kernel));
  MLG_CUDA(cudaFuncGetAttributes(&a, leight_accumulate_kernel));
  MLG_CUDA(cudaFuncGetAttributes(&a, leight_accumulate_warp_kernel));
  MLG_CUDA(cudaFuncGetAttributes(&a, leight_gather_kernel<16>));
  MLG_CUDA(cudaFuncGetAttributes(&a, leight_gather_kernel<12>));
  MLG_CUDA(cudaFuncGetAttributes(&a, leight_gather_kernel<8>));
  MLG_CUDA(cudaFuncGetAttributes(&a, leight_combine_kernel));
  return MLG_OK;
}

int leight_run(const LeightGeom& g, const LeightInputs& in, int nPt, const LeightOutput& out, LeightWorkspace& ws,
               cudaStream_t s) {
  NvtxRange range("leight gridder (tile-binned)");
  MLG_CHECK(g.ntiles < (1LL << 31), "too many tiles");
  // the per-tile counts, their scan and the bin offsets are 32-bit: refuse
  // inputs whose (tile, sample) pairs could pass 2^31 before counting them
  MLG_CHECK(leight_max_pairs(g, nPt) < (1LL << 31),
            "%d samples may meet up to %lld (tile, sample) pairs; at most 2^31 - 1 are supported", nPt,
            leight_max_pairs(g, nPt));
  const int nt = (int)g.ntiles;
  MLG_CHECK(ws.counters && ws.counters_cap >= LeightWorkspace::counters_bytes(g),
            "gridding counter workspace too small (%zu < %zu bytes)", ws.counters_cap,
            LeightWorkspace::counters_bytes(g));
  // phase 1: per-tile counters and scans
  char* p = (char*)ws.counters;
  auto take = [&](size_t bytes) {
    char* q = p;
    p += LeightWorkspace::align(bytes);
    return (void*)q;
  };
  int* count = (int*)take((size_t)nt * 4);
  int* offset = (int*)take((size_t)nt * 4);
  int* cursor = (int*)take((size_t)nt * 4);
  int* nchunk = (int*)take((size_t)nt * 4);
  int* chunk_off = (int*)take((size_t)nt * 4);
  int* nslot = (int*)take((size_t)nt * 4);
  int* slot_off = (int*)take((size_t)nt * 4);
  int* split = (int*)take((size_t)nt * 4);
  int* nsplit = (int*)take(8);  // [0]: split tiles, [1]: single-chunk tiles placed
  size_t scan_tmp = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, scan_tmp, count, offset, nt);
  void* tmp = take(scan_tmp);

  MLG_CUDA(cudaMemsetAsync(count, 0, (size_t)nt * 4, s));
  MLG_CUDA(cudaMemsetAsync(cursor, 0, (size_t)nt * 4, s));
  MLG_CUDA(cudaMemsetAsync(nsplit, 0, 4, s));
  if (nPt > 0) {
    leight_count_kernel<<<grid_for(nPt), 256, 0, s>>>(g, in, nPt, count);
    MLG_LAUNCHED();
  }
  MLG_CUDA(cub::DeviceScan::ExclusiveSum(tmp, scan_tmp, count, offset, nt, s));
  leight_chunk_count_kernel<<<grid_for(nt), 256, 0, s>>>(g.ntiles, count, nchunk, nslot, split, nsplit);
  MLG_LAUNCHED();
  MLG_CUDA(cub::DeviceScan::ExclusiveSum(tmp, scan_tmp, nchunk, chunk_off, nt, s));
  MLG_CUDA(cub::DeviceScan::ExclusiveSum(tmp, scan_tmp, nslot, slot_off, nt, s));
  // totals = last offset + last count
  int h[7];
  MLG_CUDA(cudaMemcpyAsync(h + 0, offset + nt - 1, 4, cudaMemcpyDeviceToHost, s));
  MLG_CUDA(cudaMemcpyAsync(h + 1, count + nt - 1, 4, cudaMemcpyDeviceToHost, s));
  MLG_CUDA(cudaMemcpyAsync(h + 2, chunk_off + nt - 1, 4, cudaMemcpyDeviceToHost, s));
  MLG_CUDA(cudaMemcpyAsync(h + 3, nchunk + nt - 1, 4, cudaMemcpyDeviceToHost, s));
  MLG_CUDA(cudaMemcpyAsync(h + 4, slot_off + nt - 1, 4, cudaMemcpyDeviceToHost, s));
  MLG_CUDA(cudaMemcpyAsync(h + 5, nslot + nt - 1, 4, cudaMemcpyDeviceToHost, s));
  MLG_CUDA(cudaMemcpyAsync(h + 6, nsplit, 4, cudaMemcpyDeviceToHost, s));
  MLG_CUDA(cudaStreamSynchronize(s));
  const long long npairs = (long long)h[0] + h[1];
  const long long nchunks = (long long)h[2] + h[3];
  const long long nslots = (long long)h[4] + h[5];
  const int n_split = h[6];
  ws.last_pairs = npairs;
  ws.last_chunks = nchunks;
  ws.last_slots = nslots;
  MLG_CHECK(nchunks < (1LL << 31), "too many chunks");

  // phase 2: bins
  const size_t need = LeightWorkspace::bins_bytes(g, npairs, nchunks, nslots);
  if (!ws.bins || ws.bins_cap < need) {
    if (!ws.grow_bins)
      return fail(MLG_ERR_ARG, "gridding bin workspace too small: %zu bytes available, %zu needed", ws.bins_cap,
                  need);
    MLG_TRY(ws.grow_bins(ws, need, s));
  }
  p = (char*)ws.bins;
  int* pairs = (int*)take((size_t)npairs * 4);
  int4* chunks = (int4*)take((size_t)nchunks * 16);
  float* partial = (float*)take((size_t)nslots * g.tile_cells * (2 * (size_t)g.nCh + 1) * 4);

  if (nPt > 0 && npairs > 0) {
    leight_fill_kernel<<<grid_for(nPt), 256, 0, s>>>(g, in, nPt, offset, cursor, pairs);
    MLG_LAUNCHED();
  }
  MLG_CUDA(cudaMemsetAsync(nsplit + 1, 0, 4, s));
  leight_chunk_build_kernel<<<grid_for(nt), 256, 0, s>>>(g.ntiles, count, offset, nchunk, slot_off, (int)nslots,
                                                         nsplit + 1, chunks);
  MLG_LAUNCHED();
  // a warp per sample for many channels and windows of at most 32 cells
  int W = g.nWin;
  if (g.imDim > 1) W *= g.nWin;
  if (g.imDim > 2) W *= g.nWin;
  const int G = 2 * g.nCh + 1;
  const bool warp_path = G >= 17 && G <= 32 * kWarpMaxK && W <= 32;
  if (g.smem_bytes > 48 * 1024) {
    MLG_CUDA(cudaFuncSetAttribute(leight_accumulate_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)kTileSmemBudget));
    MLG_CUDA(cudaFuncSetAttribute(leight_accumulate_warp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)kTileSmemBudget));
    MLG_CUDA(cudaFuncSetAttribute(leight_combine_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)kTileSmemBudget));
  }
  if (g.gather && g.nCh == 16)
    leight_gather_kernel<16><<<(int)nchunks, kGridThreads, 0, s>>>(g, in, pairs, chunks, partial, out);
  else if (g.gather && g.nCh == 12)
    leight_gather_kernel<12><<<(int)nchunks, kGridThreads, 0, s>>>(g, in, pairs, chunks, partial, out);
  else if (g.gather && g.nCh == 8)
    leight_gather_kernel<8><<<(int)nchunks, kGridThreads, 0, s>>>(g, in, pairs, chunks, partial, out);
  else if (warp_path)
    leight_accumulate_warp_kernel<<<(int)nchunks, kGridThreads, g.smem_bytes, s>>>(g, in, pairs, chunks, partial,
                                                                                     out);
  else
    leight_accumulate_kernel<<<(int)nchunks, kGridThreads, g.smem_bytes, s>>>(g, in, pairs, chunks, partial, out);
  MLG_LAUNCHED();
  if (n_split > 0) {
    leight_combine_kernel<<<n_split, kGridThreads, g.smem_bytes, s>>>(g, split, nchunk, slot_off, partial, out);
    MLG_LAUNCHED();
  }
  return MLG_OK;
}

// ---- cell-binned form ------------------------------------------------------
// A sample whose window starts at cell lo (0-based, lo_d in [1 - nWin, N_d -
// 1] for a window that meets the grid) is keyed by its corner cell e = lo +
// nWin - 1 in the corner grid E_d = N_d + nWin - 1.  Grid cell x is covered
// by the windows starting at x - nWin + 1 .. x, i.e. corner cells x .. x +
// nWin - 1: along the fastest axis these are consecutive keys, so a cell
// reads nWin^(imDim-1) contiguous runs of the sorted samples.  The sort is
// stable: within a corner cell the samples keep their input order, and each
// cell sums its runs in corner order -- deterministic from call to call.
struct CornerGrid {
  int E[3] = {1, 1, 1};
  long long E_tot = 1;
};

static CornerGrid corner_grid(const LeightGeom& g) {
  CornerGrid e;
  e.E_tot = 1;
  for (int d = 0; d < 3; ++d) {
    e.E[d] = d < g.imDim ? g.N[d] + g.nWin - 1 : 1;
    e.E_tot *= e.E[d];
  }
  return e;
}

__global__ void leight_key_kernel(LeightGeom g, CornerGrid e, LeightInputs in, int nPt, unsigned* __restrict__ keys,
                                  int* __restrict__ idx, int* __restrict__ count) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nPt; s += gridDim.x * blockDim.x) {
    float r[3];
    int lo[3];
    unsigned key = (unsigned)e.E_tot;  // missed windows sort after every corner cell
    if (sample_window(g, in, s, r, lo)) {
      const int k1 = g.imDim > 1 ? lo[1] + g.nWin - 1 : 0, k2 = g.imDim > 2 ? lo[2] + g.nWin - 1 : 0;
      key = (unsigned)(lo[0] + g.nWin - 1 + (long long)e.E[0] * (k1 + (long long)e.E[1] * k2));
      atomicAdd(count + key, 1);
    }
    keys[s] = key;
    idx[s] = s;
  }
}

// Sorted sample records: (t_x, t_y, t_z, Dn), the 1-based coordinates.
__global__ void leight_record_kernel(LeightGeom g, LeightInputs in, const int* __restrict__ sidx,
                                     const int* __restrict__ n_hits, float4* __restrict__ rec) {
  const int n = *n_hits;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const int s = __ldg(sidx + k);
    const float ty = g.imDim > 1 ? __ldg(in.ty + s) : 0.f, tz = g.imDim > 2 ? __ldg(in.tz + s) : 0.f;
    rec[k] = make_float4(__ldg(in.tx + s), ty, tz, __ldg(in.Dn + s));
  }
}

// CPT consecutive coils of sample s (split complex, [nPt][nCh]); the host
// picks CPT so that the vector loads are aligned.
template <int CPT>
__device__ __forceinline__ void load_coils(const float* __restrict__ re, const float* __restrict__ im, long long o,
                                           float* vr, float* vi) {
  if constexpr (CPT % 4 == 0) {
#pragma unroll
    for (int j = 0; j < CPT / 4; ++j) {
      const float4 a = __ldg(reinterpret_cast<const float4*>(re + o) + j);
      const float4 b = __ldg(reinterpret_cast<const float4*>(im + o) + j);
      vr[4 * j] = a.x, vr[4 * j + 1] = a.y, vr[4 * j + 2] = a.z, vr[4 * j + 3] = a.w;
      vi[4 * j] = b.x, vi[4 * j + 1] = b.y, vi[4 * j + 2] = b.z, vi[4 * j + 3] = b.w;
    }
  } else if constexpr (CPT == 2) {
    const float2 a = __ldg(reinterpret_cast<const float2*>(re + o));
    const float2 b = __ldg(reinterpret_cast<const float2*>(im + o));
    vr[0] = a.x, vr[1] = a.y, vi[0] = b.x, vi[1] = b.y;
  } else {  // scalar: 1 or a whole odd (or 6-coil) cell
#pragma unroll
    for (int c = 0; c < CPT; ++c) vr[c] = __ldg(re + o + c), vi[c] = __ldg(im + o + c);
  }
}

template <int CPT>
__device__ __forceinline__ void store_coils(float* re, float* im, long long o, const float* vr, const float* vi) {
  if constexpr (CPT % 4 == 0) {
#pragma unroll
    for (int j = 0; j < CPT / 4; ++j) {
      reinterpret_cast<float4*>(re + o)[j] = make_float4(vr[4 * j], vr[4 * j + 1], vr[4 * j + 2], vr[4 * j + 3]);
      reinterpret_cast<float4*>(im + o)[j] = make_float4(vi[4 * j], vi[4 * j + 1], vi[4 * j + 2], vi[4 * j + 3]);
    }
  } else if constexpr (CPT == 2) {
    *reinterpret_cast<float2*>(re + o) = make_float2(vr[0], vr[1]);
    *reinterpret_cast<float2*>(im + o) = make_float2(vi[0], vi[1]);
  } else {
#pragma unroll
    for (int c = 0; c < CPT; ++c) re[o + c] = vr[c], im[o + c] = vi[c];
  }
}

// Window weight of the grid cell with 1-based coordinates f for the sorted
// sample record rc (bmGridder_n2u_leight3_mex.cpp: squared distances summed
// x, y, z, then g1 exp(g2 d2) Dn).  The reference forms a distance as
// (t - node) - u with node = trunc(t + shift) and u = f - node; t - node is
// exact (Sterbenz), so that difference is the correctly rounded t - f --
// one subtraction here, the same value except where t + shift itself
// rounded across an integer (t within 2^-24 of a half-integer boundary).
__device__ __forceinline__ float cell_weight(const LeightGeom& g, float4 rc, float fx, float fy, float fz) {
  const float dx = rc.x - fx;
  float d2 = __fmul_rn(dx, dx);
  if (g.imDim > 1) {
    const float dy = rc.y - fy;
    d2 = __fadd_rn(d2, __fmul_rn(dy, dy));
  }
  if (g.imDim > 2) {
    const float dz = rc.z - fz;
    d2 = __fadd_rn(d2, __fmul_rn(dz, dz));
  }
  return __fmul_rn(__fmul_rn(g.g1, expf(__fmul_rn(g.g2, d2))), rc.w);
}

// Cells that gather more than kHeavyIncidences (sample, window cell)
// incidences leave the thread-per-cell kernel: up to kHugeIncidences (and at
// most kMidRows window rows) to a warp each, beyond that to a CTA each.
constexpr int kHeavyIncidences = 64;
constexpr int kHugeIncidences = 2048;
constexpr int kMidRows = 32;
constexpr int kHeavyCoils = 16;  // coils per pass of the mid and huge kernels

struct HeavyList {
  int* cells = nullptr;
  int* count = nullptr;
  long long cap = 0;
};

// A thread per (grid cell, CPT coils), cells in storage order.  Fused
// multiply-adds into the coil sums, weight sum and normalisation as in the
// reference (:341-344).  A cell with more than kHeavyIncidences entries is
// appended by its first thread to the mid list (leight_mid_kernel) or the
// huge list (leight_heavy_kernel).
// NW, DIM > 0: window width and dimension fixed at compile time, the
// window rows' run bounds loaded together and kept in registers (in-order
// issue would otherwise wait for each row's two loads in turn); 0: taken
// from g.
template <int CPT, int NW, int DIM>
__global__ void __launch_bounds__(256, 4) leight_cell_kernel(LeightGeom g, CornerGrid e, const int* __restrict__ off,
                                                          const int* __restrict__ sidx,
                                                          const float4* __restrict__ rec, LeightInputs in,
                                                          LeightOutput out, HeavyList mid, HeavyList huge, int y0,
                                                          int z0, int q0) {
  // block (coil group, x run): a cell's coil groups in adjacent lanes; grid
  // (x runs, y, z): no index division
  const int x = blockIdx.x * blockDim.y + threadIdx.y;
  if (x >= g.N[0]) return;
  const int y = y0 + blockIdx.y, z = z0 + blockIdx.z;
  const int c0 = (q0 + (int)threadIdx.x) * CPT;
  const int cell = x + g.N[0] * (y + g.N[1] * z);
  const int nW = NW ? NW : g.nWin, dim = DIM ? DIM : g.imDim;
  const int W1 = dim > 1 ? nW : 1, R = W1 * (dim > 2 ? nW : 1);
  constexpr int RS = NW ? (DIM == 3 ? NW * NW : (DIM == 2 ? NW : 1)) : 1;  // rows held in registers
  auto row_key = [&](int r) {  // corner grid below 2^31 cells: 32-bit keys
    const int iy = r % W1, iz = r / W1;
    return x + e.E[0] * ((y + iy) + e.E[1] * (z + iz));
  };
  int rb[RS], rn[RS];
  int total = 0;
  if constexpr (NW != 0) {
#pragma unroll
    for (int r = 0; r < RS; ++r) {
      const int rk = row_key(r);
      rb[r] = __ldg(off + rk);
      rn[r] = __ldg(off + rk + NW) - rb[r];
      total += rn[r];
    }
  } else {
    for (int r = 0; r < R; ++r) {
      const int rk = row_key(r);
      total += __ldg(off + rk + nW) - __ldg(off + rk);
    }
  }
  if (total > kHeavyIncidences) {
    if (c0 == 0) {
      const HeavyList& L = total > kHugeIncidences || R > kMidRows ? huge : mid;
      const int h = atomicAdd(L.count, 1);
      if (h < L.cap) L.cells[h] = cell;
    }
    return;
  }
  float ar[CPT], ai[CPT], ws = 0.f;
#pragma unroll
  for (int c = 0; c < CPT; ++c) ar[c] = ai[c] = 0.f;
  const float fx = (float)(x + 1), fy = (float)(y + 1), fz = (float)(z + 1);
  auto entry = [&](int k) {
    const float4 rc = __ldg(rec + k);
    const int s = __ldg(sidx + k);
    float vr[CPT], vi[CPT];
    load_coils<CPT>(in.re, in.im, (long long)s * g.nCh + c0, vr, vi);
    const float w = cell_weight(g, rc, fx, fy, fz);
    ws = __fadd_rn(ws, w);
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
      ar[c] = __fmaf_rn(w, vr[c], ar[c]);
      ai[c] = __fmaf_rn(w, vi[c], ai[c]);
    }
  };
  if constexpr (NW != 0) {
    // One loop over the cell's entries, rows in order: a warp's lanes
    // diverge once (on their totals), not once per window row.
    int r = -1, k = 0, end = 0;
    for (int i = 0; i < total; ++i) {
      if (k == end) {  // next non-empty row, selected without indexing the arrays
        int nr = RS;
#pragma unroll
        for (int j = 0; j < RS; ++j) {
          if (nr == RS && j > r && rn[j] > 0) {
            nr = j;
            k = rb[j];
            end = rb[j] + rn[j];
          }
        }
        r = nr;
      }
      entry(k++);
    }
  } else {
    for (int r = 0; r < R && total > 0; ++r) {
      const int rk = row_key(r);
      const int b = __ldg(off + rk), en = __ldg(off + rk + nW);
      for (int k = b; k < en; ++k) entry(k);
    }
  }
  // weight sums below 1e-5 leave the sums unscaled (:341-344); otherwise one
  // correctly rounded reciprocal and a multiply per value (within an ulp of
  // the reference's division); cells without samples store zeros
  if (ws >= 1e-5f) {
    const float inv = __frcp_rn(ws);
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
      ar[c] = __fmul_rn(ar[c], inv);
      ai[c] = __fmul_rn(ai[c], inv);
    }
  }
  store_coils<CPT>(out.re, out.im, (long long)cell * g.nCh + c0, ar, ai);
}

// Sums the coil chunk c0 .. c0 + nc of the cell's entries i = first, first +
// step, ... < T; the window rows' run starts b[r] and entry prefixes pre[r]
// (pre[0] = 0, pre[R] = T) are in shared memory.
template <bool VEC4>
__device__ __forceinline__ void heavy_partial(const LeightGeom& g, const int* b, const int* pre, int T, int first,
                                              int step, const float4* __restrict__ rec, const int* __restrict__ sidx,
                                              const LeightInputs& in, int c0, int nc, float fx, float fy, float fz,
                                              float* ar, float* ai, float& ws) {
  int r = 0;
  for (int i = first; i < T; i += step) {  // the rows' runs as one list
    while (pre[r + 1] <= i) ++r;
    const int k = b[r] + (i - pre[r]);
    const float4 rc = __ldg(rec + k);
    const long long o = (long long)__ldg(sidx + k) * g.nCh + c0;
    const float w = cell_weight(g, rc, fx, fy, fz);
    ws = __fadd_rn(ws, w);
    if (VEC4) {
#pragma unroll
      for (int c4 = 0; c4 < kHeavyCoils / 4; ++c4) {
        if (4 * c4 >= nc) break;
        float vr[4], vi[4];
        load_coils<4>(in.re, in.im, o + 4 * c4, vr, vi);
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          ar[4 * c4 + c] = __fmaf_rn(w, vr[c], ar[4 * c4 + c]);
          ai[4 * c4 + c] = __fmaf_rn(w, vi[c], ai[4 * c4 + c]);
        }
      }
    } else {
#pragma unroll
      for (int c = 0; c < kHeavyCoils; ++c) {
        if (c >= nc) break;
        ar[c] = __fmaf_rn(w, __ldg(in.re + o + c), ar[c]);
        ai[c] = __fmaf_rn(w, __ldg(in.im + o + c), ai[c]);
      }
    }
  }
}

// Warp sum of the coil partials in a fixed butterfly order: every lane ends
// with the totals.
__device__ __forceinline__ void warp_sum_coils(float* ar, float* ai, float& ws) {
#pragma unroll
  for (int sh = 16; sh > 0; sh >>= 1) {
    ws += __shfl_xor_sync(0xffffffffu, ws, sh);
#pragma unroll
    for (int c = 0; c < kHeavyCoils; ++c) {
      ar[c] += __shfl_xor_sync(0xffffffffu, ar[c], sh);
      ai[c] += __shfl_xor_sync(0xffffffffu, ai[c], sh);
    }
  }
}

// Mid cells (kHeavyIncidences < T <= kHugeIncidences, at most kMidRows
// window rows): a persistent grid of warps, one warp per listed cell at a
// time; lane r loads window row r's run, a warp scan forms the prefixes, the
// lanes split the entries and a butterfly sums them (deterministic).
template <bool VEC4>
__global__ void __launch_bounds__(256) leight_mid_kernel(LeightGeom g, CornerGrid e, const int* __restrict__ off,
                                                         const int* __restrict__ sidx, const float4* __restrict__ rec,
                                                         LeightInputs in, LeightOutput out, HeavyList mid) {
  __shared__ int s_b[8][kMidRows], s_pre[8][kMidRows + 1];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nm = (int)min((long long)*mid.count, mid.cap);
  const int nW = g.nWin, W1 = g.imDim > 1 ? nW : 1, R = W1 * (g.imDim > 2 ? nW : 1);
  for (int h = blockIdx.x * 8 + warp; h < nm; h += gridDim.x * 8) {
    const int cell = mid.cells[h];
    const unsigned q = (unsigned)cell / (unsigned)g.N[0];
    const int x = cell - (int)q * g.N[0];
    const int z = (int)(q / (unsigned)g.N[1]);
    const int y = (int)q - z * g.N[1];
    int b = 0, len = 0;
    if (lane < R) {
      const int rk = x + e.E[0] * ((y + lane % W1) + e.E[1] * (z + lane / W1));
      b = __ldg(off + rk);
      len = __ldg(off + rk + nW) - b;
    }
    int incl = len;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    __syncwarp();  // the previous cell's rows are read
    if (lane < R) {
      s_b[warp][lane] = b;
      s_pre[warp][lane + 1] = incl;
    }
    if (lane == 0) s_pre[warp][0] = 0;
    const int T = __shfl_sync(0xffffffffu, incl, 31);
    __syncwarp();
    const float fx = (float)(x + 1), fy = (float)(y + 1), fz = (float)(z + 1);
    for (int c0 = 0; c0 < g.nCh; c0 += kHeavyCoils) {
      const int nc = min(kHeavyCoils, g.nCh - c0);
      float ar[kHeavyCoils], ai[kHeavyCoils], ws = 0.f;
#pragma unroll
      for (int c = 0; c < kHeavyCoils; ++c) ar[c] = ai[c] = 0.f;
      heavy_partial<VEC4>(g, s_b[warp], s_pre[warp], T, lane, 32, rec, sidx, in, c0, nc, fx, fy, fz, ar, ai, ws);
      warp_sum_coils(ar, ai, ws);
      const float inv = ws < 1e-5f ? 1.0f : __frcp_rn(ws);  // as in leight_cell_kernel
#pragma unroll
      for (int c = 0; c < kHeavyCoils; ++c) {
        if (lane == c && c < nc) {
          out.re[(long long)cell * g.nCh + c0 + c] = __fmul_rn(ar[c], inv);
          out.im[(long long)cell * g.nCh + c0 + c] = __fmul_rn(ai[c], inv);
        }
      }
    }
  }
}

// Huge cells (more than kHugeIncidences entries, or more than kMidRows
// window rows): a persistent grid, one CTA per listed cell at a time.  The
// 256 threads split the cell's entries (thread t takes t, t + 256, ...),
// accumulate kHeavyCoils coils per pass, and the CTA sums the thread
// partials in a fixed tree (warp butterflies, then the eight warps in
// order): deterministic.  VEC4: nCh % 4 == 0 and 16-byte aligned input.
template <bool VEC4>
__global__ void __launch_bounds__(256) leight_heavy_kernel(LeightGeom g, CornerGrid e, const int* __restrict__ off,
                                                           const int* __restrict__ sidx,
                                                           const float4* __restrict__ rec, LeightInputs in,
                                                           LeightOutput out, HeavyList heavy) {
  __shared__ float red[8][2 * kHeavyCoils + 1];
  __shared__ int s_b[256], s_pre[257];  // the cell's window rows (nWin^2 <= 256): run start, prefix of lengths
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nh = (int)min((long long)*heavy.count, heavy.cap);
  const int nW = g.nWin, W1 = g.imDim > 1 ? nW : 1, R = W1 * (g.imDim > 2 ? nW : 1);
  for (int h = blockIdx.x; h < nh; h += gridDim.x) {
    const int cell = heavy.cells[h];
    const unsigned q = (unsigned)cell / (unsigned)g.N[0];
    const int x = cell - (int)q * g.N[0];
    const int z = (int)(q / (unsigned)g.N[1]);
    const int y = (int)q - z * g.N[1];
    for (int r = threadIdx.x; r < R; r += blockDim.x) {
      const int rk = x + e.E[0] * ((y + r % W1) + e.E[1] * (z + r / W1));
      s_b[r] = __ldg(off + rk);
      s_pre[r + 1] = __ldg(off + rk + nW) - s_b[r];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      s_pre[0] = 0;
      for (int r = 0; r < R; ++r) s_pre[r + 1] += s_pre[r];
    }
    __syncthreads();
    const int T = s_pre[R];
    const float fx = (float)(x + 1), fy = (float)(y + 1), fz = (float)(z + 1);
    for (int c0 = 0; c0 < g.nCh; c0 += kHeavyCoils) {
      const int nc = min(kHeavyCoils, g.nCh - c0);
      float ar[kHeavyCoils], ai[kHeavyCoils], ws = 0.f;
#pragma unroll
      for (int c = 0; c < kHeavyCoils; ++c) ar[c] = ai[c] = 0.f;
      heavy_partial<VEC4>(g, s_b, s_pre, T, threadIdx.x, 256, rec, sidx, in, c0, nc, fx, fy, fz, ar, ai, ws);
      warp_sum_coils(ar, ai, ws);
      if (lane == 0) {
        red[warp][0] = ws;
#pragma unroll
        for (int c = 0; c < kHeavyCoils; ++c) {
          red[warp][1 + 2 * c] = ar[c];
          red[warp][2 + 2 * c] = ai[c];
        }
      }
      __syncthreads();
      if ((int)threadIdx.x < nc) {
        const int c = threadIdx.x;
        float sw = 0.f, sr = 0.f, si = 0.f;
        for (int k = 0; k < 8; ++k) {
          sw += red[k][0];
          sr += red[k][1 + 2 * c];
          si += red[k][2 + 2 * c];
        }
        const float inv = sw < 1e-5f ? 1.0f : __frcp_rn(sw);  // as in leight_cell_kernel
        out.re[(long long)cell * g.nCh + c0 + c] = __fmul_rn(sr, inv);
        out.im[(long long)cell * g.nCh + c0 + c] = __fmul_rn(si, inv);
      }
      __syncthreads();  // red is reused by the next pass or cell
    }
  }
}

namespace {

struct CellLaunch {
  const LeightGeom& g;
  const CornerGrid& e;
  const int* off;
  const int* sidx;
  const float4* rec;
  const LeightInputs& in;
  const LeightOutput& out;
  const HeavyList& mid;
  const HeavyList& huge;
  cudaStream_t s;
};

// Compile-time rows for the common 3-wide windows in 2-D and 3-D.  Blocks
// of (coil group, x run of >= 32) threads, at most 256, so at most 8 groups
// per launch; the grid spans x runs, y and z, in launches of at most 65535
// along y and z.
template <int CPT>
void launch_cells(const CellLaunch& c) {
  const int Q = c.g.nCh / CPT, N0 = c.g.N[0], N1 = c.g.N[1], N2 = c.g.N[2];
  for (int q0 = 0; q0 < Q; q0 += 8) {
    const int nq = std::min(8, Q - q0);
    int bx = std::max(32, 256 / nq / 32 * 32);
    bx = std::min(bx, (N0 + 31) / 32 * 32);
    const dim3 block(nq, bx);
    for (int z0 = 0; z0 < N2; z0 += 65535)
      for (int y0 = 0; y0 < N1; y0 += 65535) {
        const dim3 grid((N0 + bx - 1) / bx, std::min(65535, N1 - y0), std::min(65535, N2 - z0));
        if (c.g.nWin == 3 && c.g.imDim == 3)
          leight_cell_kernel<CPT, 3, 3><<<grid, block, 0, c.s>>>(c.g, c.e, c.off, c.sidx, c.rec, c.in, c.out, c.mid,
                                                                 c.huge, y0, z0, q0);
        else if (c.g.nWin == 3 && c.g.imDim == 2)
          leight_cell_kernel<CPT, 3, 2><<<grid, block, 0, c.s>>>(c.g, c.e, c.off, c.sidx, c.rec, c.in, c.out, c.mid,
                                                                 c.huge, y0, z0, q0);
        else
          leight_cell_kernel<CPT, 0, 0><<<grid, block, 0, c.s>>>(c.g, c.e, c.off, c.sidx, c.rec, c.in, c.out, c.mid,
                                                                 c.huge, y0, z0, q0);
      }
  }
}

struct CellsLayout {
  size_t count, off, keys_in, keys_out, idx_in, idx_out, rec, mid, huge, lists_n, scan_tmp, sort_tmp, total;
  long long heavy_cap;
};

CellsLayout cells_layout(const LeightGeom& g, int nPt) {
  using W = LeightWorkspace;
  const CornerGrid e = corner_grid(g);
  const int ne = (int)(e.E_tot + 1);
  CellsLayout L;
  size_t scan_tmp = 0, sort_tmp = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, scan_tmp, (int*)nullptr, (int*)nullptr, ne);
  cub::DeviceRadixSort::SortPairs(nullptr, sort_tmp, (unsigned*)nullptr, (unsigned*)nullptr, (int*)nullptr,
                                  (int*)nullptr, std::max(nPt, 1));
  size_t p = 0;
  auto take = [&](size_t bytes) {
    const size_t at = p;
    p += W::align(bytes);
    return at;
  };
  L.count = take((size_t)ne * 4);
  L.off = take((size_t)ne * 4);
  L.keys_in = take((size_t)nPt * 4);
  L.keys_out = take((size_t)nPt * 4);
  L.idx_in = take((size_t)nPt * 4);
  L.idx_out = take((size_t)nPt * 4);
  L.rec = take((size_t)nPt * 16);
  // a heavy cell holds more than kHeavyIncidences of the at most nPt x
  // nWin^imDim incidences
  long long wc = 1;
  for (int d = 0; d < g.imDim; ++d) wc *= g.nWin;
  L.heavy_cap = std::min<long long>(g.Nu_tot, (long long)nPt * wc / (kHeavyIncidences + 1) + 1);
  L.mid = take((size_t)L.heavy_cap * 4);
  L.huge = take((size_t)L.heavy_cap * 4);
  L.lists_n = take(8);
  L.scan_tmp = take(scan_tmp);
  L.sort_tmp = take(sort_tmp);
  L.total = p;
  return L;
}

}  // namespace

size_t leight_cells_bytes(const LeightGeom& g, int nPt) { return cells_layout(g, nPt).total; }

int leight_run_cells(const LeightGeom& g, const LeightInputs& in, int nPt, const LeightOutput& out, void* ws,
                     size_t ws_bytes, cudaStream_t s) {
  NvtxRange range("leight gridder (cell-binned)");
  MLG_CHECK(in.layout == Layout::kPointSplit && out.layout == Layout::kPointSplit,
            "the cell-binned gridder takes split complex input and output");
  const CornerGrid e = corner_grid(g);
  MLG_CHECK(e.E_tot < (1LL << 31) - 1, "corner grid of %lld cells too large", e.E_tot);
  const CellsLayout L = cells_layout(g, nPt);
  MLG_CHECK(ws && ws_bytes >= L.total, "gridding workspace too small (%zu < %zu bytes)", ws_bytes, L.total);
  char* base = static_cast<char*>(ws);
  int* count = reinterpret_cast<int*>(base + L.count);
  int* off = reinterpret_cast<int*>(base + L.off);
  unsigned* keys_in = reinterpret_cast<unsigned*>(base + L.keys_in);
  unsigned* keys_out = reinterpret_cast<unsigned*>(base + L.keys_out);
  int* idx_in = reinterpret_cast<int*>(base + L.idx_in);
  int* idx_out = reinterpret_cast<int*>(base + L.idx_out);
  float4* rec = reinterpret_cast<float4*>(base + L.rec);
  const int ne = (int)(e.E_tot + 1);

  MLG_CUDA(cudaMemsetAsync(count, 0, (size_t)ne * 4, s));
  if (nPt > 0) {
    leight_key_kernel<<<grid_for(nPt), 256, 0, s>>>(g, e, in, nPt, keys_in, idx_in, count);
    MLG_LAUNCHED();
  }
  size_t scan_tmp = L.sort_tmp - L.scan_tmp;
  MLG_CUDA(cub::DeviceScan::ExclusiveSum(base + L.scan_tmp, scan_tmp, count, off, ne, s));
  if (nPt > 0) {
    size_t sort_tmp = L.total - L.sort_tmp;
    const int end_bit = 32 - __builtin_clz((unsigned)e.E_tot);  // the miss key E_tot included
    MLG_CUDA(cub::DeviceRadixSort::SortPairs(base + L.sort_tmp, sort_tmp, keys_in, keys_out, idx_in, idx_out, nPt, 0,
                                             end_bit, s));
    leight_record_kernel<<<grid_for(nPt), 256, 0, s>>>(g, in, idx_out, off + e.E_tot, rec);
    MLG_LAUNCHED();
  }
  // Coils per thread: 8 or 4 (16-byte vectors) when they divide nCh and the
  // buffers are aligned (16 coils: 8 measured fastest, ahead of 4 and 16); a
  // whole cell per thread for 3, 5, 6 or 7 coils (scalar loads); else 2 or 1.
  const uintptr_t align_bits = (uintptr_t)in.re | (uintptr_t)in.im | (uintptr_t)out.re | (uintptr_t)out.im;
  const bool a16 = align_bits % 16 == 0, a8 = align_bits % 8 == 0;
  int cpt = 1;
  if (g.nCh % 8 == 0 && a16)
    cpt = 8;
  else if (g.nCh % 4 == 0 && a16)
    cpt = 4;
  else if (g.nCh == 3 || g.nCh == 5 || g.nCh == 6 || g.nCh == 7)
    cpt = g.nCh;
  else if (g.nCh % 2 == 0 && a8)
    cpt = 2;
  HeavyList mid, huge;
  mid.cells = reinterpret_cast<int*>(base + L.mid);
  huge.cells = reinterpret_cast<int*>(base + L.huge);
  mid.count = reinterpret_cast<int*>(base + L.lists_n);
  huge.count = mid.count + 1;
  mid.cap = huge.cap = L.heavy_cap;
  MLG_CUDA(cudaMemsetAsync(mid.count, 0, 8, s));
  const CellLaunch cl{g, e, off, idx_out, rec, in, out, mid, huge, s};
  switch (cpt) {
    case 7:
      launch_cells<7>(cl);
      break;
    case 6:
      launch_cells<6>(cl);
      break;
    case 5:
      launch_cells<5>(cl);
      break;
    case 3:
      launch_cells<3>(cl);
      break;
    case 8:
      launch_cells<8>(cl);
      break;
    case 4:
      launch_cells<4>(cl);
      break;
    case 2:
      launch_cells<2>(cl);
      break;
    default:
      launch_cells<1>(cl);
  }
  MLG_LAUNCHED();
  if (nPt > 0) {  // persistent grids over the lists (lengths read on the device)
    const bool vec4 = (g.nCh % 4) == 0 && ((uintptr_t)in.re | (uintptr_t)in.im) % 16 == 0;
    const int mb = (int)std::min<long long>((L.heavy_cap + 7) / 8, 148LL * 8);
    const int hb = (int)std::min<long long>(L.heavy_cap, 148LL * 4);
    if (vec4) {
      leight_mid_kernel<true><<<mb, 256, 0, s>>>(g, e, off, idx_out, rec, in, out, mid);
      leight_heavy_kernel<true><<<hb, 256, 0, s>>>(g, e, off, idx_out, rec, in, out, huge);
    } else {
      leight_mid_kernel<false><<<mb, 256, 0, s>>>(g, e, off, idx_out, rec, in, out, mid);
      leight_heavy_kernel<false><<<hb, 256, 0, s>>>(g, e, off, idx_out, rec, in, out, huge);
    }
    MLG_LAUNCHED();
  }
  return MLG_OK;
}

// ---- precomputed-weight gridder (bmGridder_n2u_mex) -------------------------
__global__ void widen_kernel(const int* __restrict__ a, long long* __restrict__ b, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    b[i] = a[i];
}

__global__ void cells_check_kernel(const long long* __restrict__ cell, long long n, long long Nu,
                                   int* __restrict__ key, int* __restrict__ bad, int* __restrict__ cnt) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const long long c = cell[i];
    if (c < 0 || c >= Nu) {
      atomicExch(bad, 1);
      key[i] = 0;
    } else {
      key[i] = (int)c;
      atomicAdd(cnt + c, 1);
    }
  }
}

__global__ void iota_kernel(int* a, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    a[i] = (int)i;
}

__global__ void n2u_csr_fill_kernel(const int* __restrict__ ent, const float* __restrict__ w, long long n, int nNb,
                                    int* __restrict__ col, float* __restrict__ val) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int e = ent[i];
    col[i] = e / nNb;
    val[i] = w[e];
  }
}

__global__ void long_rows_kernel(const uint32_t* __restrict__ row_ptr, int l_size, int* __restrict__ list,
                                 int* __restrict__ n_long) {
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < l_size; r += (long long)gridDim.x * blockDim.x)
    if (row_ptr[r + 1] - row_ptr[r] > (uint32_t)kLongRow) list[atomicAdd(n_long, 1)] = (int)r;
}

__global__ void u32_from_i32_kernel(const int* __restrict__ a, uint32_t* __restrict__ b, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    b[i] = (uint32_t)a[i];
}

int n2u_build_csr(const float* d_w, const int* d_nJump, int nNb, int nPt, int Nu_tot, Csr& m, cudaStream_t s) {
  const long long n = (long long)nNb * nPt;
  MLG_CHECK(n < (1LL << 31), "nNb*nPt too large");
  DevBuf<long long> wide, cell;
  DevBuf<int> key, key_sorted, ent, ent_sorted, cnt, bad;
  MLG_TRY(wide.alloc(n, s));
  MLG_TRY(cell.alloc(n, s));
  MLG_TRY(key.alloc(n, s));
  MLG_TRY(key_sorted.alloc(n, s));
  MLG_TRY(ent.alloc(n, s));
  MLG_TRY(ent_sorted.alloc(n, s));
  MLG_TRY(cnt.alloc((size_t)Nu_tot + 1, s));
  MLG_TRY(bad.alloc(2, s));
  MLG_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(int) * ((size_t)Nu_tot + 1), s));
  MLG_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int) * 2, s));
  widen_kernel<<<grid_for(n), 256, 0, s>>>(d_nJump, wide.p, n);
  MLG_LAUNCHED();
  size_t tmp_bytes = 0, t2 = 0;
  cub::DeviceScan::InclusiveSum(nullptr, tmp_bytes, wide.p, cell.p, (int)n);
  cub::DeviceRadixSort::SortPairs(nullptr, t2, key.p, key_sorted.p, ent.p, ent_sorted.p, (int)n);
  cub::DeviceScan::ExclusiveSum(nullptr, t2 = std::max(t2, tmp_bytes), cnt.p, cnt.p, Nu_tot + 1);
  size_t tmpn = std::max(tmp_bytes, t2);
  {
    size_t t3 = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, t3, key.p, key_sorted.p, ent.p, ent_sorted.p, (int)n);
    tmpn = std::max(tmpn, t3);
    cub::DeviceScan::ExclusiveSum(nullptr, t3, cnt.p, cnt.p, Nu_tot + 1);
    tmpn = std::max(tmpn, t3);
  }
  DevBuf<char> tmp;
  MLG_TRY(tmp.alloc(tmpn, s));
  MLG_CUDA(cub::DeviceScan::InclusiveSum(tmp.p, tmpn, wide.p, cell.p, (int)n, s));
  cells_check_kernel<<<grid_for(n), 256, 0, s>>>(cell.p, n, Nu_tot, key.p, bad.p, cnt.p);
  MLG_LAUNCHED();
  iota_kernel<<<grid_for(n), 256, 0, s>>>(ent.p, n);
  MLG_LAUNCHED();
  int hbad = 0;
  MLG_CUDA(cudaMemcpyAsync(&hbad, bad.p, 4, cudaMemcpyDeviceToHost, s));
  MLG_CUDA(cudaStreamSynchronize(s));
  MLG_CHECK(!hbad, "nJump decodes to a cell outside [0, Nu_tot)");
  // stable radix sort by cell keeps each cell's entries in (point, neighbour)
  // order, the reference's accumulation order
  int end_bit = 1;
  while ((1LL << end_bit) < Nu_tot) ++end_bit;
  MLG_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tmpn, key.p, key_sorted.p, ent.p, ent_sorted.p, (int)n, 0, end_bit, s));
  m = Csr();
  m.r_size = nPt;
  m.l_size = Nu_tot;
  m.nnz = n;
  MLG_CUDA(cudaMalloc(&m.row_ptr, sizeof(uint32_t) * ((size_t)Nu_tot + 1)));
  MLG_CUDA(cudaMalloc(&m.col, sizeof(int) * (size_t)std::max<long long>(1, n)));
  MLG_CUDA(cudaMalloc(&m.val, sizeof(float) * (size_t)std::max<long long>(1, n)));
  MLG_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, tmpn, cnt.p, cnt.p, Nu_tot + 1, s));
  u32_from_i32_kernel<<<grid_for((long long)Nu_tot + 1), 256, 0, s>>>(cnt.p, m.row_ptr, (long long)Nu_tot + 1);
  MLG_LAUNCHED();
  n2u_csr_fill_kernel<<<grid_for(n), 256, 0, s>>>(ent_sorted.p, d_w, n, nNb, m.col, m.val);
  MLG_LAUNCHED();
  // long rows
  DevBuf<int> nl;
  MLG_TRY(nl.alloc(1, s));
  MLG_CUDA(cudaMemsetAsync(nl.p, 0, 4, s));
  int* list = nullptr;
  MLG_CUDA(cudaMalloc(&list, sizeof(int) * (size_t)Nu_tot));
  long_rows_kernel<<<grid_for(Nu_tot), 256, 0, s>>>(m.row_ptr, Nu_tot, list, nl.p);
  MLG_LAUNCHED();
  int hn = 0;
  MLG_CUDA(cudaMemcpyAsync(&hn, nl.p, 4, cudaMemcpyDeviceToHost, s));
  MLG_CUDA(cudaStreamSynchronize(s));
  m.long_rows = list;
  m.n_long = hn;
  MLG_TRY(csr_build_segments(m, s));
  return MLG_OK;
}

}  // namespace mlg

using namespace mlg;

namespace mlg {

int leight_host(int imDim, const float* aReal, const float* aImag, const float* tx, const float* ty, const float* tz,
                const float* Dn, int nCh, int nPt, const int* N, int nWin, float sigma, float* bReal, float* bImag) {
  MLG_TRY(ensure_device());
  MLG_CHECK(nPt >= 0, "nPt must be >= 0");
  MLG_CHECK(bReal && bImag, "NULL output");
  MLG_CHECK(nPt == 0 || (aReal && aImag && tx && Dn && (imDim < 2 || ty) && (imDim < 3 || tz)),
            "NULL input for nPt=%d", nPt);
  LeightGeom g;
  MLG_TRY(leight_geometry(imDim, nCh, N, nWin, sigma, g));
  cudaStream_t s = nullptr;
  const size_t na = (size_t)nPt * nCh, nb = (size_t)g.Nu_tot * nCh;
  DevBuf<float> dA, dT, dB;
  MLG_TRY(dA.alloc(2 * na + 1, s));
  MLG_TRY(dT.alloc((size_t)nPt * (imDim + 1) + 1, s));
  MLG_TRY(dB.alloc(2 * nb, s));
  if (nPt) {
    MLG_CUDA(cudaMemcpyAsync(dA.p, aReal, na * 4, cudaMemcpyHostToDevice, s));
    MLG_CUDA(cudaMemcpyAsync(dA.p + na, aImag, na * 4, cudaMemcpyHostToDevice, s));
    const float* ts[3] = {tx, ty, tz};
    for (int d = 0; d < imDim; ++d)
      MLG_CUDA(cudaMemcpyAsync(dT.p + (size_t)d * nPt, ts[d], (size_t)nPt * 4, cudaMemcpyHostToDevice, s));
    MLG_CUDA(cudaMemcpyAsync(dT.p + (size_t)imDim * nPt, Dn, (size_t)nPt * 4, cudaMemcpyHostToDevice, s));
  }
  LeightInputs in;
  in.layout = Layout::kPointSplit;
  in.re = dA.p;
  in.im = dA.p + na;
  in.tx = dT.p;
  in.ty = imDim > 1 ? dT.p + nPt : nullptr;
  in.tz = imDim > 2 ? dT.p + 2 * (size_t)nPt : nullptr;
  in.Dn = dT.p + (size_t)imDim * nPt;
  LeightOutput out;
  out.layout = Layout::kPointSplit;
  out.re = dB.p;
  out.im = dB.p + nb;
  DevBuf<char> ws;
  MLG_TRY(ws.alloc(leight_cells_bytes(g, nPt), s));
  int st = leight_run_cells(g, in, nPt, out, ws.p, ws.n, s);
  if (st == MLG_OK) {
    cudaError_t e1 = cudaMemcpyAsync(bReal, dB.p, nb * 4, cudaMemcpyDeviceToHost, s);
    cudaError_t e2 = cudaMemcpyAsync(bImag, dB.p + nb, nb * 4, cudaMemcpyDeviceToHost, s);
    if (e1 != cudaSuccess || e2 != cudaSuccess) st = fail(MLG_ERR_CUDA, "copy of the gridded data failed");
  }
  cudaError_t e = cudaStreamSynchronize(s);
  if (st == MLG_OK && e != cudaSuccess) st = fail(MLG_ERR_CUDA, "leight gridder: %s", cudaGetErrorString(e));
  return st;
}

}  // namespace mlg

extern "C" {

int mlg_gridder_n2u_leight(int imDim, const float* aReal, const float* aImag, const float* tx, const float* ty,
                           const float* tz, const float* Dn, int nCh, int nPt, int Nx, int Ny, int Nz, int nWin,
                           float kernelParam_1, float kernelParam_2, float* bReal, float* bImag) {
  (void)kernelParam_2;  // unused by the reference kernel too
  const int N[3] = {Nx, Ny, Nz};
  return leight_host(imDim, aReal, aImag, tx, ty, tz, Dn, nCh, nPt, N, nWin, kernelParam_1, bReal, bImag);
}

int mlg_gridder_n2u_leight_dev(int imDim, const float* aReal, const float* aImag, const float* tx, const float* ty,
                               const float* tz, const float* Dn, int nCh, int nPt, int Nx, int Ny, int Nz, int nWin,
                               float kernelParam_1, float kernelParam_2, float* bReal, float* bImag, void* stream) {
  (void)kernelParam_2;  // unused by the reference kernel too
  MLG_TRY(ensure_device());
  MLG_CHECK(nPt >= 0, "nPt must be >= 0");
  MLG_CHECK(bReal && bImag, "NULL output");
  MLG_CHECK(nPt == 0 || (aReal && aImag && tx && Dn && (imDim < 2 || ty) && (imDim < 3 || tz)),
            "NULL input for nPt=%d", nPt);
  const int N[3] = {Nx, Ny, Nz};
  LeightGeom g;
  MLG_TRY(leight_geometry(imDim, nCh, N, nWin, kernelParam_1, g));
  cudaStream_t s = (cudaStream_t)stream;
  LeightInputs in;
  in.layout = Layout::kPointSplit;
  in.re = aReal;
  in.im = aImag;
  in.tx = tx;
  in.ty = imDim > 1 ? ty : nullptr;
  in.tz = imDim > 2 ? tz : nullptr;
  in.Dn = Dn;
  LeightOutput out;
  out.layout = Layout::kPointSplit;
  out.re = bReal;
  out.im = bImag;
  DevBuf<char> ws;  // stream-ordered: freed after the run
  MLG_TRY(ws.alloc(leight_cells_bytes(g, nPt), s));
  return leight_run_cells(g, in, nPt, out, ws.p, ws.n, s);
}

int mlg_gridder_n2u(const float* aReal, const float* aImag, const float* w, const int* nJump, int nCh, int nNb,
                    int nPt, int Nu_tot, float* bReal, float* bImag) {
  MLG_TRY(ensure_device());
  MLG_CHECK(nCh >= 1 && nNb >= 1 && nPt >= 0 && Nu_tot >= 1, "invalid sizes");
  MLG_CHECK(bReal && bImag, "NULL output");
  MLG_CHECK(nPt == 0 || (aReal && aImag && w && nJump), "NULL input");
  cudaStream_t s = nullptr;
  const size_t na = (size_t)nPt * nCh, nb = (size_t)Nu_tot * nCh, ne = (size_t)nNb * nPt;
  DevBuf<float> dA, dW, dB;
  DevBuf<int> dJ;
  MLG_TRY(dA.alloc(2 * na + 1, s));
  MLG_TRY(dW.alloc(ne + 1, s));
  MLG_TRY(dJ.alloc(ne + 1, s));
  MLG_TRY(dB.alloc(2 * nb, s));
  if (nPt == 0) {
    MLG_CUDA(cudaMemsetAsync(dB.p, 0, 2 * nb * 4, s));
  } else {
    MLG_CUDA(cudaMemcpyAsync(dA.p, aReal, na * 4, cudaMemcpyHostToDevice, s));
    MLG_CUDA(cudaMemcpyAsync(dA.p + na, aImag, na * 4, cudaMemcpyHostToDevice, s));
    MLG_CUDA(cudaMemcpyAsync(dW.p, w, ne * 4, cudaMemcpyHostToDevice, s));
    MLG_CUDA(cudaMemcpyAsync(dJ.p, nJump, ne * 4, cudaMemcpyHostToDevice, s));
    Csr m;
    int st = n2u_build_csr(dW.p, dJ.p, nNb, nPt, Nu_tot, m, s);
    if (st != MLG_OK) {
      csr_free(m);
      return st;
    }
    SpmmArgs a;
    a.m = &m;
    a.nCh = nCh;
    a.in.layout = a.out.layout = Layout::kPointSplit;
    a.in.a = dA.p;
    a.in.b = dA.p + na;
    a.out.a = dB.p;
    a.out.b = dB.p + nb;
    a.normalize = true;
    st = spmm(a, s);
    cudaStreamSynchronize(s);
    csr_free(m);
    if (st != MLG_OK) return st;
  }
  MLG_CUDA(cudaMemcpyAsync(bReal, dB.p, nb * 4, cudaMemcpyDeviceToHost, s));
  MLG_CUDA(cudaMemcpyAsync(bImag, dB.p + nb, nb * 4, cudaMemcpyDeviceToHost, s));
  MLG_CUDA(cudaStreamSynchronize(s));
  return MLG_OK;
}

}  // extern "C"
