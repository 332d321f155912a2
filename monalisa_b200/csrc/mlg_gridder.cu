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

int leight_run(const LeightGeom& g, const LeightInputs& in, int nPt, const LeightOutput& out, LeightWorkspace& ws,
               cudaStream_t s) {
  MLG_CHECK(g.ntiles < (1LL << 31), "too many tiles");
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

namespace {

int grow_bins_pool(LeightWorkspace& ws, size_t bytes, cudaStream_t s) {
  if (ws.bins) dev_free(ws.bins, s);
  ws.bins = nullptr;
  ws.bins_cap = 0;
  MLG_TRY(dev_alloc(&ws.bins, bytes, s));
  ws.bins_cap = bytes;
  return MLG_OK;
}

}  // namespace

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
  DevBuf<char> counters;
  MLG_TRY(counters.alloc(LeightWorkspace::counters_bytes(g), s));
  LeightWorkspace ws;
  ws.counters = counters.p;
  ws.counters_cap = counters.n;
  ws.grow_bins = grow_bins_pool;
  int st = leight_run(g, in, nPt, out, ws, s);
  if (st == MLG_OK) {
    cudaError_t e1 = cudaMemcpyAsync(bReal, dB.p, nb * 4, cudaMemcpyDeviceToHost, s);
    cudaError_t e2 = cudaMemcpyAsync(bImag, dB.p + nb, nb * 4, cudaMemcpyDeviceToHost, s);
    if (e1 != cudaSuccess || e2 != cudaSuccess) st = fail(MLG_ERR_CUDA, "copy of the gridded data failed");
  }
  if (ws.bins) dev_free(ws.bins, s);
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
  DevBuf<char> counters;
  MLG_TRY(counters.alloc(LeightWorkspace::counters_bytes(g), s));
  LeightWorkspace ws;
  ws.counters = counters.p;
  ws.counters_cap = counters.n;
  ws.grow_bins = grow_bins_pool;
  const int st = leight_run(g, in, nPt, out, ws, s);
  if (ws.bins) dev_free(ws.bins, s);  // stream-ordered: freed after the run
  return st;
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
