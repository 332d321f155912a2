// Sparse gridding-matrix products on the device (Gu / Gut / Gn and the
// generic bmSparseMat_vec family).
//
// The reference (bmSparseMat_cC_oBlock_omp_mex.cpp:106-260) streams the whole
// matrix once per coil and per real/imaginary part.  Here one launch covers
// every coil: a thread owns one (row, coil) output and walks the row's
// entries in stored order with explicit round-to-nearest multiply and add
// (no FMA contraction), so short rows reproduce the reference's
// floating-point result bit for bit.  Rows longer than kLongRow entries (the
// k-space centre of Gut, which every radial spoke crosses) get a whole CTA
// that splits the entries over thread groups and reduces the partial sums in
// a fixed order.
//
// Two thread mappings: coil-fastest (lanes of a warp = coils of one row;
// used when the output is coil-fastest, e.g. Gu -> k-space) and row-fastest
// (lanes = consecutive rows of one coil; used when the output is coil-major,
// e.g. Gut -> grid), so the output side is always coalesced.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "mlg_internal.cuh"

namespace mlg {

struct SpmmParams {
  const uint32_t* row_ptr;
  const int* col;
  const float* val;
  const __half* val_h;  // FP16 values in place of val when set
  int l_size;
  int nCh;
  int rows_per_block;
  const int* long_rows;
  int n_long;
  Operand in;
  Operand out;
  const float* in_row_scale;
  float out_scale;
  int normalize;
  const float* sqn_w;
  double* partial;
  int partial_long_offset;
  unsigned* absmax;
  // FP16 point-layout input (pair kernel, IN_H): scale from this word and length
  const unsigned* in_h_amax;
  int in_h_len;
};

__device__ __forceinline__ float abs_max4(float4 v) {
  return fmaxf(fmaxf(fabsf(v.x), fabsf(v.y)), fmaxf(fabsf(v.z), fabsf(v.w)));
}

// The block's largest value (v >= 0) into *absmax: one atomic per block, and
// none when the recorded value is already as large -- atomics on one word
// serialise, and a product has thousands of blocks.  Every thread of the
// block must call.
__device__ __forceinline__ void block_absmax(unsigned* absmax, float v) {
  __shared__ float wmax[32];
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    float m = 0.f;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = fmaxf(m, wmax[w]);
    const unsigned u = __float_as_uint(m);
    if (u > *reinterpret_cast<volatile const unsigned*>(absmax)) atomicMax(absmax, u);
  }
}

template <Layout L>
__device__ __forceinline__ float2 ld(const Operand& o, long long row, int c, int nCh) {
  if constexpr (L == Layout::kPointC64) {
    return __ldg(reinterpret_cast<const float2*>(o.a) + row * nCh + c);
  } else if constexpr (L == Layout::kCoilC64) {
    return __ldg(reinterpret_cast<const float2*>(o.a) + (long long)c * o.rows + row);
  } else if constexpr (L == Layout::kCoilSplit) {
    const long long i = (long long)c * o.rows + row;
    return make_float2(__ldg(reinterpret_cast<const float*>(o.a) + i), __ldg(reinterpret_cast<const float*>(o.b) + i));
  } else if constexpr (L == Layout::kPointSplit) {
    const long long i = row * nCh + c;
    return make_float2(__ldg(reinterpret_cast<const float*>(o.a) + i), __ldg(reinterpret_cast<const float*>(o.b) + i));
  } else if constexpr (L == Layout::kPointReal) {
    return make_float2(__ldg(reinterpret_cast<const float*>(o.a) + row * nCh + c), 0.f);
  } else {
    return make_float2(__ldg(reinterpret_cast<const float*>(o.a) + (long long)c * o.rows + row), 0.f);
  }
}

template <Layout L>
__device__ __forceinline__ void st(const Operand& o, long long row, int c, int nCh, float2 v) {
  if constexpr (L == Layout::kPointC64) {
    reinterpret_cast<float2*>(o.a)[row * nCh + c] = v;
  } else if constexpr (L == Layout::kCoilC64) {
    reinterpret_cast<float2*>(o.a)[(long long)c * o.rows + row] = v;
  } else if constexpr (L == Layout::kCoilSplit) {
    const long long i = (long long)c * o.rows + row;
    reinterpret_cast<float*>(o.a)[i] = v.x;
    reinterpret_cast<float*>(o.b)[i] = v.y;
  } else if constexpr (L == Layout::kPointSplit) {
    const long long i = row * nCh + c;
    reinterpret_cast<float*>(o.a)[i] = v.x;
    reinterpret_cast<float*>(o.b)[i] = v.y;
  } else if constexpr (L == Layout::kPointReal) {
    reinterpret_cast<float*>(o.a)[row * nCh + c] = v.x;
  } else {
    reinterpret_cast<float*>(o.a)[(long long)c * o.rows + row] = v.x;
  }
}

__device__ __forceinline__ float val_at(const SpmmParams& p, uint32_t k) {
  return p.val_h ? __half2float(p.val_h[k]) : __ldg(p.val + k);
}

// Accumulates entries [b, e) with stride `step` of one row for coil c.
template <Layout IN>
__device__ __forceinline__ void accumulate(const SpmmParams& p, uint32_t b, uint32_t e, uint32_t step, int c,
                                           float& ax, float& ay, float& ws) {
  const bool scale = p.in_row_scale != nullptr;
#pragma unroll 4
  for (uint32_t k = b; k < e; k += step) {
    const int j = __ldg(p.col + k);
    const float m = val_at(p, k);
    float2 v = ld<IN>(p.in, j, c, p.nCh);
    if (scale) {
      const float h = __ldg(p.in_row_scale + j);
      v.x = __fmul_rn(h, v.x);
      v.y = __fmul_rn(h, v.y);
    }
    ax = __fadd_rn(ax, __fmul_rn(m, v.x));
    ay = __fadd_rn(ay, __fmul_rn(m, v.y));
    ws = __fadd_rn(ws, m);
  }
}

template <Layout OUT>
__device__ __forceinline__ double finish(const SpmmParams& p, long long r, int c, float ax, float ay, float ws) {
  if (p.normalize) {
    // bmGridder_n2u_mex.cpp:178-191: divide by the weight sum, 1 if < 1e-5
    const float s = ws < 1e-5f ? 1.0f : ws;
    ax = __fdiv_rn(ax, s);
    ay = __fdiv_rn(ay, s);
  }
  if (p.out_scale != 1.0f) {
    ax = __fmul_rn(ax, p.out_scale);
    ay = __fmul_rn(ay, p.out_scale);
  }
  st<OUT>(p.out, r, c, p.nCh, make_float2(ax, ay));
  if (p.absmax) atomicMax(p.absmax, __float_as_uint(fmaxf(fabsf(ax), fabsf(ay))));
  if (p.partial) {
    const double w = p.sqn_w ? (double)__ldg(p.sqn_w + r) : 1.0;
    return w * ((double)ax * ax + (double)ay * ay);
  }
  return 0.0;
}

__device__ __forceinline__ double block_sum(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0) {
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += sh[i];
  }
  return t;
}

template <Layout IN, Layout OUT, bool ROW_FAST>
__global__ void __launch_bounds__(256) spmm_short_kernel(SpmmParams p) {
  __shared__ double sh[32];
  const long long r0 = (long long)blockIdx.x * p.rows_per_block;
  const int nrows = (int)min((long long)p.rows_per_block, (long long)p.l_size - r0);
  const int items = nrows * p.nCh;
  double sq = 0.0;
  for (int it = threadIdx.x; it < items; it += blockDim.x) {
    int lr, c;
    if (ROW_FAST) {
      lr = it % nrows;
      c = it / nrows;
    } else {
      c = it % p.nCh;
      lr = it / p.nCh;
    }
    const long long r = r0 + lr;
    const uint32_t b = __ldg(p.row_ptr + r), e = __ldg(p.row_ptr + r + 1);
    if (e - b > (uint32_t)kLongRow) continue;  // owned by spmm_long_kernel
    float ax = 0.f, ay = 0.f, ws = 0.f;
    accumulate<IN>(p, b, e, 1u, c, ax, ay, ws);
    sq += finish<OUT>(p, r, c, ax, ay, ws);
  }
  if (p.partial) {
    const double t = block_sum(sq, sh);
    if (threadIdx.x == 0) p.partial[blockIdx.x] = t;
  }
}

// Long rows: one CTA per segment of at most kSegLen entries.  Thread groups
// of `cper` coils split the segment's entries (stride = number of groups);
// the group partials are summed in group order and written, per coil, to
// seg_scratch[segment][coil] = (re, im, weight sum).
template <Layout IN>
__global__ void __launch_bounds__(256) spmm_seg_kernel(SpmmParams p, const uint32_t* __restrict__ seg_lo,
                                                       const uint32_t* __restrict__ seg_hi, float3* scratch) {
  __shared__ float3 part[256];
  const uint32_t b = __ldg(seg_lo + blockIdx.x), e = __ldg(seg_hi + blockIdx.x);
  const int cper = min(p.nCh, (int)blockDim.x);   // coils per pass
  const int groups = (int)blockDim.x / cper;      // entry groups per coil
  for (int c0 = 0; c0 < p.nCh; c0 += cper) {
    const int cl = threadIdx.x % cper, g = threadIdx.x / cper;
    const int c = c0 + cl;
    float ax = 0.f, ay = 0.f, ws = 0.f;
    if (g < groups && c < p.nCh) accumulate<IN>(p, b + g, e, (uint32_t)groups, c, ax, ay, ws);
    __syncthreads();
    part[threadIdx.x] = make_float3(ax, ay, ws);
    __syncthreads();
    if ((int)threadIdx.x < cper && c0 + (int)threadIdx.x < p.nCh) {
      float sx = 0.f, sy = 0.f, sw = 0.f;
      for (int gg = 0; gg < groups; ++gg) {  // fixed order: deterministic
        const float3 q = part[gg * cper + threadIdx.x];
        sx = __fadd_rn(sx, q.x);
        sy = __fadd_rn(sy, q.y);
        sw = __fadd_rn(sw, q.z);
      }
      scratch[(long long)blockIdx.x * p.nCh + c0 + threadIdx.x] = make_float3(sx, sy, sw);
    }
  }
}

// One CTA per long row: sums its segments in segment order, then finishes
// (normalise / scale / store / FP64 partial) like the short-row kernel.
template <Layout OUT>
__global__ void __launch_bounds__(256) spmm_seg_combine_kernel(SpmmParams p, const int* __restrict__ seg0,
                                                               const float3* __restrict__ scratch) {
  __shared__ double sh[32];
  const long long r = __ldg(p.long_rows + blockIdx.x);
  const int s0 = __ldg(seg0 + blockIdx.x), s1 = __ldg(seg0 + blockIdx.x + 1);
  double sq = 0.0;
  for (int c = threadIdx.x; c < p.nCh; c += blockDim.x) {
    float sx = 0.f, sy = 0.f, sw = 0.f;
    for (int k = s0; k < s1; ++k) {
      const float3 q = scratch[(long long)k * p.nCh + c];
      sx = __fadd_rn(sx, q.x);
      sy = __fadd_rn(sy, q.y);
      sw = __fadd_rn(sw, q.z);
    }
    sq += finish<OUT>(p, r, c, sx, sy, sw);
  }
  if (p.partial) {
    const double t = block_sum(sq, sh);
    if (threadIdx.x == 0) p.partial[p.partial_long_offset + blockIdx.x] = t;
  }
}

// Point layout in and out, even nCh: a thread owns a (row, coil pair) output
// and moves 16 bytes per load/store; the row's column/value stream is read
// once per pair instead of once per coil.  `rows` (optional) lists the rows
// to compute, in that order (the matrix's ord_rows: non-empty rows, or all
// rows, in blocks of nearby cells), and `bounds` their entry ranges; other
// rows are left untouched.  Entries
// are summed in stored order with round-to-nearest multiply/add, or, with
// CONTRACT (operators inside plans), with the row scale folded into the
// matrix value and fused multiply-adds: 9 instead of 16 arithmetic and load
// instructions per entry and coil pair.
// A coil pair: two complex values (float4) in and out.

struct MidRows {
  const int* rows = nullptr;
  const uint2* bounds = nullptr;
  int n = 0;
  int blocks = 0;
};

// Rows with kMidRow < n <= kLongRow entries inside the operators (CONTRACT
// semantics, FP32 point layout in and out, no partials): a warp per row at
// a time, lane = (entry group eg, coil pair pi) for P <= 16 pairs, EG = 32 /
// P groups; group eg takes entries eg, eg + EG, ... and the groups' sums are
// added in group order (a fixed order: deterministic, but not the row's
// stored order).  AM: p.absmax is raised to the largest output component.
template <bool AM>
__device__ __forceinline__ void mid_rows_block(const SpmmParams& p, const int* __restrict__ rows,
                                               const uint2* __restrict__ bounds, int n_rows, int block,
                                               int nblocks) {
  const int P = p.nCh >> 1, EG = 32 / P;
  const int lane = threadIdx.x & 31, eg = lane / P, pi = lane - eg * P;
  const bool active = eg < EG;
  const bool scale = p.in_row_scale != nullptr;
  const float4* in = reinterpret_cast<const float4*>(p.in.a);
  float amax = 0.f;
  for (int i = block * 8 + (int)(threadIdx.x >> 5); i < n_rows; i += nblocks * 8) {
    const uint2 be = __ldg(bounds + i);
    if (be.y - be.x > (uint32_t)kLongRow) continue;  // segment kernels own it (uniform in the warp)
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    if (active) {
      for (uint32_t k = be.x + eg; k < be.y; k += EG) {
        const int j = __ldg(p.col + k);
        float m = val_at(p, k);
        if (scale) m = __fmul_rn(m, __ldg(p.in_row_scale + j));
        const float4 v = __ldg(in + (long long)j * P + pi);
        acc.x = __fmaf_rn(m, v.x, acc.x);
        acc.y = __fmaf_rn(m, v.y, acc.y);
        acc.z = __fmaf_rn(m, v.z, acc.z);
        acc.w = __fmaf_rn(m, v.w, acc.w);
      }
    }
    float4 s = acc;
    for (int e = 1; e < EG; ++e) {  // lanes of group 0 add the other groups in order
      const int src = pi + e * P;
      s.x += __shfl_sync(0xffffffffu, acc.x, src);
      s.y += __shfl_sync(0xffffffffu, acc.y, src);
      s.z += __shfl_sync(0xffffffffu, acc.z, src);
      s.w += __shfl_sync(0xffffffffu, acc.w, src);
    }
    if (eg == 0) {
      if (p.out_scale != 1.0f)
        s = make_float4(__fmul_rn(s.x, p.out_scale), __fmul_rn(s.y, p.out_scale), __fmul_rn(s.z, p.out_scale),
                        __fmul_rn(s.w, p.out_scale));
      reinterpret_cast<float4*>(p.out.a)[(long long)__ldg(rows + i) * P + pi] = s;
      if constexpr (AM) amax = fmaxf(amax, abs_max4(s));
    }
  }
  if constexpr (AM) block_absmax(p.absmax, amax);  // every thread of the block reaches it
}

// PPT coil pairs per thread: the row's bounds and each entry's column and
// value are loaded once for PPT pairs.  Per coil the entries are summed in
// the same order for every PPT, so the outputs do not depend on it.
// Resident blocks per SM: the gathers are latency-bound, so occupancy beats
// spill-free code -- one pair per thread at 8 blocks (32 registers, a few
// spilled bytes) took Gut on the 4096-spoke 16-coil koosh case from 0.757
// (6 blocks) to 0.671 ms; 5 blocks gave 0.841 ms.
template <int PPT>
constexpr int pair_min_blocks() {
  return PPT == 1 ? 8 : (PPT == 2 ? 5 : 4);
}

// With mid_blocks > 0 (CONTRACT, FP32 output) the first mid_blocks blocks
// gather the mid rows, a warp per row (mid_rows_block), and the others the
// listed short rows: one launch, the long-running mid rows started first.
// IN_H: the input holds __half2 values times a power of two (the
// mixed-precision forward grid; the scale as its writer computed it from
// p.in_h_amax / p.in_h_len), read as 8 bytes per coil pair.
template <bool CONTRACT, int PPT, bool IN_H = false>
__global__ void __launch_bounds__(256, pair_min_blocks<PPT>()) spmm_pair_kernel(SpmmParams p,
                                                                               const int* __restrict__ rows,
                                                                               const uint2* __restrict__ bounds,
                                                                               int n_rows, MidRows mid) {
  __shared__ double sh[32];
  if ((int)blockIdx.x < mid.blocks) {
    if constexpr (CONTRACT) {
      if (p.absmax)
        mid_rows_block<true>(p, mid.rows, mid.bounds, mid.n, blockIdx.x, mid.blocks);
      else
        mid_rows_block<false>(p, mid.rows, mid.bounds, mid.n, blockIdx.x, mid.blocks);
    }
    return;
  }
  const int bid = (int)blockIdx.x - mid.blocks;
  const int P = p.nCh >> 1, G = P / PPT;  // pairs per row, thread groups per row
  const long long i0 = (long long)bid * p.rows_per_block;
  const int nr = (int)min((long long)p.rows_per_block, (long long)n_rows - i0);
  const int total = nr * G;
  const bool scale = p.in_row_scale != nullptr;
  const float hin = IN_H ? 1.f / half_store_scale(p.in_h_amax, p.in_h_len) : 1.f;  // a power of two
  float amax = 0.f;
  double sq = 0.0;
  // item -> row, first coil pair and entry range (empty for rows the segment kernels own)
  auto fetch = [&](int it, long long& r, int& pi, uint32_t& b, uint32_t& n) {
    const int lr = it / G;
    pi = (it - lr * G) * PPT;
    uint32_t e;
    if (rows) {  // listed rows: bounds loaded beside the row index, not after it
      r = __ldg(rows + i0 + lr);
      const uint2 be = __ldg(bounds + i0 + lr);
      b = be.x;
      e = be.y;
    } else {
      r = i0 + lr;
      b = __ldg(p.row_ptr + r);
      e = __ldg(p.row_ptr + r + 1);
    }
    n = e - b;
  };
  auto entry = [&](uint32_t k, int pi, float4* acc) {
    const int j = __ldg(p.col + k);
    float m = val_at(p, k);
    float4 v[PPT];
    if constexpr (IN_H) {
      const uint2* src = reinterpret_cast<const uint2*>(p.in.a) + (long long)j * P + pi;
#pragma unroll
      for (int u = 0; u < PPT; ++u) {
        const uint2 q = __ldg(src + u);
        const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&q.x));
        const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&q.y));
        v[u] = make_float4(a.x * hin, a.y * hin, b.x * hin, b.y * hin);
      }
    } else {
      const float4* src = reinterpret_cast<const float4*>(p.in.a) + (long long)j * P + pi;
#pragma unroll
      for (int u = 0; u < PPT; ++u) v[u] = __ldg(src + u);
    }
    if constexpr (CONTRACT) {
      if (scale) m = __fmul_rn(m, __ldg(p.in_row_scale + j));
#pragma unroll
      for (int u = 0; u < PPT; ++u) {
        acc[u].x = __fmaf_rn(m, v[u].x, acc[u].x);
        acc[u].y = __fmaf_rn(m, v[u].y, acc[u].y);
        acc[u].z = __fmaf_rn(m, v[u].z, acc[u].z);
        acc[u].w = __fmaf_rn(m, v[u].w, acc[u].w);
      }
    } else {
      const float h = scale ? __ldg(p.in_row_scale + j) : 1.f;
#pragma unroll
      for (int u = 0; u < PPT; ++u) {
        float4 w = v[u];
        if (scale) w = make_float4(__fmul_rn(h, w.x), __fmul_rn(h, w.y), __fmul_rn(h, w.z), __fmul_rn(h, w.w));
        acc[u].x = __fadd_rn(acc[u].x, __fmul_rn(m, w.x));
        acc[u].y = __fadd_rn(acc[u].y, __fmul_rn(m, w.y));
        acc[u].z = __fadd_rn(acc[u].z, __fmul_rn(m, w.z));
        acc[u].w = __fadd_rn(acc[u].w, __fmul_rn(m, w.w));
      }
    }
  };
  auto finish_pair = [&](long long r, int pi, float4 acc, double w) {
    if (p.out_scale != 1.0f)
      acc = make_float4(__fmul_rn(acc.x, p.out_scale), __fmul_rn(acc.y, p.out_scale), __fmul_rn(acc.z, p.out_scale),
                        __fmul_rn(acc.w, p.out_scale));
    reinterpret_cast<float4*>(p.out.a)[r * P + pi] = acc;
    amax = fmaxf(amax, abs_max4(acc));
    if (p.partial)
      sq += w * ((double)acc.x * acc.x + (double)acc.y * acc.y + (double)acc.z * acc.z + (double)acc.w * acc.w);
  };
  for (int it = threadIdx.x; it < total; it += blockDim.x) {
    long long r;
    int pi;
    uint32_t b, n;
    fetch(it, r, pi, b, n);
    if (n > (uint32_t)kLongRow) continue;  // segment kernels own it
    float4 acc[PPT];
#pragma unroll
    for (int u = 0; u < PPT; ++u) acc[u] = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll 4
    for (uint32_t k = b; k < b + n; ++k) entry(k, pi, acc);
    const double w = p.partial && p.sqn_w ? (double)__ldg(p.sqn_w + r) : 1.0;
#pragma unroll
    for (int u = 0; u < PPT; ++u) finish_pair(r, pi + u, acc[u], w);
  }
  if (p.absmax) block_absmax(p.absmax, amax);
  if (p.partial) {
    const double t = block_sum(sq, sh);
    if (threadIdx.x == 0) p.partial[bid] = t;
  }
}

template <int PPT>
static void launch_pair_ppt(bool contract, const SpmmParams& p, const int* rows, const uint2* rp, int nrows, int grid,
                            const MidRows& mid, cudaStream_t s) {
  grid += mid.blocks;
  if (p.in_h_amax)  // FP16 input: contracted operator products only (checked by spmm)
    spmm_pair_kernel<true, PPT, true><<<grid, 256, 0, s>>>(p, rows, rp, nrows, mid);
  else if (contract)
    spmm_pair_kernel<true, PPT><<<grid, 256, 0, s>>>(p, rows, rp, nrows, mid);
  else
    spmm_pair_kernel<false, PPT><<<grid, 256, 0, s>>>(p, rows, rp, nrows, mid);
}

static void launch_pair(int ppt, bool contract, const SpmmParams& p, const int* rows, const uint2* rp, int nrows,
                        int grid, const MidRows& mid, cudaStream_t s) {
  (void)ppt;  // one pair per thread (pair_ppt)
  launch_pair_ppt<1>(contract, p, rows, rp, nrows, grid, mid, s);
}

// Short rows of an ordered non-empty product from their records (CONTRACT,
// FP32 point layout in and out): a thread per (row, coil pair) reads the
// row's 32-byte record -- cell, count and up to kRecInline (column, value)
// pairs -- and issues every gather of the row at once, so such a row costs
// two dependent loads (record -> inputs) instead of three (bounds -> entry ->
// input), and the record stream is smaller than the bounds and entries it
// replaces.  Rows with more entries loop over their CSR entries.  Per coil
// the entries are summed in stored order with the same fused multiply-adds
// as spmm_pair_kernel: the outputs are identical.  With FP16 matrix values
// (p.val_h) the inline FP32 values are rounded to FP16 as they are read,
// which gives the values the CSR rows read from val_h.  The first mid.blocks
// blocks gather the mid rows a warp each, as there.  p.absmax (optional) is
// raised to the largest output component.  Eight blocks per SM, as the pair
// kernel.
// (Loading two rows' records before either row's gathers -- two rows in
// flight per thread at five blocks per SM, the registers of two records --
// measured slower on c2: 0.709 against 0.610 ms.)
template <bool HV, bool AM>
__global__ void __launch_bounds__(256, 8) spmm_rec_kernel(SpmmParams p, const uint4* __restrict__ rec, int n_rows,
                                                          MidRows mid) {
  if ((int)blockIdx.x < mid.blocks) {
    mid_rows_block<AM>(p, mid.rows, mid.bounds, mid.n, blockIdx.x, mid.blocks);
    return;
  }
  const int bid = (int)blockIdx.x - mid.blocks;
  const int P = p.nCh >> 1;
  const long long i0 = (long long)bid * p.rows_per_block;
  const int nr = (int)min((long long)p.rows_per_block, (long long)n_rows - i0);
  const int total = nr * P;
  const bool scale = p.in_row_scale != nullptr;
  const float4* in = reinterpret_cast<const float4*>(p.in.a);
  float amax = 0.f;
  auto row = [&](const uint4 h0, const uint4 h1, const int pi) {
    const long long r = (int)h0.x;
    const uint32_t n = h0.y;
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    auto fma4 = [&](float m, float4 v) {
      acc.x = __fmaf_rn(m, v.x, acc.x);
      acc.y = __fmaf_rn(m, v.y, acc.y);
      acc.z = __fmaf_rn(m, v.z, acc.z);
      acc.w = __fmaf_rn(m, v.w, acc.w);
    };
    if (n <= (uint32_t)kRecInline) {
      const uint32_t c0 = h0.z, c1 = h1.x, c2 = h1.z;
      float4 v0 = make_float4(0.f, 0.f, 0.f, 0.f), v1 = v0, v2 = v0;
      float m0 = __uint_as_float(h0.w), m1 = __uint_as_float(h1.y), m2 = __uint_as_float(h1.w);
      if constexpr (HV) {  // FP16 matrix values: the inline FP32 values rounded alike
        m0 = __half2float(__float2half_rn(m0));
        m1 = __half2float(__float2half_rn(m1));
        m2 = __half2float(__float2half_rn(m2));
      }
      if (n > 0) v0 = __ldg(in + (long long)c0 * P + pi);
      if (n > 1) v1 = __ldg(in + (long long)c1 * P + pi);
      if (n > 2) v2 = __ldg(in + (long long)c2 * P + pi);
      if (scale) {
        if (n > 0) m0 = __fmul_rn(m0, __ldg(p.in_row_scale + c0));
        if (n > 1) m1 = __fmul_rn(m1, __ldg(p.in_row_scale + c1));
        if (n > 2) m2 = __fmul_rn(m2, __ldg(p.in_row_scale + c2));
      }
      if (n > 0) fma4(m0, v0);
      if (n > 1) fma4(m1, v1);
      if (n > 2) fma4(m2, v2);
    } else {
      const uint32_t b = h0.z;
#pragma unroll 4
      for (uint32_t k = b; k < b + n; ++k) {
        const int j = __ldg(p.col + k);
        float m = HV ? __half2float(p.val_h[k]) : __ldg(p.val + k);
        const float4 v = __ldg(in + (long long)j * P + pi);
        if (scale) m = __fmul_rn(m, __ldg(p.in_row_scale + j));
        fma4(m, v);
      }
    }
    if (p.out_scale != 1.0f)
      acc = make_float4(__fmul_rn(acc.x, p.out_scale), __fmul_rn(acc.y, p.out_scale), __fmul_rn(acc.z, p.out_scale),
                        __fmul_rn(acc.w, p.out_scale));
    reinterpret_cast<float4*>(p.out.a)[r * P + pi] = acc;
    if constexpr (AM) amax = fmaxf(amax, abs_max4(acc));
  };
  for (int it = threadIdx.x; it < total; it += blockDim.x) {
    const int lr = it / P;
    const uint4* rp = rec + (i0 + lr) * 2;
    row(__ldg(rp), __ldg(rp + 1), it - lr * P);
  }
  if constexpr (AM) block_absmax(p.absmax, amax);
}

__global__ void rec_build_kernel(const int* __restrict__ rows, const uint2* __restrict__ bounds, int n,
                                 const int* __restrict__ col, const float* __restrict__ val,
                                 uint32_t* __restrict__ rec) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint2 be = bounds[i];
    const uint32_t len = be.y - be.x;
    uint32_t w[8] = {};
    w[0] = (uint32_t)rows[i];
    w[1] = len;
    if (len <= (uint32_t)kRecInline) {
      for (uint32_t k = 0; k < len; ++k) {
        w[2 + 2 * k] = (uint32_t)col[be.x + k];
        w[3 + 2 * k] = __float_as_uint(val[be.x + k]);
      }
    } else {
      w[2] = be.x;
    }
    uint4* o = reinterpret_cast<uint4*>(rec) + 2 * (size_t)i;
    o[0] = make_uint4(w[0], w[1], w[2], w[3]);
    o[1] = make_uint4(w[4], w[5], w[6], w[7]);
  }
}

// MLG_GUT_REC=0 / 1 forces the CSR rows / the records in every product;
// unset: SpmmArgs::records (the plan's variant) decides.
static int records_forced() {
  static const int v = [] {
    const char* e = std::getenv("MLG_GUT_REC");
    return e ? (std::strcmp(e, "0") == 0 ? 0 : (std::strcmp(e, "1") == 0 ? 1 : -1)) : -1;
  }();
  return v;
}

int csr_build_records(Csr& c, cudaStream_t s) {
  if (c.ord_rec || !c.ord_rows || !c.ord_nonempty || c.ord_short <= 0 || !c.val) return MLG_OK;
  MLG_CUDA(cudaMalloc(&c.ord_rec, 32 * (size_t)c.ord_short));
  const int g = std::max(1, std::min(148 * 16, (c.ord_short + 255) / 256));
  rec_build_kernel<<<g, 256, 0, s>>>(c.ord_rows, c.ord_bounds, c.ord_short, c.col, c.val, c.ord_rec);
  MLG_LAUNCHED();
  return MLG_OK;
}

static bool use_pair_kernel(const SpmmArgs& a) {
  return a.in.layout == Layout::kPointC64 &&
         a.out.layout == Layout::kPointC64 && (a.nCh % 2) == 0 &&
         !a.normalize;
}

// Coil pairs per thread of the pair kernel, as measured on a B200: one.
// With eight 256-thread blocks per SM (32 registers) one pair per thread
// matched two on the 4096 x 256-sample 16-coil Gu (0.381 vs 0.379 ms) and
// beat it on a 1500-spoke one (0.164 vs 0.174 ms); at lower occupancy two
// pairs had helped only that 16-coil Gu and slowed 12- and 8-coil products
// and the non-empty-row Gut.
static int pair_ppt(const SpmmArgs&) { return 1; }

static int rows_per_block(const SpmmArgs& a) {
  if (use_pair_kernel(a)) return std::max(1, 1024 / (a.nCh / 2 / pair_ppt(a)));
  return std::max(1, 1024 / std::max(1, a.nCh));
}

static long long spmm_rows(const SpmmArgs& a) { return a.nonempty_only ? a.m->n_nonempty : a.m->l_size; }

int spmm_partial_count(const SpmmArgs& a) {
  const int rpb = rows_per_block(a);
  return (int)((spmm_rows(a) + rpb - 1) / rpb) + a.m->n_long;
}

size_t spmm_scratch_floats(const Csr& m, int nCh) { return 3 * (size_t)m.n_seg * (size_t)nCh; }

template <Layout IN, Layout OUT, bool ROW_FAST>
static int launch(const SpmmParams& p, const Csr& m, float3* scratch, int grid_short, cudaStream_t s) {
  if (grid_short > 0) {
    spmm_short_kernel<IN, OUT, ROW_FAST><<<grid_short, 256, 0, s>>>(p);
    MLG_LAUNCHED();
  }
  if (p.n_long > 0) {
    spmm_seg_kernel<IN><<<m.n_seg, 256, 0, s>>>(p, m.seg_lo, m.seg_hi, scratch);
    MLG_LAUNCHED();
    spmm_seg_combine_kernel<OUT><<<p.n_long, 256, 0, s>>>(p, m.long_seg0, scratch);
    MLG_LAUNCHED();
  }
  return MLG_OK;
}

int spmm(const SpmmArgs& a, cudaStream_t s) {
  const Csr& m = *a.m;
  MLG_CHECK(a.nCh >= 1, "nCh must be >= 1");
  SpmmParams p;
  p.row_ptr = m.row_ptr;
  p.col = m.col;
  p.val = m.val;
  MLG_CHECK(!a.half_values || m.val_h || m.nnz == 0, "FP16 values requested but not built");
  p.val_h = a.half_values ? m.val_h : nullptr;
  p.l_size = m.l_size;
  p.nCh = a.nCh;
  p.rows_per_block = rows_per_block(a);
  p.long_rows = m.long_rows;
  p.n_long = m.n_long;
  p.in = a.in;
  p.out = a.out;
  p.in_row_scale = a.in_row_scale;
  p.out_scale = a.out_scale;
  p.normalize = a.normalize ? 1 : 0;
  p.sqn_w = a.sqn_row_weight;
  p.partial = a.partial;
  p.absmax = a.absmax;
  p.in_h_amax = a.in_half_amax;
  p.in_h_len = a.in_half_len;
  MLG_CHECK(!a.in_half_amax || (use_pair_kernel(a) && a.contract && m.n_long == 0 && !a.nonempty_only),
            "FP16 input: contracted coil-pair products without long rows only");
  MLG_CHECK(!a.nonempty_only || (m.ord_rows && m.ord_nonempty && use_pair_kernel(a)),
            "non-empty-row products need the ordered row list and the coil-pair kernel");
  const long long nrows = spmm_rows(a);
  const int grid_all = (int)((nrows + p.rows_per_block - 1) / p.rows_per_block);
  const int grid_short = a.long_only ? 0 : grid_all;
  p.partial_long_offset = grid_all;
  MLG_CHECK(m.n_long == 0 || m.n_seg > 0, "long rows without segment tables");
  DevBuf<float> own;
  float* scratch = a.seg_scratch;
  if (m.n_long > 0 && !scratch) {
    MLG_TRY(own.alloc(spmm_scratch_floats(m, a.nCh), s));
    scratch = own.p;
  }
  float3* sc3 = reinterpret_cast<float3*>(scratch);
  using L = Layout;
  const L i = a.in.layout, o = a.out.layout;
  if (use_pair_kernel(a)) {
    if (grid_short > 0) {
      // the matrix's processing order when it covers the requested rows
      const bool ordered = m.ord_rows && m.ord_nonempty == a.nonempty_only;
      MLG_CHECK(ordered || !a.nonempty_only, "non-empty-row products need the ordered row list");
      // operator products over a split order: the short rows by the pair
      // kernel, the longer ones by a warp each
      const bool split = ordered && a.contract && m.ord_short >= 0 && !a.partial && a.nCh / 2 <= 16;
      const int n_pair = split ? m.ord_short : (int)nrows;
      MidRows mid;
      if (split && nrows > n_pair) {  // about two mid rows per warp
        mid.rows = m.ord_rows + n_pair;
        mid.bounds = m.ord_bounds + n_pair;
        mid.n = (int)nrows - n_pair;
        mid.blocks = (mid.n + 15) / 16;
      }
      const int grid_pair = split ? (n_pair + p.rows_per_block - 1) / p.rows_per_block : grid_short;
      const bool recs = records_forced() >= 0 ? records_forced() == 1 : a.records;
      if (split && m.ord_rec && recs && grid_pair + mid.blocks > 0) {
        const uint4* rec = reinterpret_cast<const uint4*>(m.ord_rec);
        const int g = grid_pair + mid.blocks;
        if (p.val_h)
          p.absmax ? spmm_rec_kernel<true, true><<<g, 256, 0, s>>>(p, rec, n_pair, mid)
                   : spmm_rec_kernel<true, false><<<g, 256, 0, s>>>(p, rec, n_pair, mid);
        else
          p.absmax ? spmm_rec_kernel<false, true><<<g, 256, 0, s>>>(p, rec, n_pair, mid)
                   : spmm_rec_kernel<false, false><<<g, 256, 0, s>>>(p, rec, n_pair, mid);
        MLG_LAUNCHED();
      } else if (grid_pair + mid.blocks > 0) {
        launch_pair(pair_ppt(a), a.contract, p, ordered ? m.ord_rows : nullptr,
                    ordered ? m.ord_bounds : nullptr, n_pair, grid_pair, mid, s);
        MLG_LAUNCHED();
      }
    }
    // long rows (segment kernels) with the same element types
    return launch<L::kPointC64, L::kPointC64, false>(p, m, sc3, 0, s);
  }
  if (i == L::kCoilC64 && o == L::kPointC64) return launch<L::kCoilC64, L::kPointC64, false>(p, m, sc3, grid_short, s);
  if (i == L::kPointC64 && o == L::kCoilC64) return launch<L::kPointC64, L::kCoilC64, true>(p, m, sc3, grid_short, s);
  if (i == L::kPointC64 && o == L::kPointC64)
    return launch<L::kPointC64, L::kPointC64, false>(p, m, sc3, grid_short, s);
  if (i == L::kCoilSplit && o == L::kCoilSplit)
    return launch<L::kCoilSplit, L::kCoilSplit, true>(p, m, sc3, grid_short, s);
  if (i == L::kPointSplit && o == L::kPointSplit)
    return launch<L::kPointSplit, L::kPointSplit, false>(p, m, sc3, grid_short, s);
  if (i == L::kCoilReal && o == L::kCoilReal) return launch<L::kCoilReal, L::kCoilReal, true>(p, m, sc3, grid_short, s);
  if (i == L::kPointReal && o == L::kPointReal)
    return launch<L::kPointReal, L::kPointReal, false>(p, m, sc3, grid_short, s);
  return fail(MLG_ERR_UNSUPPORTED, "spmm: layout pair (%d,%d) not instantiated", (int)i, (int)o);
}

// ---- sign-folded copies (fftshift as a (-1)^(x+y+z) modulation) ------------
__device__ __forceinline__ float cell_sign(long long i, int imDim, int Nx, int Ny) {
  long long x = i % Nx;
  long long s = x;
  if (imDim > 1) {
    const long long q = i / Nx;
    s += q % Ny;
    if (imDim > 2) s += q / Ny;
  }
  return (s & 1) ? -1.0f : 1.0f;
}

__global__ void sign_by_col_kernel(const int* __restrict__ col, const float* __restrict__ val, float* out,
                                   long long nnz, int imDim, int Nx, int Ny, float gs) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nnz; k += (long long)gridDim.x * blockDim.x)
    out[k] = val[k] * (gs * cell_sign(col[k], imDim, Nx, Ny));
}

__global__ void sign_by_row_kernel(const uint32_t* __restrict__ row_ptr, const float* __restrict__ val, float* out,
                                   int l_size, int imDim, int Nx, int Ny, float gs) {
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < l_size; r += (long long)gridDim.x * blockDim.x) {
    const float sg = gs * cell_sign(r, imDim, Nx, Ny);
    for (uint32_t k = row_ptr[r]; k < row_ptr[r + 1]; ++k) out[k] = val[k] * sg;
  }
}

void csr_free_sign_copy(Csr& c) {
  cudaFree(c.val);
  cudaFree(c.val_h);
  cudaFree(c.ord_rec);
  c = Csr();
}

__global__ void to_half_kernel(const float* __restrict__ v, long long n, __half* __restrict__ h) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    h[i] = __float2half_rn(v[i]);
}

int csr_make_half(Csr& c, cudaStream_t s) {
  if (c.val_h || c.nnz == 0) return MLG_OK;
  MLG_CUDA(cudaMalloc(&c.val_h, sizeof(__half) * (size_t)c.nnz));
  to_half_kernel<<<(int)std::max<long long>(1, std::min<long long>(148LL * 16, (c.nnz + 255) / 256)), 256, 0, s>>>(
      c.val, c.nnz, c.val_h);
  MLG_LAUNCHED();
  return MLG_OK;
}

int csr_sign_copy(const Csr& src, bool by_row, int imDim, const int* N, float global_sign, Csr& dst,
                  cudaStream_t s) {
  dst = src;  // shares row_ptr / col / long_rows with src (not owned)
  dst.val = nullptr;
  dst.val_h = nullptr;
  dst.ord_rec = nullptr;
  MLG_CUDA(cudaMalloc(&dst.val, sizeof(float) * (size_t)std::max<long long>(1, src.nnz)));
  const int Nx = N[0], Ny = imDim > 1 ? N[1] : 1;
  if (by_row) {
    sign_by_row_kernel<<<std::max(1, std::min(65535, (src.l_size + 255) / 256)), 256, 0, s>>>(
        src.row_ptr, src.val, dst.val, src.l_size, imDim, Nx, Ny, global_sign);
  } else {
    sign_by_col_kernel<<<(int)std::max<long long>(1, std::min<long long>(65535, (src.nnz + 255) / 256)), 256, 0, s>>>(
        src.col, src.val, dst.val, src.nnz, imDim, Nx, Ny, global_sign);
  }
  MLG_LAUNCHED();
  return MLG_OK;
}

// ---- host-buffer SpMV entry points ------------------------------------------
namespace {

struct HostCall {
  cudaStream_t s = nullptr;
  Csr m;
  ~HostCall() { csr_free(m); }
};

int vec_call(int r_size, const int* r_jump, const int* r_nJump, const float* m_val, int l_size,
             const int* l_jump, int l_nJump, const float* vR, const float* vI, int nVec, float* wR,
             float* wI, Layout layout, int nBlock = 0, const int* block_length = nullptr,
             const int* l_block_start = nullptr, const long long* m_block_start = nullptr) {
  MLG_TRY(ensure_device());
  MLG_CHECK(nVec >= 1, "n_vec must be >= 1");
  const bool cplx = layout != Layout::kCoilReal && layout != Layout::kPointReal;
  MLG_CHECK(vR && wR && (!cplx || (vI && wI)), "NULL vector buffer");
  HostCall hc;
  MLG_TRY(csr_from_jump(r_size, r_jump, r_nJump, m_val, l_size, l_jump, l_nJump, hc.m, hc.s, nBlock, block_length,
                        l_block_start, m_block_start));
  const size_t nin = (size_t)r_size * nVec, nout = (size_t)l_size * nVec;
  DevBuf<float> din, dout;
  MLG_TRY(din.alloc(nin * (cplx ? 2 : 1), hc.s));
  MLG_TRY(dout.alloc(nout * (cplx ? 2 : 1), hc.s));
  MLG_CUDA(cudaMemcpyAsync(din.p, vR, nin * sizeof(float), cudaMemcpyHostToDevice, hc.s));
  if (cplx) MLG_CUDA(cudaMemcpyAsync(din.p + nin, vI, nin * sizeof(float), cudaMemcpyHostToDevice, hc.s));
  SpmmArgs a;
  a.m = &hc.m;
  a.nCh = nVec;
  a.in.layout = a.out.layout = layout;
  a.in.a = din.p;
  a.in.b = cplx ? din.p + nin : nullptr;
  a.in.rows = r_size;
  a.out.a = dout.p;
  a.out.b = cplx ? dout.p + nout : nullptr;
  a.out.rows = l_size;
  MLG_TRY(spmm(a, hc.s));
  MLG_CUDA(cudaMemcpyAsync(wR, dout.p, nout * sizeof(float), cudaMemcpyDeviceToHost, hc.s));
  if (cplx) MLG_CUDA(cudaMemcpyAsync(wI, dout.p + nout, nout * sizeof(float), cudaMemcpyDeviceToHost, hc.s));
  MLG_CUDA(cudaStreamSynchronize(hc.s));
  return MLG_OK;
}

}  // namespace
}  // namespace mlg

using namespace mlg;

extern "C" {

int mlg_sparsemat_vec_cC(int r_size, const int* r_jump, const int* r_nJump, const float* m_val, int l_size,
                         const int* l_jump, int l_nJump, const float* vReal, const float* vImag, int nVec,
                         float* wReal, float* wImag) {
  return vec_call(r_size, r_jump, r_nJump, m_val, l_size, l_jump, l_nJump, vReal, vImag, nVec, wReal, wImag,
                  Layout::kCoilSplit);
}

int mlg_sparsemat_vec_cR(int r_size, const int* r_jump, const int* r_nJump, const float* m_val, int l_size,
                         const int* l_jump, int l_nJump, const float* vReal, const float* vImag, int nVec,
                         float* wReal, float* wImag) {
  return vec_call(r_size, r_jump, r_nJump, m_val, l_size, l_jump, l_nJump, vReal, vImag, nVec, wReal, wImag,
                  Layout::kPointSplit);
}

int mlg_sparsemat_vec_rC(int r_size, const int* r_jump, const int* r_nJump, const float* m_val, int l_size,
                         const int* l_jump, int l_nJump, const float* v, int nVec, float* w) {
  return vec_call(r_size, r_jump, r_nJump, m_val, l_size, l_jump, l_nJump, v, nullptr, nVec, w, nullptr,
                  Layout::kCoilReal);
}

int mlg_sparsemat_r_nJump2index(int l_size, const int* r_nJump, long long out_length, int* out) {
  // bmSparseMat_r_nJump2index_mex.cpp:70-80.  A setup-time helper of the
  // matrix builder: runs on the host (there is no device work to amortise).
  MLG_CHECK(l_size >= 0 && (l_size == 0 || r_nJump), "r_nJump missing");
  MLG_CHECK(out || out_length == 0, "NULL output");
  long long n = 0;
  for (int i = 0; i < l_size; ++i) {
    MLG_CHECK(r_nJump[i] >= 0, "negative r_nJump");
    MLG_CHECK(n + r_nJump[i] <= out_length, "out_length %lld smaller than sum(r_nJump)", out_length);
    for (int j = 0; j < r_nJump[i]; ++j) out[n++] = i;
  }
  MLG_CHECK(n == out_length, "out_length %lld differs from sum(r_nJump)=%lld", out_length, n);
  return MLG_OK;
}

int mlg_matrix_create_blocks(int r_size, const int* r_jump, const int* r_nJump, const float* m_val, int l_size,
                             const int* l_jump, int l_nJump, int nBlock, const int* block_length,
                             const int* l_block_start, const long long* m_block_start, mlg_matrix_t* out) {
  MLG_CHECK(out, "NULL output handle");
  *out = nullptr;
  MLG_CHECK(nBlock >= 0, "nBlock must be >= 0");
  MLG_TRY(ensure_device());
  mlg_matrix_s* h = new mlg_matrix_s();
  cudaGetDevice(&h->device);
  int st = csr_from_jump(r_size, r_jump, r_nJump, m_val, l_size, l_jump, l_nJump, h->csr, nullptr, nBlock,
                         block_length, l_block_start, m_block_start);
  if (st != MLG_OK) {
    delete h;
    return st;
  }
  *out = h;
  return MLG_OK;
}

int mlg_matrix_create(int r_size, const int* r_jump, const int* r_nJump, const float* m_val, int l_size,
                      const int* l_jump, int l_nJump, mlg_matrix_t* out) {
  return mlg_matrix_create_blocks(r_size, r_jump, r_nJump, m_val, l_size, l_jump, l_nJump, 0, nullptr, nullptr,
                                  nullptr, out);
}

int mlg_sparsemat_vec(int layout, int r_size, const int* r_jump, const int* r_nJump, const float* m_val, int l_size,
                      const int* l_jump, int l_nJump, int nBlock, const int* block_length, const int* l_block_start,
                      const long long* m_block_start, const float* vR, const float* vI, int nVec, float* wR,
                      float* wI) {
  Layout L;
  switch (layout) {
    case MLG_LAYOUT_CC: L = Layout::kCoilSplit; break;
    case MLG_LAYOUT_CR: L = Layout::kPointSplit; break;
    case MLG_LAYOUT_RC: L = Layout::kCoilReal; break;
    case MLG_LAYOUT_RR: L = Layout::kPointReal; break;
    default: return fail(MLG_ERR_ARG, "unknown layout %d", layout);
  }
  MLG_CHECK(nBlock >= 0, "nBlock must be >= 0");
  return vec_call(r_size, r_jump, r_nJump, m_val, l_size, l_jump, l_nJump, vR, vI, nVec, wR, wI, L, nBlock,
                  block_length, l_block_start, m_block_start);
}

int mlg_sparsemat_vec_rR(int r_size, const int* r_jump, const int* r_nJump, const float* m_val, int l_size,
                         const int* l_jump, int l_nJump, const float* v, int nVec, float* w) {
  return vec_call(r_size, r_jump, r_nJump, m_val, l_size, l_jump, l_nJump, v, nullptr, nVec, w, nullptr,
                  Layout::kPointReal);
}

int mlg_matrix_destroy(mlg_matrix_t m) {
  if (!m) return MLG_OK;
  cudaSetDevice(m->device);
  csr_free(m->csr);
  delete m;
  return MLG_OK;
}

int mlg_matrix_info(mlg_matrix_t m, long long* nnz, int* r_size, int* l_size) {
  MLG_CHECK(m, "NULL matrix");
  if (nnz) *nnz = m->csr.nnz;
  if (r_size) *r_size = m->csr.r_size;
  if (l_size) *l_size = m->csr.l_size;
  return MLG_OK;
}

int mlg_matrix_row_stats(mlg_matrix_t m, int* nonempty_rows, int* long_rows) {
  MLG_CHECK(m, "NULL matrix");
  if (nonempty_rows) *nonempty_rows = m->csr.n_nonempty;
  if (long_rows) *long_rows = m->csr.n_long;
  return MLG_OK;
}

int mlg_matrix_download(mlg_matrix_t m, int* r_jump, int* r_nJump, float* m_val, int* l_jump, int* l_nJump_out) {
  MLG_CHECK(m && r_jump && r_nJump && m_val, "NULL argument");
  const Csr& c = m->csr;
  MLG_CUDA(cudaSetDevice(m->device));
  std::vector<uint32_t> rp((size_t)c.l_size + 1);
  std::vector<int> col((size_t)c.nnz);
  MLG_CUDA(cudaMemcpy(rp.data(), c.row_ptr, sizeof(uint32_t) * rp.size(), cudaMemcpyDeviceToHost));
  if (c.nnz) {
    MLG_CUDA(cudaMemcpy(col.data(), c.col, sizeof(int) * (size_t)c.nnz, cudaMemcpyDeviceToHost));
    MLG_CUDA(cudaMemcpy(m_val, c.val, sizeof(float) * (size_t)c.nnz, cudaMemcpyDeviceToHost));
  }
  long long prevc = 0;
  for (long long e = 0; e < c.nnz; ++e) {
    r_jump[e] = (int)(col[(size_t)e] - prevc);
    prevc = col[(size_t)e];
  }
  // l_jump != NULL: squeezed form (non-empty rows only, bmSparseMat.m:62-94)
  int n = 0;
  long long prevr = 0;
  for (int r = 0; r < c.l_size; ++r) {
    const int len = (int)(rp[(size_t)r + 1] - rp[r]);
    if (l_jump) {
      if (len == 0) continue;
      l_jump[n] = (int)(r - prevr);
      prevr = r;
    }
    r_nJump[n++] = len;
  }
  if (l_nJump_out) *l_nJump_out = n;
  return MLG_OK;
}

int mlg_matrix_spmm_dev(mlg_matrix_t m, const void* v, int nVec, void* w, void* stream) {
  MLG_CHECK(m && v && w && nVec >= 1, "invalid argument");
  MLG_CUDA(cudaSetDevice(m->device));
  SpmmArgs a;
  a.m = &m->csr;
  a.nCh = nVec;
  a.in.layout = a.out.layout = Layout::kPointC64;
  a.in.a = const_cast<void*>(v);
  a.in.rows = m->csr.r_size;
  a.out.a = w;
  a.out.rows = m->csr.l_size;
  return spmm(a, (cudaStream_t)stream);
}

}  // extern "C"
