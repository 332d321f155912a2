// Pruned, fused line-FFT passes (see mlg_fft.cuh): the pass kernel template
// and its launch helpers.  The instantiations are spread over the
// mlg_fft_pass_*.cu translation units (one per pass mode and direction) so
// that they compile in parallel; mlg_fft.cu holds the host side.
//
// One CTA transforms `cols` = L lines x C coils of length N = N1 * N2 held
// in shared memory as s[n][col] (col fastest), with the four-step
// decomposition:
//   A. for every n2 < N2 and column: an N1-point FFT over n1 (elements
//      n1*N2 + n2), each output k1 multiplied by W_N^(n2*k1);
//   C. for every k1 < N1 and column: an N2-point FFT over n2 (elements
//      k1*N2 + n2) -> X[k1 + N1*k2] stored at position k1*N2 + k2.
// Sub-FFTs of size 2^a 3^b run as unrolled radix-2/radix-3 butterflies in
// registers (templated fast path); other sizes <= 32 use a direct DFT
// (runtime path).  Twiddles come from a per-axis table exp(-2 pi i j/N)
// computed on the host in double precision.
#pragma once

#include <algorithm>
#include <cmath>
#include <utility>
#include <vector>

#include "mlg_fft.cuh"

namespace mlg {

constexpr int kFftThreads = 256;     // target threads per CTA
constexpr int kFftMaxThreads = 512;  // launch bound (columns that need lcm(cols, 32) > 256)
constexpr size_t kFftSmemCap = 100 * 1024;

// Threads per CTA: a multiple of the CTA's columns (and of the warp) so that
// every thread keeps one column (or coil pair) through the load, the
// transform and the store; the multiple nearest kFftThreads.  Columns whose
// lcm with 32 exceeds kFftMaxThreads take kFftThreads and the per-element
// paths.
constexpr int cta_threads(int cols) {
  int g = cols, b = 32;
  while (b) {
    const int t = g % b;
    g = b;
    b = t;
  }
  const int l = cols / g * 32;  // lcm(cols, 32)
  if (l > kFftMaxThreads) return kFftThreads;
  const int k = (kFftThreads + l / 2) / l > 1 ? (kFftThreads + l / 2) / l : 1;
  return kFftMaxThreads / l * l < k * l ? kFftMaxThreads / l * l : k * l;
}
static_assert(cta_threads(16) == 256 && cta_threads(32) == 256 && cta_threads(24) == 288, "CTA sizes");
constexpr int kGatherBatch = 8;  // cells gathered concurrently per thread (kGutIn)

__device__ __forceinline__ float2 cmulf(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// The same product with every rounding explicit (no contraction into fused
// multiply-adds, which the compiler may choose differently at each call
// site): the forward x passes' x .* KFC, so that their TMA, pipelined and
// unpipelined kernels agree bit for bit.
__device__ __forceinline__ float2 cmulf_rn(float2 a, float2 b) {
  return make_float2(__fsub_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)),
                     __fadd_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x)));
}

// One coil pair's share of the inverse x pass's coil sum: the two coils'
// values times the modulation-and-scale factor sg, times their KFC_conj
// values, added (explicit roundings; the pipelined and unpipelined kernels
// share it, so they give the same image bit for bit).
__device__ __forceinline__ float2 nak_pair_term(float4 sv, float4 kv, float sg) {
  const float2 t0 = cmulf_rn(make_float2(__fmul_rn(sv.x, sg), __fmul_rn(sv.y, sg)), make_float2(kv.x, kv.y));
  const float2 t1 = cmulf_rn(make_float2(__fmul_rn(sv.z, sg), __fmul_rn(sv.w, sg)), make_float2(kv.z, kv.w));
  return make_float2(__fadd_rn(t0.x, t1.x), __fadd_rn(t0.y, t1.y));
}

// Largest component magnitude of two complex values.
__device__ __forceinline__ float absmax4(float4 v) {
  return fmaxf(fmaxf(fabsf(v.x), fabsf(v.y)), fmaxf(fabsf(v.z), fabsf(v.w)));
}

// Raises *amax to the warp's largest v (every lane calls; v >= 0).
__device__ __forceinline__ void warp_amax(unsigned* amax, float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) atomicMax(amax, __float_as_uint(v));
}

template <int DIR>
__device__ __forceinline__ float2 twid(const float2* __restrict__ tw, int j) {
  const float2 w = __ldg(tw + j);
  return DIR < 0 ? w : make_float2(w.x, -w.y);
}

// ---- in-register radix-2 FFT with compile-time twiddles ----------------------
// The sub-FFT twiddles W_R^j depend only on template parameters: they are
// evaluated at compile time (constexpr series for sin/cos in double, rounded
// to float) and become instruction immediates -- no twiddle loads.
constexpr double kPiD = 3.14159265358979323846264338327950288;

constexpr double cx_sin_red(double x) {  // |x| <= pi
  double term = x, sum = x;
  for (int k = 1; k < 16; ++k) {
    term *= -x * x / ((2.0 * k) * (2.0 * k + 1.0));
    sum += term;
  }
  return sum;
}
constexpr double cx_cos_red(double x) {  // |x| <= pi
  double term = 1.0, sum = 1.0;
  for (int k = 1; k < 16; ++k) {
    term *= -x * x / ((2.0 * k - 1.0) * (2.0 * k));
    sum += term;
  }
  return sum;
}
constexpr double cx_reduce(double x) {  // to [-pi, pi]
  while (x > kPiD) x -= 2 * kPiD;
  while (x < -kPiD) x += 2 * kPiD;
  return x;
}

template <class F, int... Is>
__device__ __forceinline__ void sfor_impl(F&& f, std::integer_sequence<int, Is...>) {
  (f(std::integral_constant<int, Is>{}), ...);
}
template <int N, class F>
__device__ __forceinline__ void sfor(F&& f) {
  sfor_impl(f, std::make_integer_sequence<int, N>{});
}

constexpr int bitrev(int i, int R) {
  int j = 0;
  for (int b = 1; b < R; b <<= 1, i >>= 1) j = (j << 1) | (i & 1);
  return j;
}

template <int R, int DIR, int LEN>
__device__ __forceinline__ void rstage(float2 (&r)[R]) {
  sfor<R / LEN>([&](auto ic) {
    constexpr int I = decltype(ic)::value * LEN;
    sfor<LEN / 2>([&](auto jc) {
      constexpr int J = decltype(jc)::value;
      constexpr double ang = cx_reduce((double)DIR * 2.0 * kPiD * (double)J / (double)LEN);
      constexpr float wr = (float)cx_cos_red(ang), wi = (float)cx_sin_red(ang);
      const float2 u = r[I + J], v = r[I + J + LEN / 2];
      float2 t;
      if constexpr (J == 0) {
        t = v;
      } else if constexpr (4 * J == LEN) {  // +-i: a swap and a sign
        t = DIR < 0 ? make_float2(v.y, -v.x) : make_float2(-v.y, v.x);
      } else {
        t = make_float2(wr * v.x - wi * v.y, wr * v.y + wi * v.x);
      }
      r[I + J] = make_float2(u.x + t.x, u.y + t.y);
      r[I + J + LEN / 2] = make_float2(u.x - t.x, u.y - t.y);
    });
  });
}

template <int R, int DIR, int LEN = 2>
__device__ __forceinline__ void rstages(float2 (&r)[R]) {
  if constexpr (LEN <= R) {
    rstage<R, DIR, LEN>(r);
    rstages<R, DIR, LEN * 2>(r);
  }
}

constexpr bool cx_pow2(int v) { return v > 0 && (v & (v - 1)) == 0; }

template <int R, int DIR>
__device__ __forceinline__ void reg_fft(float2 (&r)[R]);

// R = 3M (M = 2^a 3^b): decimation in time by 3.  The three M-point
// transforms of r[3m], r[3m+1], r[3m+2] are combined by radix-3 butterflies
// with compile-time twiddles W_R^k, W_R^2k:
//   X[k] = a + b + c,  X[k+M], X[k+2M] = a - (b+c)/2 -+ DIR i (sqrt3/2)(b-c)
// where b, c carry their twiddles (DIR = -1 forward, +1 inverse).
template <int R, int DIR>
__device__ __forceinline__ void reg_fft_radix3(float2 (&r)[R]) {
  constexpr int M = R / 3;
  float2 a[M], b[M], c[M];
  sfor<M>([&](auto mc) {
    constexpr int m = decltype(mc)::value;
    a[m] = r[3 * m];
    b[m] = r[3 * m + 1];
    c[m] = r[3 * m + 2];
  });
  reg_fft<M, DIR>(a);
  reg_fft<M, DIR>(b);
  reg_fft<M, DIR>(c);
  constexpr float h = (float)(0.86602540378443864676 * (double)DIR);  // DIR * sqrt(3)/2
  sfor<M>([&](auto kc) {
    constexpr int k = decltype(kc)::value;
    constexpr double a1 = cx_reduce((double)DIR * 2.0 * kPiD * (double)k / (double)R);
    constexpr double a2 = cx_reduce((double)DIR * 2.0 * kPiD * (double)(2 * k) / (double)R);
    constexpr float w1r = (float)cx_cos_red(a1), w1i = (float)cx_sin_red(a1);
    constexpr float w2r = (float)cx_cos_red(a2), w2i = (float)cx_sin_red(a2);
    float2 bv = b[k], cv = c[k];
    if constexpr (k != 0) {
      bv = make_float2(w1r * b[k].x - w1i * b[k].y, w1r * b[k].y + w1i * b[k].x);
      cv = make_float2(w2r * c[k].x - w2i * c[k].y, w2r * c[k].y + w2i * c[k].x);
    }
    const float2 s = make_float2(bv.x + cv.x, bv.y + cv.y);
    const float2 d = make_float2(bv.x - cv.x, bv.y - cv.y);
    const float2 m = make_float2(a[k].x - 0.5f * s.x, a[k].y - 0.5f * s.y);
    r[k] = make_float2(a[k].x + s.x, a[k].y + s.y);
    r[k + M] = make_float2(m.x - h * d.y, m.y + h * d.x);      // m + h i d
    r[k + 2 * M] = make_float2(m.x + h * d.y, m.y - h * d.x);  // m - h i d
  });
}

// DIR < 0: X[k] = sum_j r[j] exp(-2 pi i jk/R) (forward); DIR > 0: inverse.
// R = 2^a 3^b.
template <int R, int DIR>
__device__ __forceinline__ void reg_fft(float2 (&r)[R]) {
  if constexpr (R > 1 && !cx_pow2(R)) {
    static_assert(R % 3 == 0, "register FFT length must be 2^a 3^b");
    reg_fft_radix3<R, DIR>(r);
  } else if constexpr (R > 1) {
    sfor<R>([&](auto ic) {  // bit-reversal permutation
      constexpr int i = decltype(ic)::value;
      constexpr int j = bitrev(i, R);
      if constexpr (j > i) {
        const float2 t = r[i];
        r[i] = r[j];
        r[j] = t;
      }
    });
    rstages<R, DIR>(r);
  }
}

// Direct DFT of runtime size R <= 32 (slow path).
template <int DIR>
__device__ __forceinline__ void dft_any(float2* r, int R, const float2* __restrict__ tw, int tstride) {
  float2 o[32];
  for (int k = 0; k < R; ++k) {
    float2 acc = make_float2(0.f, 0.f);
    for (int j = 0; j < R; ++j) {
      const float2 w = twid<DIR>(tw, ((j * k) % R) * tstride);
      const float2 t = cmulf(w, r[j]);
      acc.x += t.x;
      acc.y += t.y;
    }
    o[k] = acc;
  }
  for (int k = 0; k < R; ++k) r[k] = o[k];
}

struct Lines {
  int u, v;       // non-FFT axes, u groups adjacent lines
  int u0, vi;     // first u index of this CTA, v index
  int L;          // lines per CTA
};

__device__ __forceinline__ Lines lines_of(const PassDesc& d, int L) {
  Lines ln;
  ln.u = d.ax == 0 ? 1 : 0;
  ln.v = d.ax == 2 ? 1 : 2;
  const int gu = (d.dims[ln.u] + L - 1) / L;
  ln.u0 = (int)(blockIdx.x % gu) * L;
  ln.vi = (int)(blockIdx.x / gu);
  ln.L = L;
  return ln;
}

template <PassMode MODE>
__device__ __forceinline__ float2 load_elem(const PassDesc& d, const Lines& ln, int n, int l, int c) {
  const int ui = ln.u0 + l;
  if (ui >= d.dims[ln.u] || n < d.in_lo || n >= d.in_lo + d.in_len) return make_float2(0.f, 0.f);
  if constexpr (MODE == PassMode::kShannaIn) {
    // axis x: pixel (n - in_lo, ui, vi) of the n_x * n_y * n_z image
    const long long m = (n - d.in_lo) + (long long)d.in_len * (ui + (long long)d.dims[1] * ln.vi);
    const float2 xv = __ldg(d.img + (d.img_per_coil ? m * d.C + c : m));
    float2 v = cmulf_rn(xv, __ldg(d.kfc + m * d.C + c));
    if ((n + d.coord_off[1] + ui + d.coord_off[2] + ln.vi) & 1) v = make_float2(-v.x, -v.y);
    return v;
  } else {
    if (d.in_mask) {
      const long long cell = (long long)ui * d.cell_stride[ln.u] + (long long)ln.vi * d.cell_stride[ln.v] +
                             (long long)n * d.cell_stride[d.ax];
      if (!((__ldg(d.in_mask + (cell >> 5)) >> (cell & 31)) & 1u)) return make_float2(0.f, 0.f);
    }
    const long long off = (long long)(n - d.in_lo) * d.in_stride[d.ax] + (long long)ui * d.in_stride[ln.u] +
                          (long long)ln.vi * d.in_stride[ln.v] + c;
    return __ldg(d.in + off);
  }
}

template <int DIR>
__device__ __forceinline__ void step_twiddle(float2* r, int R, int n2, const float2* tw) {
  for (int k1 = 1; k1 < R; ++k1) {
    if (n2 == 0) break;
    r[k1] = cmulf(r[k1], twid<DIR>(tw, n2 * k1));
  }
}

// The in-shared-memory transform; N1/N2 > 0 select the unrolled path.
template <int N1, int N2, int DIR>
__device__ __forceinline__ void smem_fft(float2* s, int cols, int rN1, int rN2, const float2* __restrict__ tw) {
  const int n1s = N1 > 0 ? N1 : rN1, n2s = N2 > 0 ? N2 : rN2;
  const int N = n1s * n2s;
  if constexpr (N1 > 0) {
    if ((int)blockDim.x % cols == 0) {
      // fixed column per thread, rows strided by the number of row groups
      const int col = threadIdx.x % cols, g = threadIdx.x / cols, G = blockDim.x / cols;
      for (int n2 = g; n2 < N2; n2 += G) {
        float2 r[N1];
#pragma unroll
        for (int n1 = 0; n1 < N1; ++n1) r[n1] = s[(n1 * N2 + n2) * cols + col];
        reg_fft<N1, DIR>(r);
        if (n2) {
#pragma unroll
          for (int k1 = 1; k1 < N1; ++k1) r[k1] = cmulf(r[k1], twid<DIR>(tw, n2 * k1));
        }
#pragma unroll
        for (int k1 = 0; k1 < N1; ++k1) s[(k1 * N2 + n2) * cols + col] = r[k1];
      }
      __syncthreads();
      for (int k1 = g; k1 < N1; k1 += G) {
        float2 r[N2];
#pragma unroll
        for (int n2 = 0; n2 < N2; ++n2) r[n2] = s[(k1 * N2 + n2) * cols + col];
        reg_fft<N2, DIR>(r);
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) s[(k1 * N2 + k2) * cols + col] = r[k2];
      }
      __syncthreads();
      return;
    }
  }
  // step A
  for (int it = threadIdx.x; it < n2s * cols; it += blockDim.x) {
    const int n2 = it / cols, col = it - (it / cols) * cols;
    if constexpr (N1 > 0) {
      float2 r[N1];
#pragma unroll
      for (int n1 = 0; n1 < N1; ++n1) r[n1] = s[(n1 * N2 + n2) * cols + col];
      reg_fft<N1, DIR>(r);
#pragma unroll
      for (int k1 = 1; k1 < N1; ++k1)
        if (n2) r[k1] = cmulf(r[k1], twid<DIR>(tw, n2 * k1));
#pragma unroll
      for (int k1 = 0; k1 < N1; ++k1) s[(k1 * N2 + n2) * cols + col] = r[k1];
    } else {
      float2 r[32];
      for (int n1 = 0; n1 < n1s; ++n1) r[n1] = s[(n1 * n2s + n2) * cols + col];
      dft_any<DIR>(r, n1s, tw, N / n1s);
      step_twiddle<DIR>(r, n1s, n2, tw);
      for (int k1 = 0; k1 < n1s; ++k1) s[(k1 * n2s + n2) * cols + col] = r[k1];
    }
  }
  __syncthreads();
  // step C
  for (int it = threadIdx.x; it < n1s * cols; it += blockDim.x) {
    const int k1 = it / cols, col = it - (it / cols) * cols;
    if constexpr (N2 > 0) {
      float2 r[N2];
#pragma unroll
      for (int n2 = 0; n2 < N2; ++n2) r[n2] = s[(k1 * N2 + n2) * cols + col];
      reg_fft<N2, DIR>(r);
#pragma unroll
      for (int k2 = 0; k2 < N2; ++k2) s[(k1 * N2 + k2) * cols + col] = r[k2];
    } else {
      float2 r[32];
      for (int n2 = 0; n2 < n2s; ++n2) r[n2] = s[(k1 * n2s + n2) * cols + col];
      dft_any<DIR>(r, n2s, tw, N / n2s);
      for (int k2 = 0; k2 < n2s; ++k2) s[(k1 * n2s + k2) * cols + col] = r[k2];
    }
  }
  __syncthreads();
}

// kGutIn load: each thread owns V adjacent coils (V = 2: 16-byte loads) of
// one line and walks the line's cells with a stride; four cells are
// gathered at a time so four dependency chains (row pointer -> entry ->
// k-space row) are in flight per thread.  Per cell the entries are summed in
// stored order with round-to-nearest multiply/add, as the SpMM kernels do.
template <int V>
__device__ __forceinline__ void gut_load(const PassDesc& d, const Lines& ln, float2* s, int N, int cols) {
  using VT = typename std::conditional<V == 2, float4, float2>::type;
  const int C = d.C;
  const int cv = cols / V;
  const int vc = threadIdx.x % cv, rstep = blockDim.x / cv;
  const int col0 = vc * V, l = col0 / C, c = col0 - l * C;
  const int ui = ln.u0 + l;
  const bool line_ok = ui < d.dims[ln.u];
  const long long cell_base = (long long)ui * d.cell_stride[ln.u] + (long long)ln.vi * d.cell_stride[ln.v];
  const long long cst = d.cell_stride[d.ax];
  VT* sv = reinterpret_cast<VT*>(s);
  constexpr int B = kGatherBatch;
  for (int n0 = threadIdx.x / cv; n0 < N; n0 += B * rstep) {
    uint32_t b[B], len[B];
    float acc[B][2 * V];
#pragma unroll
    for (int j = 0; j < B; ++j) {
      const int n = n0 + j * rstep;
      b[j] = len[j] = 0;
#pragma unroll
      for (int q = 0; q < 2 * V; ++q) acc[j][q] = 0.f;
      if (line_ok && n < N) {
        const long long cell = cell_base + (long long)n * cst;
        b[j] = __ldg(d.g_rowptr + cell);
        len[j] = __ldg(d.g_rowptr + cell + 1) - b[j];
        if (len[j] > (uint32_t)kLongRow) {  // precomputed by the long-row kernel
          const float* gl = reinterpret_cast<const float*>(d.g_long + cell * C + c);
#pragma unroll
          for (int q = 0; q < 2 * V; ++q) acc[j][q] = gl[q];
          len[j] = 0;
        }
      }
    }
    uint32_t maxlen = 0;
#pragma unroll
    for (int j = 0; j < B; ++j) maxlen = max(maxlen, len[j]);
    for (uint32_t t = 0; t < maxlen; ++t) {
#pragma unroll
      for (int j = 0; j < B; ++j) {
        if (t < len[j]) {
          const uint32_t k = b[j] + t;
          const int jc = __ldg(d.g_col + k);
          const float m = __ldg(d.g_val + k);
          const float h = d.g_hy ? __ldg(d.g_hy + jc) : 1.0f;
          const VT yv = *reinterpret_cast<const VT*>(d.g_y + (long long)jc * C + c);
          const float* yf = reinterpret_cast<const float*>(&yv);
#pragma unroll
          for (int q = 0; q < 2 * V; ++q) {
            const float hv = d.g_hy ? __fmul_rn(h, yf[q]) : yf[q];
            acc[j][q] = __fadd_rn(acc[j][q], __fmul_rn(m, hv));
          }
        }
      }
    }
#pragma unroll
    for (int j = 0; j < B; ++j) {
      const int n = n0 + j * rstep;
      if (n < N) {
        VT o;
        float* of = reinterpret_cast<float*>(&o);
#pragma unroll
        for (int q = 0; q < 2 * V; ++q) of[q] = acc[j][q];
        sv[n * cv + vc] = o;
      }
    }
  }
}

// MAXT: the launch bound, kFftThreads for the usual CTAs (the register
// budget that keeps three 256-thread CTAs per SM) or kFftMaxThreads for the
// wider CTAs some coil counts need.
template <int N1, int N2, int DIR, PassMode MODE, int MAXT>
__global__ void __launch_bounds__(MAXT) fft_pass_kernel(PassDesc d, int L, int rN1, int rN2,
                                                        const float2* __restrict__ tw) {
  extern __shared__ float2 s[];
  const int n1s = N1 > 0 ? N1 : rN1, n2s = N2 > 0 ? N2 : rN2;
  const int N = n1s * n2s;
  const int C = d.C;
  const int cols = L * C;
  const Lines ln = lines_of(d, L);
  // load (zero-filled outside the stored input range)
  const int cv = cols >> 1;  // coil pairs when C is even: 16-byte accesses
  if constexpr (MODE == PassMode::kGutIn) {
    if ((C & 1) == 0 && (int)blockDim.x % cv == 0) {
      gut_load<2>(d, ln, s, N, cols);
    } else if ((int)blockDim.x % cols == 0) {
      gut_load<1>(d, ln, s, N, cols);
    } else {
      for (int it = threadIdx.x; it < N * cols; it += blockDim.x) {
        const int n = it / cols, col = it - (it / cols) * cols;
        const int l = col / C, c = col - (col / C) * C;
        const int ui = ln.u0 + l;
        float2 a = make_float2(0.f, 0.f);
        if (ui < d.dims[ln.u]) {
          const long long cell = (long long)ui * d.cell_stride[ln.u] + (long long)ln.vi * d.cell_stride[ln.v] +
                                 (long long)n * d.cell_stride[d.ax];
          const uint32_t b = __ldg(d.g_rowptr + cell), e = __ldg(d.g_rowptr + cell + 1);
          if (e - b > (uint32_t)kLongRow) {
            a = d.g_long[cell * C + c];
          } else {
            for (uint32_t k = b; k < e; ++k) {
              const int jc = __ldg(d.g_col + k);
              const float m = __ldg(d.g_val + k);
              float2 v = __ldg(d.g_y + (long long)jc * C + c);
              if (d.g_hy) {
                const float h = __ldg(d.g_hy + jc);
                v = make_float2(__fmul_rn(h, v.x), __fmul_rn(h, v.y));
              }
              a = make_float2(__fadd_rn(a.x, __fmul_rn(m, v.x)), __fadd_rn(a.y, __fmul_rn(m, v.y)));
            }
          }
        }
        s[n * cols + col] = a;
      }
    }
  } else if ((C & 1) == 0 && (int)blockDim.x % cv == 0) {
    // fixed coil pair per thread, rows strided: no divisions in the loop and
    // several independent 16-byte loads in flight per thread
    const int vc = threadIdx.x % cv, rstep = blockDim.x / cv;
    const int col = vc * 2, l = col / C, c = col - l * C;
    const int ui = ln.u0 + l;
    const bool line_ok = ui < d.dims[ln.u];
    float4* s4 = reinterpret_cast<float4*>(s);
    if constexpr (MODE == PassMode::kShannaIn) {
      const long long mrow = (long long)d.in_len * (ui + (long long)d.dims[1] * ln.vi);
      const int par = (d.coord_off[1] + ui + d.coord_off[2] + ln.vi) & 1;
#pragma unroll 4
      for (int n = threadIdx.x / cv; n < N; n += rstep) {
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (line_ok && n >= d.in_lo && n < d.in_lo + d.in_len) {
          const long long m = mrow + (n - d.in_lo);
          const float4 k = __ldg(reinterpret_cast<const float4*>(d.kfc + m * C + c));
          float2 a, b;
          if (d.img_per_coil) {
            const float4 xv = __ldg(reinterpret_cast<const float4*>(d.img + m * C + c));
            a = make_float2(xv.x, xv.y);
            b = make_float2(xv.z, xv.w);
          } else {
            a = b = __ldg(d.img + m);
          }
          float2 r0 = cmulf(a, make_float2(k.x, k.y)), r1 = cmulf(b, make_float2(k.z, k.w));
          if ((n + par) & 1) {
            r0 = make_float2(-r0.x, -r0.y);
            r1 = make_float2(-r1.x, -r1.y);
          }
          v = make_float4(r0.x, r0.y, r1.x, r1.y);
        }
        s4[n * cv + vc] = v;
      }
    } else {
      const float2* base = d.in + (long long)ui * d.in_stride[ln.u] + (long long)ln.vi * d.in_stride[ln.v] + c;
      const long long st = d.in_stride[d.ax];
      const uint32_t* mask = d.in_mask;
      const long long cell0 = (long long)ui * d.cell_stride[ln.u] + (long long)ln.vi * d.cell_stride[ln.v];
      const long long cst = d.cell_stride[d.ax];
#pragma unroll 4
      for (int n = threadIdx.x / cv; n < N; n += rstep) {
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        bool ld = line_ok && n >= d.in_lo && n < d.in_lo + d.in_len;
        if (ld && mask) {
          const long long cell = cell0 + (long long)n * cst;
          ld = (__ldg(mask + (cell >> 5)) >> (cell & 31)) & 1u;
        }
        if (ld) v = __ldg(reinterpret_cast<const float4*>(base + (long long)(n - d.in_lo) * st));
        s4[n * cv + vc] = v;
      }
    }
  } else {
    for (int it = threadIdx.x; it < N * cols; it += blockDim.x) {
      const int n = it / cols, col = it - (it / cols) * cols;
      const int l = col / C, c = col - (col / C) * C;
      s[n * cols + col] = load_elem<MODE>(d, ln, n, l, c);
    }
  }
  __syncthreads();
  smem_fft<N1, N2, DIR>(s, cols, n1s, n2s, tw);
  // X[k] sits at position (k % n1s) * n2s + k / n1s
  if constexpr (MODE == PassMode::kNakatshaOut) {
    __shared__ double red[MAXT / 32];
    // group of gc lanes per output pixel, lanes over coils, fixed-order tree;
    // with a power-of-two number of coil pairs, a lane per pair summed as the
    // pipelined and TMA inverse x passes sum (nak_pair_term, then the tree)
    const bool pairs = (C & 1) == 0 && ((C / 2) & (C / 2 - 1)) == 0 && C / 2 <= 32;
    int gc = 1;
    if (pairs)
      gc = C / 2;
    else
      while (gc < C && gc < 32) gc <<= 1;
    const int groups = blockDim.x / gc;
    const int lane = threadIdx.x % gc, grp = threadIdx.x / gc;
    double sq = 0.0;
    const int nout = L * d.out_len;
    // loop bound uniform across the warp so every lane reaches the shuffles
    const int rounds = (nout + groups - 1) / groups;
    for (int rd = 0; rd < rounds; ++rd) {
      const int o = rd * groups + grp;
      const bool live = o < nout;
      const int l = live ? o / d.out_len : 0;
      const int k = d.out_lo + (live ? o - l * d.out_len : 0);
      const int ui = ln.u0 + l;
      const bool ok = live && ui < d.dims[1];
      const long long m = (k - d.out_lo) + (long long)d.out_len * (ui + (long long)d.dims[1] * ln.vi);
      const int pos = (k % n1s) * n2s + k / n1s;
      const float sg = ((k + d.coord_off[1] + ui + d.coord_off[2] + ln.vi) & 1) ? -d.sfac : d.sfac;
      float2 acc = make_float2(0.f, 0.f);
      if (ok && pairs) {
        const float4 sv = *reinterpret_cast<const float4*>(s + pos * cols + l * C + 2 * lane);
        const float4 kv = __ldg(reinterpret_cast<const float4*>(d.kfc + m * C + 2 * lane));
        acc = nak_pair_term(sv, kv, sg);
      } else if (ok) {
        for (int c = lane; c < C; c += gc) {
          float2 v = s[pos * cols + l * C + c];
          v = make_float2(v.x * sg, v.y * sg);
          const float2 t = cmulf(v, __ldg(d.kfc + m * C + c));
          acc.x += t.x;
          acc.y += t.y;
        }
      }
      for (int w = gc / 2; w > 0; w >>= 1) {
        acc.x = __fadd_rn(acc.x, __shfl_xor_sync(0xffffffffu, acc.x, w, gc));
        acc.y = __fadd_rn(acc.y, __shfl_xor_sync(0xffffffffu, acc.y, w, gc));
      }
      if (ok && lane == 0) {
        d.img_out[m] = acc;
        sq += (double)acc.x * acc.x + (double)acc.y * acc.y;
      }
    }
    if (d.partial) {
      for (int o = 16; o > 0; o >>= 1) sq += __shfl_down_sync(0xffffffffu, sq, o);
      if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = sq;
      __syncthreads();
      if (threadIdx.x == 0) {
        double t = 0.0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += red[i];
        d.partial[blockIdx.x] = t;
      }
    }
  } else if ((C & 1) == 0 && (int)blockDim.x % cv == 0) {
    const int vc = threadIdx.x % cv, rstep = blockDim.x / cv;
    const int col = vc * 2, l = col / C, c = col - l * C;
    const int ui = ln.u0 + l;
    if (ui < d.dims[ln.u]) {
      const float4* s4 = reinterpret_cast<const float4*>(s);
      float2* base = d.out + (long long)ui * d.out_stride[ln.u] + (long long)ln.vi * d.out_stride[ln.v] + c;
      const long long st = d.out_stride[d.ax];
#pragma unroll 4
      for (int kk = threadIdx.x / cv; kk < d.out_len; kk += rstep) {
        const int k = d.out_lo + kk;
        const int pos = (k % n1s) * n2s + k / n1s;
        *reinterpret_cast<float4*>(base + (long long)kk * st) = s4[pos * cv + vc];
      }
    }
  } else {
    for (int it = threadIdx.x; it < d.out_len * cols; it += blockDim.x) {
      const int kk = it / cols, col = it - (it / cols) * cols;
      const int l = col / C, c = col - (col / C) * C;
      const int ui = ln.u0 + l;
      if (ui >= d.dims[ln.u]) continue;
      const int k = d.out_lo + kk;
      const int pos = (k % n1s) * n2s + k / n1s;
      const long long off = (long long)kk * d.out_stride[d.ax] + (long long)ui * d.out_stride[ln.u] +
                            (long long)ln.vi * d.out_stride[ln.v] + c;
      d.out[off] = s[pos * cols + col];
    }
  }
}

// ---- pipelined plain passes ------------------------------------------------------
// A persistent CTA walks the line bundles b = blockIdx.x, + gridDim.x, ...
// with two shared buffers: while it transforms and stores bundle b from one,
// the next bundle's lines arrive in the other through 16-byte asynchronous
// copies (cp.async); cells outside the stored input range or unset in the
// occupancy mask are written as zeros directly.  Loads thus overlap the
// transform and the stores inside every CTA instead of only across CTAs.
// Coil pairs per thread (even C), fixed column per thread (blockDim a
// multiple of the columns), templated transform sizes only.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int PENDING>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(PENDING) : "memory");
}

// The transform of smem_fft for a compile-time column count COLS and CTA
// size NT (a multiple of COLS): every shared-memory offset is an immediate.
// SMEM_TW: tw is the twiddle table copied into shared memory (a short
// shared-memory load instead of a global one per twiddle).
template <int N1, int N2, int DIR, int COLS, int NT, bool SMEM_TW = false>
__device__ __forceinline__ void smem_fft_fixed(float2* s, const float2* __restrict__ tw) {
  static_assert(NT % COLS == 0, "CTA size must be a multiple of the columns");
  constexpr int G = NT / COLS;  // row groups
  const int col = threadIdx.x % COLS, g = threadIdx.x / COLS;
  float2* const sc = s + col;
#pragma unroll
  for (int n2b = 0; n2b < N2; n2b += G) {
    const int n2 = n2b + g;
    if (N2 % G == 0 || n2 < N2) {
      float2* const p = sc + n2 * COLS;
      float2 r[N1];
#pragma unroll
      for (int n1 = 0; n1 < N1; ++n1) r[n1] = p[n1 * N2 * COLS];
      reg_fft<N1, DIR>(r);
      if (n2) {
#pragma unroll
        for (int k1 = 1; k1 < N1; ++k1) {
          float2 w;
          if constexpr (SMEM_TW) {
            w = tw[n2 * k1];
            if (DIR > 0) w.y = -w.y;
          } else {
            w = twid<DIR>(tw, n2 * k1);
          }
          r[k1] = cmulf(r[k1], w);
        }
      }
#pragma unroll
      for (int k1 = 0; k1 < N1; ++k1) p[k1 * N2 * COLS] = r[k1];
    }
  }
  __syncthreads();
#pragma unroll
  for (int k1b = 0; k1b < N1; k1b += G) {
    const int k1 = k1b + g;
    if (N1 % G == 0 || k1 < N1) {
      float2* const p = sc + k1 * N2 * COLS;
      float2 r[N2];
#pragma unroll
      for (int n2 = 0; n2 < N2; ++n2) r[n2] = p[n2 * COLS];
      reg_fft<N2, DIR>(r);
#pragma unroll
      for (int k2 = 0; k2 < N2; ++k2) p[k2 * COLS] = r[k2];
    }
  }
  __syncthreads();
}

// Issues (without committing) the asynchronous copies of line bundle b into
// dst ([N][cv] float4, coil pairs): thread (r0, vc) copies rows r0, r0 +
// rstep, ... of its coil pair; rows outside the stored input range, cells
// unset in the occupancy mask and lines past the grid edge are written as
// zeros.  EXACT: rstep divides N (every thread has the same row count).
// lbits (optional): the bundle's line masks in shared memory (lw words per
// line), read in place of the occupancy mask in global memory.
template <int N, bool EXACT>
__device__ __forceinline__ void pipe_issue_lines(const PassDesc& d, int L, int gu, int l, int c, int vc, int r0,
                                                 int cv, int rstep, int b, float4* dst, const uint32_t* lbits,
                                                 int lw) {
  const int u = d.ax == 0 ? 1 : 0, v = d.ax == 2 ? 1 : 2;
  const long long ist = d.in_stride[d.ax], cst = d.cell_stride[d.ax];
  const uint32_t* mask = d.in_mask;
  const int in_lo = d.in_lo, in_hi = d.in_lo + d.in_len;
  const int ui = (b % gu) * L + l, vi = b / gu;
  const bool line_ok = ui < d.dims[u];
  const float2* src = d.in + (long long)ui * d.in_stride[u] + (long long)vi * d.in_stride[v] + c +
                      (long long)(r0 - in_lo) * ist;
  const long long cell0 = (long long)ui * d.cell_stride[u] + (long long)vi * d.cell_stride[v] + (long long)r0 * cst;
  float4* const drow = dst + r0 * cv + vc;
  // rows in batches of 8: the batch's mask words are loaded together before
  // any copy depends on them
  constexpr int kB = 8;
#pragma unroll
  for (int nb0 = 0; nb0 < N; nb0 += kB * rstep) {
    bool ld[kB];
#pragma unroll
    for (int j = 0; j < kB; ++j) {
      const int n = nb0 + j * rstep + r0;
      const bool row = EXACT ? nb0 + j * rstep < N : n < N;
      ld[j] = line_ok && row && n >= in_lo && n < in_hi;
    }
    if (lbits) {
      const uint32_t* lb = lbits + l * lw;
#pragma unroll
      for (int j = 0; j < kB; ++j) {
        const int n = nb0 + j * rstep + r0;
        ld[j] = ld[j] && ((lb[n >> 5] >> (n & 31)) & 1u);
      }
    } else if (mask) {
      uint32_t w[kB];
#pragma unroll
      for (int j = 0; j < kB; ++j) {
        const long long cell = cell0 + (long long)(nb0 + j * rstep) * cst;
        w[j] = ld[j] ? __ldg(mask + (cell >> 5)) >> (cell & 31) : 0u;
      }
#pragma unroll
      for (int j = 0; j < kB; ++j) ld[j] = ld[j] && (w[j] & 1u);
    }
#pragma unroll
    for (int j = 0; j < kB; ++j) {
      const int nrel = nb0 + j * rstep;
      const bool row = EXACT ? nrel < N : nrel + r0 < N;
      if (row) {
        float4* dp = drow + nrel * cv;
        if (ld[j])
          cp_async16(dp, src + (long long)nrel * ist);
        else
          *dp = make_float4(0.f, 0.f, 0.f, 0.f);
      }
    }
  }
}

// Resident CTAs per SM the pipelined pass asks the register allocator for:
// what its shared memory allows (two N x cols buffers), at most 3.
constexpr int pipe_min_blocks(int N, int cols, int maxt) {
  if (cols == 0) return maxt > 256 ? 1 : (N <= 256 ? 3 : 2);
  const int by_smem = (227 * 1024) / (2 * N * cols * 8 + 1024);
  return by_smem < 1 ? 1 : (by_smem > 3 ? 3 : by_smem);
}

// COLS > 0: the CTA covers exactly COLS columns with cta_threads(COLS)
// threads, both compile-time; COLS == 0: L * C columns, blockDim threads.
template <int N1, int N2, int DIR, int MAXT, int COLS>
__global__ void __launch_bounds__(COLS > 0 ? cta_threads(COLS) : MAXT,
                                  pipe_min_blocks(N1 * N2, COLS, COLS > 0 ? cta_threads(COLS) : MAXT))
    fft_pass_pipe_kernel(PassDesc d, int L, int nbundles, const float2* __restrict__ tw) {
  extern __shared__ float4 s4all[];
  constexpr int N = N1 * N2;
  constexpr int NT = COLS > 0 ? cta_threads(COLS) : 0;
  constexpr int kRstep = COLS > 0 ? NT / (COLS / 2) : 0;
  constexpr bool kExact = COLS > 0 && N % kRstep == 0;  // every thread has the same rows
  const int C = d.C;
  const int cols = COLS > 0 ? COLS : L * C, cv = cols >> 1;
  const int nthr = COLS > 0 ? NT : (int)blockDim.x;
  float4* const buf0 = s4all;
  float4* const buf1 = s4all + (size_t)N * cv;
  const int vc = threadIdx.x % cv, rstep = nthr / cv, r0 = threadIdx.x / cv;
  const int col = vc * 2, l = col / C, c = col - l * C;
  const int u = d.ax == 0 ? 1 : 0, v = d.ax == 2 ? 1 : 2;
  const int gu = (d.dims[u] + L - 1) / L;
  const long long ost = d.out_stride[d.ax];
  // line masks (optional): a ring of 4 slots of L x LW words after the two
  // buffers; the masks of the bundle three iterations ahead are copied with
  // the next bundle's lines, so they have landed (and a barrier has passed)
  // before the iteration that issues that bundle's copies reads them
  const int LW = d.lmask_words;
  uint32_t* const ring = d.in_lmask ? reinterpret_cast<uint32_t*>(s4all + 2 * (size_t)N * cv) : nullptr;
  auto slot = [&](int k) { return ring + (k & 3) * L * LW; };
  auto fetch_masks = [&](int bk, uint32_t* dst) {
    const int per_line = LW >> 2;
    for (int t = threadIdx.x; t < L * per_line; t += nthr) {
      const int ll = t / per_line, w4 = t - ll * per_line;
      const int ui = (bk % gu) * L + ll, vi = bk / gu;
      if (ui < d.dims[u])
        cp_async16(dst + ll * LW + 4 * w4, d.in_lmask + ((long long)ui + (long long)d.dims[u] * vi) * LW + 4 * w4);
    }
  };

  int b = blockIdx.x;
  if (b >= nbundles) return;
  const int G = gridDim.x;
  const float hs = d.out_half ? half_store_scale(d.h_amax, d.h_len) : 1.f;
  if (ring) {  // masks of the first three bundles
    for (int k = 0; k < 3; ++k)
      if (b + k * G < nbundles) fetch_masks(b + k * G, slot(k));
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
  }
  pipe_issue_lines<N, kExact>(d, L, gu, l, c, vc, r0, cv, rstep, b, buf0, ring ? slot(0) : nullptr, LW);
  cp_async_commit();
  for (int it = 0; b < nbundles; ++it, b += G) {
    float4* cur = (it & 1) ? buf1 : buf0;
    const int nb = b + G;
    if (nb < nbundles) {
      pipe_issue_lines<N, kExact>(d, L, gu, l, c, vc, r0, cv, rstep, nb, (it & 1) ? buf0 : buf1,
                                  ring ? slot(it + 1) : nullptr, LW);
      if (ring && b + 3 * G < nbundles) fetch_masks(b + 3 * G, slot(it + 3));
      cp_async_commit();
      cp_async_wait<1>();  // all but the copies just issued have landed
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    if constexpr (COLS > 0)
      smem_fft_fixed<N1, N2, DIR, COLS, NT>(reinterpret_cast<float2*>(cur), tw);  // ends with a barrier
    else
      smem_fft<N1, N2, DIR>(reinterpret_cast<float2*>(cur), cols, N1, N2, tw);
    const int ui = (b % gu) * L + l, vi = b / gu;
    if (ui < d.dims[u]) {
      const long long obase = (long long)ui * d.out_stride[u] + (long long)vi * d.out_stride[v] + c;
      const float4* const scol = cur + vc;
      if (d.out_half) {  // FP16 intermediate (mixed precision): complex -> __half2, times hs
        __half2* const hb = reinterpret_cast<__half2*>(d.out) + obase;
#pragma unroll 4
        for (int kk = r0; kk < d.out_len; kk += rstep) {
          const int k = d.out_lo + kk;
          const float4 w = scol[((k % N1) * N2 + k / N1) * cv];
          const __half2 h0 = __floats2half2_rn(w.x * hs, w.y * hs), h1 = __floats2half2_rn(w.z * hs, w.w * hs);
          uint2 q;
          q.x = *reinterpret_cast<const unsigned*>(&h0);
          q.y = *reinterpret_cast<const unsigned*>(&h1);
          *reinterpret_cast<uint2*>(hb + (long long)kk * ost) = q;
        }
      } else {
        float2* const ob = d.out + obase;
#pragma unroll 4
        for (int kk = r0; kk < d.out_len; kk += rstep) {
          const int k = d.out_lo + kk;
          const int pos = (k % N1) * N2 + k / N1;
          *reinterpret_cast<float4*>(ob + (long long)kk * ost) = scol[pos * cv];
        }
      }
    }
    __syncthreads();  // cur is refilled by the copies issued in the next iteration
  }
}

// Pipelined forward x pass fused with x .* KFC, the zero-fill and the
// (-1)^(x+y+z) modulation (kShannaIn, one image shared by the coils).  The
// descriptor's `in` / `in_stride` describe KFC ([pixel][C], lines of in_len
// pixels): its rows arrive through pipe_issue_lines (zero outside [in_lo,
// in_lo + in_len)) and the bundle's image rows (L x in_len pixels,
// contiguous) through 8-byte copies in the same group.  The product is formed
// in shared memory before the transform.
template <int N1, int N2, int COLS>
__global__ void __launch_bounds__(cta_threads(COLS), pipe_min_blocks(N1 * N2, COLS, cta_threads(COLS)))
    fft_shanna_pipe_kernel(PassDesc d, int L, int nbundles, const float2* __restrict__ tw) {
  constexpr int N = N1 * N2, NT = cta_threads(COLS), CV = COLS / 2, RSTEP = NT / CV;
  extern __shared__ float4 s4all[];
  const int C = d.C, in_lo = d.in_lo, in_len = d.in_len, in_hi = d.in_lo + d.in_len;
  float4* const lb0 = s4all;
  float4* const lb1 = s4all + N * CV;
  float2* const xb0 = reinterpret_cast<float2*>(s4all + 2 * N * CV);
  float2* const xb1 = xb0 + L * in_len;
  float2* const tws = xb1 + L * in_len;  // twiddle table (N values), copied once
  const int vc = threadIdx.x % CV, r0 = threadIdx.x / CV;
  const int col = vc * 2, l = col / C, c = col - l * C;
  const int gu = (d.dims[1] + L - 1) / L;  // x pass: lines over (y, z)
  for (int i = threadIdx.x; i < N; i += NT) tws[i] = __ldg(tw + i);  // visible after the loop's first barrier

  auto issue = [&](int b, float4* ldst, float2* xdst) {
    pipe_issue_lines<N, N % RSTEP == 0>(d, L, gu, l, c, vc, r0, CV, RSTEP, b, ldst, nullptr, 0);
    const int u0 = (b % gu) * L, vi = b / gu;
    const int nl = min(L, d.dims[1] - u0);
    const float2* xsrc = d.img + (long long)in_len * (u0 + (long long)d.dims[1] * vi);
    for (int i = threadIdx.x; i < nl * in_len; i += NT) cp_async8(xdst + i, xsrc + i);
    cp_async_commit();
  };

  int b = blockIdx.x;
  if (b >= nbundles) return;
  float amax = 0.f;
  issue(b, lb0, xb0);
  for (int it = 0; b < nbundles; ++it, b += gridDim.x) {
    float4* const cur = (it & 1) ? lb1 : lb0;
    const float2* const xcur = (it & 1) ? xb1 : xb0;
    const int nb = b + gridDim.x;
    if (nb < nbundles) {
      issue(nb, (it & 1) ? lb0 : lb1, (it & 1) ? xb0 : xb1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const int ui = (b % gu) * L + l, vi = b / gu;
    if (ui < d.dims[1]) {  // other lines hold zeros (and no image rows)
      const int par = (d.coord_off[1] + ui + d.coord_off[2] + vi) & 1;
      const float2* const xl = xcur + l * in_len - in_lo;
      for (int n = r0; n < N; n += RSTEP) {
        if (n >= in_lo && n < in_hi) {
          const float4 k = cur[n * CV + vc];
          const float2 a = xl[n];
          float2 p0 = cmulf_rn(a, make_float2(k.x, k.y)), p1 = cmulf_rn(a, make_float2(k.z, k.w));
          if ((n + par) & 1) {
            p0 = make_float2(-p0.x, -p0.y);
            p1 = make_float2(-p1.x, -p1.y);
          }
          cur[n * CV + vc] = make_float4(p0.x, p0.y, p1.x, p1.y);
        }
      }
    }
    __syncthreads();
    smem_fft_fixed<N1, N2, -1, COLS, NT, true>(reinterpret_cast<float2*>(cur), tws);  // ends with a barrier
    if (ui < d.dims[1]) {
      float2* obase = d.out + (long long)ui * d.out_stride[1] + (long long)vi * d.out_stride[2] + c;
      const float4* const scol = cur + vc;
      const long long ost = d.out_stride[0];
#pragma unroll 4
      for (int kk = r0; kk < d.out_len; kk += RSTEP) {
        const int k = d.out_lo + kk;
        const int pos = (k % N1) * N2 + k / N1;
        const float4 w = scol[pos * CV];
        *reinterpret_cast<float4*>(obase + (long long)kk * ost) = w;
        amax = fmaxf(amax, absmax4(w));
      }
    }
    __syncthreads();  // both buffers are refilled by the next iteration's copies
  }
  if (d.out_absmax) warp_amax(d.out_absmax, amax);  // the FP16 passes' scale (mixed precision)
}

// Pipelined inverse x pass fused with .* KFC_conj and the coil sum
// (kNakatshaOut) for coil counts C = 2 CP with CP | 8 (2, 4, 8, 16 coils):
// 16 columns (L = 16 / C lines) per bundle.  The bundle's KFC_conj rows
// (contiguous: L lines x out_len pixels x C coils) arrive in the same copy
// group as its lines.  After the transform a group of CP lanes per output
// pixel multiplies its coil pairs and sums them by a shuffle tree; the
// group's first lane stores the pixel and adds |x|^2 (FP64) to the thread's
// sum, reduced per CTA into partial[blockIdx.x].  CTA 0 zeroes the slots
// [gridDim.x, n_slots) so that the caller reduces n_slots values.
template <int N1, int N2, int CP>
__global__ void __launch_bounds__(256, 2)
    fft_nak_pipe_kernel(PassDesc d, int L, int nbundles, int n_slots, const float2* __restrict__ tw) {
  constexpr int COLS = 16, NT = 256, N = N1 * N2, CV = COLS / 2, RSTEP = NT / CV;
  static_assert(cta_threads(COLS) == NT && CV % CP == 0, "bundle shape");
  constexpr int G = NT / CP;  // pixel groups per round
  extern __shared__ float4 s4all[];
  __shared__ double red[NT / 32];
  const int C = 2 * CP;
  const int out_len = d.out_len;
  float4* const lb0 = s4all;
  float4* const lb1 = s4all + N * CV;
  float4* const kb0 = s4all + 2 * N * CV;
  float4* const kb1 = kb0 + out_len * CV;
  float2* const tws = reinterpret_cast<float2*>(kb1 + out_len * CV);  // twiddle table (N values)
  for (int i = threadIdx.x; i < N; i += NT) tws[i] = __ldg(tw + i);  // visible after the loop's first barrier
  const int vc = threadIdx.x % CV, r0 = threadIdx.x / CV;
  const int col = vc * 2, l = col / C, c = col - l * C;
  const int gu = (d.dims[1] + L - 1) / L;  // x pass: lines over (y, z)
  const int q = threadIdx.x % CP, grp = threadIdx.x / CP;

  auto issue = [&](int b, float4* ldst, float4* kdst) {
    pipe_issue_lines<N, N % RSTEP == 0>(d, L, gu, l, c, vc, r0, CV, RSTEP, b, ldst, nullptr, 0);
    const int u0 = (b % gu) * L, vi = b / gu;
    const int nl = min(L, d.dims[1] - u0);  // lines inside the grid
    const float4* ksrc =
        reinterpret_cast<const float4*>(d.kfc + (long long)out_len * (u0 + (long long)d.dims[1] * vi) * C);
    const int n4 = nl * out_len * CP;
    for (int i = threadIdx.x; i < n4; i += NT) cp_async16(kdst + i, ksrc + i);
    cp_async_commit();
  };

  double sq = 0.0;
  int b = blockIdx.x;
  if (b < nbundles) issue(b, lb0, kb0);
  for (int it = 0; b < nbundles; ++it, b += gridDim.x) {
    float4* const cur = (it & 1) ? lb1 : lb0;
    const float4* const kcur = (it & 1) ? kb1 : kb0;
    const int nb = b + gridDim.x;
    if (nb < nbundles) {
      issue(nb, (it & 1) ? lb0 : lb1, (it & 1) ? kb0 : kb1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    smem_fft_fixed<N1, N2, 1, COLS, NT, true>(reinterpret_cast<float2*>(cur), tws);  // ends with a barrier
    const int u0 = (b % gu) * L, vi = b / gu;
    const int total = L * out_len;
    const int rounds = (total + G - 1) / G;  // uniform: every lane reaches the shuffles
    for (int rd = 0; rd < rounds; ++rd) {
      const int o = rd * G + grp;
      const bool live = o < total;
      const int ll = live ? o / out_len : 0;
      const int kk = live ? o - ll * out_len : 0;
      const int ui = u0 + ll;
      const bool ok = live && ui < d.dims[1];
      const int k = d.out_lo + kk;
      float2 acc = make_float2(0.f, 0.f);
      if (ok) {
        const int pos = (k % N1) * N2 + k / N1;
        const float sg = ((k + d.coord_off[1] + ui + d.coord_off[2] + vi) & 1) ? -d.sfac : d.sfac;
        const float4 sv = cur[pos * CV + ll * CP + q];
        const float4 kv = kcur[(ll * out_len + kk) * CP + q];
        acc = nak_pair_term(sv, kv, sg);
      }
#pragma unroll
      for (int w = CP / 2; w > 0; w >>= 1) {
        acc.x = __fadd_rn(acc.x, __shfl_xor_sync(0xffffffffu, acc.x, w, CP));
        acc.y = __fadd_rn(acc.y, __shfl_xor_sync(0xffffffffu, acc.y, w, CP));
      }
      if (ok && q == 0) {
        d.img_out[kk + (long long)out_len * (ui + (long long)d.dims[1] * vi)] = acc;
        sq += (double)acc.x * acc.x + (double)acc.y * acc.y;
      }
    }
    __syncthreads();  // both buffers are refilled by the next iteration's copies
  }
  if (d.partial) {
    for (int o = 16; o > 0; o >>= 1) sq += __shfl_down_sync(0xffffffffu, sq, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = sq;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int i = 0; i < NT / 32; ++i) t += red[i];
      d.partial[blockIdx.x] = t;
    }
    if (blockIdx.x == 0)
      for (int i = (int)gridDim.x + threadIdx.x; i < n_slots; i += NT) d.partial[i] = 0.0;
  }
}

}  // namespace mlg

#include "mlg_fft_tma.cuh"

namespace mlg {

// ---- launch helpers ------------------------------------------------------------
// Lines per CTA: 32 columns (256-byte row segments) for streaming passes; the
// gathering pass uses 16 columns so that twice as many CTAs (and gathers)
// are resident per SM.
static inline int lines_per_cta(const FftAxisPlan& a, int C, PassMode mode) {
  const int target = mode == PassMode::kGutIn ? 16 : 32;
  int L = std::max(1, (target + C - 1) / C);
  while (L > 1 && (size_t)a.N * L * C * sizeof(float2) > kFftSmemCap) --L;
  return L;
}

static inline int blocks_for(const PassDesc& d, int L) {
  const int u = d.ax == 0 ? 1 : 0, v = d.ax == 2 ? 1 : 2;
  return ((d.dims[u] + L - 1) / L) * d.dims[v];
}

static inline int threads_for(int cols) { return cta_threads(cols); }

// A pass descriptor asks for an FP16 intermediate or a recorded maximum that
// the pass shape's kernel does not provide (no message for a dry run).
static inline int half_unsupported(const PassDesc& d) {
  if (d.dry) return MLG_ERR_UNSUPPORTED;
  return fail(MLG_ERR_UNSUPPORTED, "FP16 pass intermediate / maximum not available for this pass shape");
}

template <int N1, int N2, int DIR, PassMode MODE, int MAXT>
static int launch_bounded(const FftAxisPlan& a, const PassDesc& d, int L, int threads, cudaStream_t s) {
  if (d.dry) return MLG_OK;
  const size_t smem = (size_t)a.N * L * d.C * sizeof(float2);
  static bool attr = false;  // per instantiation
  if (!attr) {
    MLG_CUDA(cudaFuncSetAttribute(fft_pass_kernel<N1, N2, DIR, MODE, MAXT>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(200 * 1024)));
    attr = true;
  }
  fft_pass_kernel<N1, N2, DIR, MODE, MAXT><<<blocks_for(d, L), threads, smem, s>>>(d, L, a.N1, a.N2, a.tw);
  MLG_LAUNCHED();
  return MLG_OK;
}

// Pipelined plain pass: ~16 columns per bundle (the two buffers take the
// shared memory of one 32-column buffer), a persistent grid of (resident
// CTAs per SM) x SMs.
template <int N1, int N2, int DIR, int MAXT, int COLS>
static int launch_pipe(const FftAxisPlan& a, const PassDesc& d, int Lp, int threads, cudaStream_t s) {
  if (d.dry) return MLG_OK;
  const size_t smem = 2 * (size_t)a.N * Lp * d.C * sizeof(float2) +
                      (d.in_lmask ? 4 * (size_t)Lp * d.lmask_words * sizeof(uint32_t) : 0);
  // per instantiation and host thread (serving workers launch concurrently);
  // recomputed when the coil count changes the CTA's shared memory or threads
  thread_local int per_sm = 0, sms = 0, per_sm_threads = 0;
  thread_local size_t per_sm_smem = 0;
  if (per_sm == 0 || per_sm_smem != smem || per_sm_threads != threads) {
    MLG_CUDA(cudaFuncSetAttribute(fft_pass_pipe_kernel<N1, N2, DIR, MAXT, COLS>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(200 * 1024)));
    int dev = 0;
    MLG_CUDA(cudaGetDevice(&dev));
    MLG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    MLG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fft_pass_pipe_kernel<N1, N2, DIR, MAXT, COLS>,
                                                           threads, smem));
    per_sm = std::max(1, per_sm);
    per_sm_smem = smem;
    per_sm_threads = threads;
  }
  const int nb = blocks_for(d, Lp);
  const int grid = std::max(1, std::min(nb, per_sm * sms));
  fft_pass_pipe_kernel<N1, N2, DIR, MAXT, COLS><<<grid, threads, smem, s>>>(d, Lp, nb, a.tw);
  MLG_LAUNCHED();
  return MLG_OK;
}

// TMA pass (fft_pass_tma_kernel, NSLOT bundle buffers) for a plain pass:
// *launched stays false when the shape does not fit the TMA boxes (the
// caller then takes the cp.async pipelined pass).  The masked first inverse
// pass runs as MASKED (16-row chunk boxes loaded where the line masks have
// occupied rows) when its line masks exist and a bundle's mask words fit one
// slot; copying each occupied row by itself instead had measured slower than
// the cp.async pass (c2: 1.19 against 0.69 ms).
template <int N1, int N2, int DIR, int COLS, int NSLOT>
static int launch_tma(const FftAxisPlan& a, const PassDesc& d, int Lp, cudaStream_t s, bool* launched) {
  constexpr int N = N1 * N2, NT = cta_threads(COLS);
  *launched = false;
  // register budget of step C: shapes beyond it are not instantiated
  if constexpr (tma_step_c_iters<N1, N2, COLS, NT>() * N2 > 32) return MLG_OK;
  else {
  if (d.in_lo < 0 || d.in_len < 1 || d.in_lo + d.in_len > N || d.out_lo < 0 || d.out_len < 1 ||
      d.out_lo + d.out_len > N || Lp * d.C != COLS)
    return MLG_OK;
  const bool ih = d.in_half != 0, oh = d.out_half != 0;
  // masked: the first inverse pass over the whole stored line, with masks of
  // N / 32 words per line for at most kTmaMaskWords words per bundle
  const bool masked = d.in_mask != nullptr;
  if (masked && (DIR < 0 || !d.in_lmask || N % 32 || N / kTmaChunkRows > 32 || ih || d.in_lo != 0 ||
                 d.in_len != N || Lp * (N / 32) > kTmaMaskWords || d.lmask_words < N / 32))
    return MLG_OK;
  // masked stores (optional: without them every chunk is stored): the last
  // forward pass over the whole line, the same mask geometry
  const bool mask_out = d.out_lmask != nullptr && DIR < 0 && N % 32 == 0 && N / kTmaChunkRows <= 32 && !masked &&
                        d.out_lo == 0 && d.out_len == N && Lp * (N / 32) <= kTmaMaskWords &&
                        d.lmask_words >= N / 32;
  if constexpr (N2 > NT / COLS) {  // FP16 input needs one step-A line per thread
    if (ih) return MLG_OK;
  }
  const int u = d.ax == 0 ? 1 : 0, v = d.ax == 2 ? 1 : 2;
  TmaPass t;
  t.L = Lp;
  t.gu = (d.dims[u] + Lp - 1) / Lp;
  t.nbundles = blocks_for(d, Lp);
  t.in_chunks = masked ? N / kTmaChunkRows : (N + 255) / 256;
  t.out_chunks = mask_out ? N / kTmaChunkRows : (d.out_len + 255) / 256;
  if (N % t.in_chunks || d.out_len % t.out_chunks) return MLG_OK;
  t.in_rows = N / t.in_chunks;
  t.out_rows = d.out_len / t.out_chunks;
  t.in_lo = d.in_lo;
  t.out_lo = d.out_lo;
  t.err = d.wait_err;
  t.test_stall = tma_test_stall() ? 1 : 0;
  t.h_amax = d.h_amax;
  t.h_len = d.h_len;
  t.h_len_out = d.h_len_out;
  if (masked || mask_out) {
    t.lmask = masked ? d.in_lmask : d.out_lmask;
    t.lw = d.lmask_words;
    t.du = d.dims[u];
  }
  if ((ih || oh) && (!d.h_amax || (4 * d.C) % 16)) return MLG_OK;
  // shared-memory box starts on 128-byte boundaries
  const long long rowb_in = (long long)COLS * (ih ? 4 : 8), rowb_out = (long long)COLS * (oh ? 4 : 8);
  if ((t.in_rows * rowb_in) % 128 || (t.out_lo * rowb_out) % 128 || (t.out_rows * rowb_out) % 128) return MLG_OK;
  CUtensorMap tin, tout;
  if (tma_line_map(&tin, d.in, d.C, d.dims[u], d.in_stride[u], d.in_len, d.in_stride[d.ax], d.dims[v],
                   d.in_stride[v], Lp, t.in_rows, ih) != MLG_OK ||
      tma_line_map(&tout, d.out, d.C, d.dims[u], d.out_stride[u], d.out_len, d.out_stride[d.ax], d.dims[v],
                   d.out_stride[v], Lp, t.out_rows, oh) != MLG_OK)
    return MLG_OK;
  // an FP16 bundle lands in the upper half of its buffer: 128-byte aligned
  if (ih && ((size_t)N * COLS * 4) % 128) return MLG_OK;
  const size_t smem = (size_t)NSLOT * N * COLS * 8 + 2 * NSLOT * sizeof(uint64_t) + (size_t)N * 8 + 128 +
                      (masked || mask_out ? (size_t)NSLOT * (kTmaMaskWords + 1) * 4 : 0);
  if (smem > 200 * 1024) return MLG_OK;
  if (d.dry) {
    *launched = true;
    return MLG_OK;
  }
  auto kern = fft_pass_tma_kernel<N1, N2, DIR, COLS, NSLOT, false, false>;
  const int vi = (ih ? 1 : 0) + (oh ? 2 : 0) + (masked ? 4 : 0) + (mask_out ? 8 : 0);
  if constexpr (N2 <= NT / COLS) {
    if (ih) kern = oh ? fft_pass_tma_kernel<N1, N2, DIR, COLS, NSLOT, true, true>
                      : fft_pass_tma_kernel<N1, N2, DIR, COLS, NSLOT, true, false>;
  }
  if (oh && !ih) kern = fft_pass_tma_kernel<N1, N2, DIR, COLS, NSLOT, false, true>;
  if constexpr (DIR > 0 && N % 32 == 0) {  // the masked first inverse pass
    if (masked) kern = oh ? fft_pass_tma_kernel<N1, N2, DIR, COLS, NSLOT, false, true, true>
                          : fft_pass_tma_kernel<N1, N2, DIR, COLS, NSLOT, false, false, true>;
  }
  if constexpr (DIR < 0 && N % 32 == 0) {  // the last forward pass with masked stores
    if (mask_out && !ih)
      kern = oh ? fft_pass_tma_kernel<N1, N2, DIR, COLS, NSLOT, false, true, false, true>
                : fft_pass_tma_kernel<N1, N2, DIR, COLS, NSLOT, false, false, false, true>;
    if constexpr (N2 <= NT / COLS) {
      if (mask_out && ih)
        kern = oh ? fft_pass_tma_kernel<N1, N2, DIR, COLS, NSLOT, true, true, false, true>
                  : fft_pass_tma_kernel<N1, N2, DIR, COLS, NSLOT, true, false, false, true>;
    }
  }
  // per instantiation, variant and host thread
  thread_local int per_sm[16] = {}, sms = 0;
  thread_local size_t per_sm_smem[16] = {};
  if (per_sm[vi] == 0 || per_sm_smem[vi] != smem) {
    MLG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(200 * 1024)));
    int dev = 0;
    MLG_CUDA(cudaGetDevice(&dev));
    MLG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    MLG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[vi], kern, NT + 32, smem));
    per_sm[vi] = std::max(1, per_sm[vi]);
    per_sm_smem[vi] = smem;
  }
  const int grid = std::max(1, std::min(t.nbundles, per_sm[vi] * sms));
  kern<<<grid, NT + 32, smem, s>>>(tin, tout, t, a.tw);
  MLG_LAUNCHED();
  *launched = true;
  return MLG_OK;
  }
}

static inline int pipe_lines(const FftAxisPlan& a, int C) {
  int L = std::max(1, (16 + C - 1) / C);
  while (L > 1 && 2 * (size_t)a.N * L * C * sizeof(float2) > kFftSmemCap) --L;
  return L;
}

// Pipelined kNakatshaOut pass; n_slots = the CTA count of the unpipelined
// pass (the partial-sum slots the caller reduces), an upper bound of the grid.
// TMA forward x pass (fft_pass_tma_kernel SHANNA): the bundle's KFC rows
// are the loaded box (the coil-map volume seen as x lines, zero outside the
// stored x range), the lines' image values one bulk copy; AMAX when the
// pass records its largest output component.  *launched stays false when
// the shape does not fit (the caller then takes the cp.async pass).
template <int N1, int N2, int COLS, int NSLOT>
static int launch_tma_shanna(const FftAxisPlan& a, const PassDesc& d, int Lp, cudaStream_t s, bool* launched) {
  constexpr int N = N1 * N2, NT = cta_threads(COLS);
  *launched = false;
  if constexpr (tma_step_c_iters<N1, N2, COLS, NT>() * N2 > 32) return MLG_OK;
  else {
  // the image bulk copy: an even line length and a 16-byte aligned image
  if (d.img_per_coil || !d.img || !d.kfc || d.in_lo < 0 || d.in_len < 2 || (d.in_len & 1) ||
      d.in_lo + d.in_len > N || d.out_lo < 0 || d.out_len < 1 || d.out_lo + d.out_len > N || Lp * d.C != COLS ||
      d.out_half || ((uintptr_t)d.img & 15))
    return MLG_OK;
  TmaPass t;
  t.L = Lp;
  t.gu = (d.dims[1] + Lp - 1) / Lp;
  t.nbundles = blocks_for(d, Lp);
  t.in_chunks = (N + 255) / 256;
  t.out_chunks = (d.out_len + 255) / 256;
  if (N % t.in_chunks || d.out_len % t.out_chunks) return MLG_OK;
  t.in_rows = N / t.in_chunks;
  t.out_rows = d.out_len / t.out_chunks;
  t.in_lo = d.in_lo;
  t.out_lo = d.out_lo;
  t.err = d.wait_err;
  t.test_stall = tma_test_stall() ? 1 : 0;
  t.du = d.dims[1];
  t.img = d.img;
  t.img_len = d.in_len;
  t.par0 = (d.coord_off[1] + d.coord_off[2]) & 1;
  t.amax = d.out_absmax;
  const long long rowb = (long long)COLS * 8;  // shared-memory box starts on 128-byte boundaries
  if ((t.in_rows * rowb) % 128 || (t.out_lo * rowb) % 128 || (t.out_rows * rowb) % 128) return MLG_OK;
  CUtensorMap tin, tout;
  // KFC [pixel][coil] as a volume of x lines: lines along y (u) and z (v)
  if (tma_line_map(&tin, d.kfc, d.C, d.dims[1], (long long)d.in_len * d.C, d.in_len, d.C, d.dims[2],
                   (long long)d.in_len * d.dims[1] * d.C, Lp, t.in_rows) != MLG_OK ||
      tma_line_map(&tout, d.out, d.C, d.dims[1], d.out_stride[1], d.out_len, d.out_stride[0], d.dims[2],
                   d.out_stride[2], Lp, t.out_rows) != MLG_OK)
    return MLG_OK;
  const size_t smem = (size_t)NSLOT * N * COLS * 8 + 2 * NSLOT * sizeof(uint64_t) + (size_t)N * 8 + 128 +
                      (size_t)NSLOT * Lp * d.in_len * 8;
  if (smem > 200 * 1024) return MLG_OK;
  if (d.dry) {
    *launched = true;
    return MLG_OK;
  }
  auto kern = d.out_absmax ? fft_pass_tma_kernel<N1, N2, -1, COLS, NSLOT, false, false, false, false, true, true>
                           : fft_pass_tma_kernel<N1, N2, -1, COLS, NSLOT, false, false, false, false, true, false>;
  const int vi = d.out_absmax ? 1 : 0;
  thread_local int per_sm[2] = {}, sms = 0;
  thread_local size_t per_sm_smem[2] = {};
  if (per_sm[vi] == 0 || per_sm_smem[vi] != smem) {
    MLG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(200 * 1024)));
    int dev = 0;
    MLG_CUDA(cudaGetDevice(&dev));
    MLG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    MLG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[vi], kern, NT + 32, smem));
    per_sm[vi] = std::max(1, per_sm[vi]);
    per_sm_smem[vi] = smem;
  }
  const int grid = std::max(1, std::min(t.nbundles, per_sm[vi] * sms));
  kern<<<grid, NT + 32, smem, s>>>(tin, tout, t, a.tw);
  MLG_LAUNCHED();
  *launched = true;
  return MLG_OK;
  }
}

template <int N1, int N2, int CP>
static int launch_nak_pipe(const FftAxisPlan& a, const PassDesc& d, int n_slots, cudaStream_t s) {
  if (d.dry) return MLG_OK;
  const int Lp = 16 / (2 * CP);
  const size_t smem = 2 * ((size_t)a.N + d.out_len) * 16 * sizeof(float2) + (size_t)a.N * sizeof(float2);
  thread_local int per_sm = 0, sms = 0;
  thread_local size_t per_sm_smem = 0;
  if (per_sm == 0 || per_sm_smem != smem) {
    MLG_CUDA(cudaFuncSetAttribute(fft_nak_pipe_kernel<N1, N2, CP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(200 * 1024)));
    int dev = 0;
    MLG_CUDA(cudaGetDevice(&dev));
    MLG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    MLG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fft_nak_pipe_kernel<N1, N2, CP>, 256, smem));
    per_sm = std::max(1, per_sm);
    per_sm_smem = smem;
  }
  const int nb = blocks_for(d, Lp);
  const int grid = std::max(1, std::min(std::min(nb, per_sm * sms), n_slots));
  fft_nak_pipe_kernel<N1, N2, CP><<<grid, 256, smem, s>>>(d, Lp, nb, n_slots, a.tw);
  MLG_LAUNCHED();
  return MLG_OK;
}

// Pipelined kShannaIn pass over COLS columns (Lp lines).
template <int N1, int N2, int COLS>
static int launch_shanna_pipe(const FftAxisPlan& a, const PassDesc& d, int Lp, cudaStream_t s) {
  if (d.dry) return MLG_OK;
  PassDesc k = d;  // KFC as the copied input: rows of C values, lines of in_len rows
  k.in = d.kfc;
  k.in_stride[0] = d.C;
  k.in_stride[1] = (long long)d.in_len * d.C;
  k.in_stride[2] = (long long)d.in_len * d.dims[1] * d.C;
  k.in_mask = nullptr;
  k.in_lmask = nullptr;
  const size_t smem = 2 * (size_t)a.N * COLS * sizeof(float2) + 2 * (size_t)Lp * d.in_len * sizeof(float2) +
                      (size_t)a.N * sizeof(float2);
  thread_local int per_sm = 0, sms = 0;
  thread_local size_t per_sm_smem = 0;
  if (per_sm == 0 || per_sm_smem != smem) {
    MLG_CUDA(cudaFuncSetAttribute(fft_shanna_pipe_kernel<N1, N2, COLS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(200 * 1024)));
    int dev = 0;
    MLG_CUDA(cudaGetDevice(&dev));
    MLG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    MLG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fft_shanna_pipe_kernel<N1, N2, COLS>,
                                                           cta_threads(COLS), smem));
    per_sm = std::max(1, per_sm);
    per_sm_smem = smem;
  }
  const int nb = blocks_for(d, Lp);
  const int grid = std::max(1, std::min(nb, per_sm * sms));
  fft_shanna_pipe_kernel<N1, N2, COLS><<<grid, cta_threads(COLS), smem, s>>>(k, Lp, nb, a.tw);
  MLG_LAUNCHED();
  return MLG_OK;
}

template <int N1, int N2, int DIR, PassMode MODE>
static int launch_pass(const FftAxisPlan& a, const PassDesc& d, int L, cudaStream_t s) {
  if ((d.in_half || d.out_half) && !d.h_amax) return half_unsupported(d);
  if constexpr (MODE == PassMode::kShannaIn && N1 > 0) {
    // one image shared by the coils, even C, 16 / 24 / 32 columns per bundle
    const int Lp = pipe_lines(a, d.C), cols = Lp * d.C;
    if (!d.img_per_coil && (d.C & 1) == 0 && tma_passes_enabled() && d.tma_slots >= 2) {  // TMA x pass
      bool done = false;
      int st = MLG_OK;
      const bool three = d.tma_slots >= 3;
      switch (cols) {
        case 16:
          st = three ? launch_tma_shanna<N1, N2, 16, 3>(a, d, Lp, s, &done)
                     : launch_tma_shanna<N1, N2, 16, 2>(a, d, Lp, s, &done);
          break;
        case 24:
          st = three ? launch_tma_shanna<N1, N2, 24, 3>(a, d, Lp, s, &done)
                     : launch_tma_shanna<N1, N2, 24, 2>(a, d, Lp, s, &done);
          break;
        case 32:
          st = three ? launch_tma_shanna<N1, N2, 32, 3>(a, d, Lp, s, &done)
                     : launch_tma_shanna<N1, N2, 32, 2>(a, d, Lp, s, &done);
          break;
        default: break;
      }
      if (st != MLG_OK || done) return st;
    }
    if (!d.img_per_coil && (d.C & 1) == 0 && 2 * (size_t)a.N * cols * sizeof(float2) <= kFftSmemCap) {
      switch (cols) {
        case 16: return launch_shanna_pipe<N1, N2, 16>(a, d, Lp, s);
        case 24: return launch_shanna_pipe<N1, N2, 24>(a, d, Lp, s);
        case 32: return launch_shanna_pipe<N1, N2, 32>(a, d, Lp, s);
        default: break;
      }
    }
  }
  if constexpr (MODE == PassMode::kNakatshaOut && N1 > 0) {
    // 2, 4, 8 or 16 coils, two bundles of lines and KFC rows within ~100 KB
    if (2 * ((size_t)a.N + d.out_len) * 16 * sizeof(float2) <= 104 * 1024) {
      const int n_slots = blocks_for(d, L);
      switch (d.C) {
        case 16: return launch_nak_pipe<N1, N2, 8>(a, d, n_slots, s);
        case 8: return launch_nak_pipe<N1, N2, 4>(a, d, n_slots, s);
        case 4: return launch_nak_pipe<N1, N2, 2>(a, d, n_slots, s);
        case 2: return launch_nak_pipe<N1, N2, 1>(a, d, n_slots, s);
        default: break;
      }
    }
  }
  if constexpr (MODE == PassMode::kPlain && N1 > 0) {
    const int Lp = pipe_lines(a, d.C);
    const int cols = Lp * d.C, tp = threads_for(cols);
    if ((d.C & 1) == 0 && tp % cols == 0 && 2 * (size_t)a.N * cols * sizeof(float2) <= kFftSmemCap) {
      if (tma_passes_enabled() && d.tma_slots >= 2) {  // bundles moved by the TMA unit
        bool done = false;
        int st = MLG_OK;
        const bool three = d.tma_slots >= 3;
        switch (cols) {
          case 16:
            st = three ? launch_tma<N1, N2, DIR, 16, 3>(a, d, Lp, s, &done) : launch_tma<N1, N2, DIR, 16, 2>(a, d, Lp, s, &done);
            break;
          case 24:
            st = three ? launch_tma<N1, N2, DIR, 24, 3>(a, d, Lp, s, &done) : launch_tma<N1, N2, DIR, 24, 2>(a, d, Lp, s, &done);
            break;
          case 32:
            st = three ? launch_tma<N1, N2, DIR, 32, 3>(a, d, Lp, s, &done) : launch_tma<N1, N2, DIR, 32, 2>(a, d, Lp, s, &done);
            break;
          default: break;
        }
        if (st != MLG_OK || done) return st;
      }
      // FP16 input exists only on the TMA passes; the cp.async passes below
      // store FP16 but load FP32 only
      if (d.in_half) return half_unsupported(d);
      // the column counts of 2, 4, 8, 12, 16, 24 and 32 coils: compile-time
      switch (cols) {
        case 16: return launch_pipe<N1, N2, DIR, kFftThreads, 16>(a, d, Lp, tp, s);
        case 24: return launch_pipe<N1, N2, DIR, kFftMaxThreads, 24>(a, d, Lp, tp, s);
        case 32: return launch_pipe<N1, N2, DIR, kFftThreads, 32>(a, d, Lp, tp, s);
        default: break;
      }
      if (tp <= kFftThreads) return launch_pipe<N1, N2, DIR, kFftThreads, 0>(a, d, Lp, tp, s);
      return launch_pipe<N1, N2, DIR, kFftMaxThreads, 0>(a, d, Lp, tp, s);
    }
  }
  // the FP16 intermediates and the recorded maximum exist only on the
  // pipelined passes above
  if (d.in_half || d.out_half || d.out_absmax) return half_unsupported(d);
  const int threads = threads_for(L * d.C);
  if (threads <= kFftThreads) return launch_bounded<N1, N2, DIR, MODE, kFftThreads>(a, d, L, threads, s);
  return launch_bounded<N1, N2, DIR, MODE, kFftMaxThreads>(a, d, L, threads, s);
}

template <int DIR, PassMode MODE>
static int dispatch_size(const FftAxisPlan& a, const PassDesc& d, int L, cudaStream_t s) {
  if (a.fast) {
    switch (a.N1 * 100 + a.N2) {
      case 404: return launch_pass<4, 4, DIR, MODE>(a, d, L, s);
      case 408: return launch_pass<4, 8, DIR, MODE>(a, d, L, s);
      case 808: return launch_pass<8, 8, DIR, MODE>(a, d, L, s);
      case 816: return launch_pass<8, 16, DIR, MODE>(a, d, L, s);
      case 1616: return launch_pass<16, 16, DIR, MODE>(a, d, L, s);
      case 1632: return launch_pass<16, 32, DIR, MODE>(a, d, L, s);
      case 3232: return launch_pass<32, 32, DIR, MODE>(a, d, L, s);
      case 608: return launch_pass<6, 8, DIR, MODE>(a, d, L, s);
      case 812: return launch_pass<8, 12, DIR, MODE>(a, d, L, s);
      case 1216: return launch_pass<12, 16, DIR, MODE>(a, d, L, s);
      case 1624: return launch_pass<16, 24, DIR, MODE>(a, d, L, s);
      case 2432: return launch_pass<24, 32, DIR, MODE>(a, d, L, s);
      default: break;
    }
  }
  return launch_pass<0, 0, DIR, MODE>(a, d, L, s);
}

// one instantiation set per translation unit (mlg_fft_pass_*.cu)
int fft_dispatch_plain_fwd(const FftAxisPlan& a, const PassDesc& d, int L, cudaStream_t s);
int fft_dispatch_plain_inv(const FftAxisPlan& a, const PassDesc& d, int L, cudaStream_t s);
int fft_dispatch_shanna_in(const FftAxisPlan& a, const PassDesc& d, int L, cudaStream_t s);
int fft_dispatch_nakatsha_out(const FftAxisPlan& a, const PassDesc& d, int L, cudaStream_t s);
int fft_dispatch_gut_in(const FftAxisPlan& a, const PassDesc& d, int L, cudaStream_t s);

}  // namespace mlg
