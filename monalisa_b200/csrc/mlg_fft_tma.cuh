// Line-FFT passes moved by the tensor memory accelerator (TMA): the plain
// pipelined pass (zero-filled load, transform, cropped store) with its line
// bundles copied global -> shared and shared -> global by
// cp.async.bulk.tensor instead of per-thread 16-byte copies.  Included by
// mlg_fft_kernels.cuh (it uses the register transforms defined there).
//
// A CTA = NT transform threads (a multiple of the bundle's columns, as in
// fft_pass_pipe_kernel) + one producer warp.  The bundle of line group b
// (L lines x C coils, N rows) is one 4-D box of the volume
//   d0: the 2C floats of one cell, d1: line index u, d2: the FFT axis,
//   d3: line index v
// so one instruction loads it.  The input tensor's FFT-axis extent is the
// stored range [in_lo, in_lo + in_len) and the box starts at -in_lo: rows
// outside that range (and lines past the grid edge) arrive as zeros from the
// TMA unit's out-of-bounds fill.  The transform leaves the line in natural
// order, so the kept rows [out_lo, out_lo + out_len) are one contiguous box
// for the store.  NSLOT shared buffers rotate: the producer loads bundle
// it + NSLOT - 1 ahead while the transform threads work on bundle it; after
// a bundle's transform it stores the bundle and, once the store has read the
// buffer, loads the next bundle into it.
//
// MASKED (the first inverse pass of the masked adjoint, whose input grid
// holds Gut's non-empty rows and stale values elsewhere): the load boxes are
// chunks of kTmaChunkRows rows, and the producer loads only the chunks in
// which some line of the bundle has an occupied cell -- its line-mask bits
// for those rows are not all zero -- after copying the bundle's mask words into a per-slot
// shared area; the transform threads read each row's occupancy bit there and
// take zero for an unoccupied row (skipped chunks and stale cells alike).
// The producer fetches the mask words before it waits for the slot, so their
// latency overlaps that wait.
//
// MASK_OUT (the last forward pass, whose output grid is read only at cells
// Gut marks occupied): the store boxes are kTmaChunkRows-row chunks, and the producer
// stores only the chunks in which some line of the bundle has an occupied
// cell (mask words kept in the slot's shared area since the bundle's load);
// the other cells of the grid keep stale values, which no reader touches.
//
// Empty bundles (lines outside the occupied region: no chunk holds an
// occupied cell): the producer publishes the bundle's chunk bits in the
// slot's word `slot_any`; with MASK_OUT such a bundle is neither loaded nor
// transformed (nothing of it is stored), with MASKED its input is all zero,
// so the transform threads write zeros for its kept rows instead of
// transforming it.
//
// SHANNA (the forward x pass of the forward operator, bmShanna's x .* KFC,
// zero-fill and first FFT): the loaded box holds the bundle's KFC rows (the
// coil-map volume seen as x lines, zero outside the stored x range), one
// untiled bulk copy brings the lines' image values onto the same barrier,
// and the transform threads form x .* KFC with the centring modulation in
// place before the transform.  AMAX: the transform threads record the
// largest output component (the scale of the mixed-precision intermediate).
//
// Every wait is bounded (kTmaWaitNs of wall-clock time): a wait that runs out
// sets *err, makes the CTA's other waits give up at once, and the CTA returns
// after the copies it issued have finished.  No multicast form is used: each
// CTA reads and writes this GPU's own buffers only.
#pragma once

#include <cuda.h>

#include <cstdint>

namespace mlg {

constexpr unsigned long long kTmaWaitNs = 2000000000ull;  // 2 s per wait
constexpr int kTmaMaskWords = 32;  // mask words per slot (lines x words per line)
constexpr int kTmaChunkRows = 16;  // rows per load / store box of the masked passes
static_assert(32 % kTmaChunkRows == 0, "a mask word covers whole chunks");

// Chunk bits of mask word w of a line: bit w * (32 / kTmaChunkRows) + q set
// when rows [q * kTmaChunkRows, (q + 1) * kTmaChunkRows) of the word hold an
// occupied cell.
__device__ __forceinline__ uint32_t tma_chunk_bits(uint32_t word, int w) {
  constexpr int CPW = 32 / kTmaChunkRows;
  uint32_t r = 0;
#pragma unroll
  for (int q = 0; q < CPW; ++q) {
    const uint32_t part = CPW == 1 ? word : (word >> (q * kTmaChunkRows)) & ((1u << (kTmaChunkRows % 32)) - 1u);
    if (part) r |= 1u << (w * CPW + q);
  }
  return r;
}

struct TmaPass {
  int L = 1;          // lines per bundle
  int gu = 1;         // bundles along u
  int nbundles = 0;
  int in_chunks = 1;  // load boxes per bundle
  int in_rows = 0;    // rows per load box (in_chunks * in_rows = N)
  int in_lo = 0;      // first stored input row
  int out_lo = 0;     // first kept output row
  int out_chunks = 1;
  int out_rows = 0;   // rows per store box (out_chunks * out_rows = out_len)
  int* err = nullptr; // set to 1 when a wait runs out (device word), or NULL
  // FP16 input (IN_H) or output (OUT_H) bundles: the scale comes from the
  // component maximum the writer of the first FP16 pass's input recorded
  // (half_store_scale(h_amax, h_len))
  const unsigned* h_amax = nullptr;
  int h_len = 1;
  int h_len_out = 0;  // FP16 input and output: the output's length (0: h_len)
  // MASKED: line masks (lw words per line; line = u index + du * v index;
  // word w, bit j = occupancy of row 32 w + j)
  const uint32_t* lmask = nullptr;
  int lw = 0;
  int du = 0;  // (also SHANNA) lines along u in the volume
  // SHANNA: the image (img_len pixels per x line, shared by the coils) and
  // the parity of the modulation's line offset; AMAX: the recorded maximum
  const float2* img = nullptr;
  int img_len = 0;
  int par0 = 0;
  unsigned* amax = nullptr;
  // test hook (MLG_TEST_WAIT_TIMEOUT=1): CTA 0 never loads its first bundle,
  // so its transform threads' bounded wait runs out and the timeout path runs
  int test_stall = 0;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t addr, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(addr), "r"(parity)
      : "memory");
  return ok != 0;
}

// Waits for phase `parity` of *bar to complete.  Gives up (returns false)
// when *abort is set or after kTmaWaitNs, in which case it sets *abort and
// *err.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort, int* err) {
  const uint32_t addr = smem_u32(bar);
  if (mbar_try(addr, parity)) return true;
  const unsigned long long t0 = global_ns();
  for (;;) {
    if (mbar_try(addr, parity)) return true;
    if (*abort) return false;
    if (global_ns() - t0 > kTmaWaitNs) {
      *abort = 1;
      if (err) atomicExch(err, 1);
      return false;
    }
  }
}

// The same wait without the abort flag (draining copies already issued).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  const uint32_t addr = smem_u32(bar);
  const unsigned long long t0 = global_ns();
  while (!mbar_try(addr, parity))
    if (global_ns() - t0 > kTmaWaitNs) return false;
  return true;
}

__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
      "%5}], [%6];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
      : "memory");
}

// Untiled bulk copy global -> shared onto an mbarrier (no multicast); both
// addresses 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tma_store_4d(const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                             const void* src) {
  asm volatile("cp.async.bulk.tensor.4d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3, %4}], [%5];" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(src))
               : "memory");
}

__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read_all() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// barrier 1 over the NT transform threads (the producer warp never joins)
template <int NT>
__device__ __forceinline__ void bar_transform() {
  asm volatile("bar.sync 1, %0;" ::"n"(NT) : "memory");
}

// barrier 1 over the NT transform threads returning the OR of v
template <int NT>
__device__ __forceinline__ bool bar_transform_or(bool v) {
  uint32_t r;
  asm volatile(
      "{\n .reg .pred p, q;\n setp.ne.u32 q, %1, 0;\n bar.red.or.pred p, 1, %2, q;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(r)
      : "r"((uint32_t)v), "n"(NT)
      : "memory");
  return r != 0;
}

// Sub-transforms of step C per thread: all of a thread's step-C inputs stay
// in registers until every thread has read its own (KI * N2 values).
template <int N1, int N2, int COLS, int NT>
constexpr int tma_step_c_iters() {
  return (N1 + NT / COLS - 1) / (NT / COLS);
}

// smem_fft_fixed with the result in natural order (X[k] at row k): step A
// as there; step C reads all of a thread's rows, waits for every thread to
// have read its own, then writes row k1 + N1 k2.  Barriers are over the NT
// transform threads only.  tws: the axis' twiddle table exp(-2 pi i j/N)
// copied into shared memory (the same values as the global table).
// IN_H: the bundle arrived as FP16 in the upper half of the buffer; step A
// reads its rows from there (times hs_in), waits for every thread to have read,
// then writes FP32 (one n2 per thread: N2 <= NT / COLS).  OUT_H: step C
// writes the rows as FP16 (times hs_out) into the lower half, row k at k.
// MASKED: lbits = the thread's line's occupancy words; step A takes zero for
// a row whose bit is clear.
// AMAX: *amax is raised to the largest component the thread writes.
template <int N1, int N2, int DIR, int COLS, int NT, bool IN_H = false, bool OUT_H = false, bool MASKED = false,
          bool AMAX = false>
__device__ __forceinline__ void smem_fft_natural(float2* s, const float2* tws, float hs_in, float hs_out,
                                                 const uint32_t* lbits = nullptr, float* amax = nullptr) {
  constexpr int G = NT / COLS;
  constexpr int KI = tma_step_c_iters<N1, N2, COLS, NT>();
  const int col = threadIdx.x % COLS, g = threadIdx.x / COLS;
  float2* const sc = s + col;
  if constexpr (IN_H) {
    static_assert(N2 <= G, "FP16 input: one step-A line per thread");
    const __half2* const hsrc = reinterpret_cast<const __half2*>(s + (size_t)N1 * N2 * COLS / 2) + col;
    const int n2 = g;
    float2 r[N1];
    if (n2 < N2) {
#pragma unroll
      for (int n1 = 0; n1 < N1; ++n1) {
        const float2 v = __half22float2(hsrc[(n1 * N2 + n2) * COLS]);
        r[n1] = make_float2(v.x * hs_in, v.y * hs_in);
      }
    }
    bar_transform<NT>();  // every FP16 row read before FP32 rows overwrite them
    if (n2 < N2) {
      float2* const p = sc + n2 * COLS;
      reg_fft<N1, DIR>(r);
      if (n2) {
#pragma unroll
        for (int k1 = 1; k1 < N1; ++k1) {
          const float2 w = tws[n2 * k1];
          r[k1] = cmulf(r[k1], DIR < 0 ? w : make_float2(w.x, -w.y));
        }
      }
#pragma unroll
      for (int k1 = 0; k1 < N1; ++k1) p[k1 * N2 * COLS] = r[k1];
    }
  } else {
#pragma unroll
    for (int n2b = 0; n2b < N2; n2b += G) {
      const int n2 = n2b + g;
      if (N2 % G == 0 || n2 < N2) {
        float2* const p = sc + n2 * COLS;
        float2 r[N1];
#pragma unroll
        for (int n1 = 0; n1 < N1; ++n1) {
          if constexpr (MASKED) {
            const int row = n1 * N2 + n2;
            r[n1] = ((lbits[row >> 5] >> (row & 31)) & 1u) ? p[n1 * N2 * COLS] : make_float2(0.f, 0.f);
          } else {
            r[n1] = p[n1 * N2 * COLS];
          }
        }
        reg_fft<N1, DIR>(r);
        if (n2) {
#pragma unroll
          for (int k1 = 1; k1 < N1; ++k1) {
            const float2 w = tws[n2 * k1];
            r[k1] = cmulf(r[k1], DIR < 0 ? w : make_float2(w.x, -w.y));
          }
        }
#pragma unroll
        for (int k1 = 0; k1 < N1; ++k1) p[k1 * N2 * COLS] = r[k1];
      }
    }
  }
  bar_transform<NT>();
  float2 r[KI][N2];
#pragma unroll
  for (int i = 0; i < KI; ++i) {
    const int k1 = i * G + g;
    if (N1 % G == 0 || k1 < N1) {
      const float2* const p = sc + k1 * N2 * COLS;
#pragma unroll
      for (int n2 = 0; n2 < N2; ++n2) r[i][n2] = p[n2 * COLS];
      reg_fft<N2, DIR>(r[i]);
    }
  }
  bar_transform<NT>();
#pragma unroll
  for (int i = 0; i < KI; ++i) {
    const int k1 = i * G + g;
    if (N1 % G == 0 || k1 < N1) {
#pragma unroll
      for (int k2 = 0; k2 < N2; ++k2) {
        if constexpr (OUT_H)
          reinterpret_cast<__half2*>(s)[(k1 + N1 * k2) * COLS + col] =
              __floats2half2_rn(r[i][k2].x * hs_out, r[i][k2].y * hs_out);
        else
          sc[(k1 + N1 * k2) * COLS] = r[i][k2];
        if constexpr (AMAX) *amax = fmaxf(*amax, fmaxf(fabsf(r[i][k2].x), fabsf(r[i][k2].y)));
      }
    }
  }
}

template <int N, int COLS, int NSLOT>
constexpr int tma_min_blocks() {
  const int per = NSLOT * N * COLS * 8 + N * 8 + 2048;
  const int by_smem = (227 * 1024) / per;
  return by_smem < 1 ? 1 : (by_smem > 3 ? 3 : by_smem);
}

template <int N1, int N2, int DIR, int COLS, int NSLOT, bool IN_H = false, bool OUT_H = false, bool MASKED = false,
          bool MASK_OUT = false, bool SHANNA = false, bool AMAX = false>
__global__ void __launch_bounds__(cta_threads(COLS) + 32, (tma_min_blocks<N1 * N2, COLS, NSLOT>()))
    fft_pass_tma_kernel(const __grid_constant__ CUtensorMap tin, const __grid_constant__ CUtensorMap tout, TmaPass a,
                        const float2* __restrict__ tw) {
  constexpr int N = N1 * N2, NT = cta_threads(COLS);
  constexpr unsigned kBuf = (unsigned)N * COLS * 8;  // bytes per bundle
  extern __shared__ unsigned char tma_smem_raw[];
  // 128-byte aligned buffers (TMA boxes in shared memory), then the barriers
  unsigned char* base =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(tma_smem_raw) + 127) & ~uintptr_t(127));
  uint64_t* full = reinterpret_cast<uint64_t*>(base + NSLOT * kBuf);
  uint64_t* done = full + NSLOT;
  float2* tws = reinterpret_cast<float2*>(done + NSLOT);  // twiddle table, N values
  uint32_t* masks = reinterpret_cast<uint32_t*>(tws + N);  // MASKED: NSLOT x kTmaMaskWords
  uint32_t* slot_any = masks + NSLOT * kTmaMaskWords;      // MASKED / MASK_OUT: chunk bits per slot
  float2* xbuf = tws + N;  // SHANNA: NSLOT x (L x img_len) image values (in place of the masks)
  static_assert(!SHANNA || (!MASKED && !MASK_OUT && !IN_H && DIR < 0), "the forward x pass");
  constexpr int NW = (N + 31) / 32;                        // mask words per line
  static_assert(!MASKED || (N % 32 == 0 && !IN_H), "masked passes: whole mask words of an FP32 input");
  static_assert(!MASK_OUT || (N % 32 == 0 && !MASKED), "masked stores: whole mask words");
  constexpr bool kMasks = MASKED || MASK_OUT;  // the producer fetches the bundles' mask words
  __shared__ int abort_flag;
  const int tid = threadIdx.x;
  for (int i = tid; i < N; i += blockDim.x) tws[i] = __ldg(tw + i);
  if (tid == 0) {
    abort_flag = 0;
#pragma unroll
    for (int i = 0; i < NSLOT; ++i) {
      mbar_init(full + i, 1);
      mbar_init(done + i, NT);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  volatile int* abort = &abort_flag;
  const int G = gridDim.x;
  if (tid >= NT) {
    if (tid != NT) return;
    // producer: one thread
    constexpr int kInElem = IN_H ? 4 : 8, kOutElem = OUT_H ? 4 : 8;  // bytes per complex value
    // MASKED: the bundle's mask words (lines past the grid edge: zeros)
    uint32_t mw[kMasks ? kTmaMaskWords : 1];
    auto fetch_masks = [&](int b) {
      if constexpr (kMasks) {
        const int ui0 = (b % a.gu) * a.L, vi = b / a.gu;
#pragma unroll
        for (int i = 0; i < kTmaMaskWords; ++i) {
          const int l = i / NW, w = i - (i / NW) * NW;
          mw[i] = (l < a.L && ui0 + l < a.du)
                      ? __ldg(a.lmask + ((long long)(ui0 + l) + (long long)a.du * vi) * a.lw + w)
                      : 0u;
        }
      }
    };
    auto load = [&](int slot, int b) {
      unsigned char* dst = base + slot * kBuf + (IN_H ? kBuf / 2 : 0);
      const int c1 = (b % a.gu) * a.L, c3 = b / a.gu;
      if constexpr (MASKED) {
        uint32_t any = 0;  // bit k: chunk k holds an occupied row of some line
#pragma unroll
        for (int i = 0; i < kTmaMaskWords; ++i) {
          masks[slot * kTmaMaskWords + i] = mw[i];
          any |= tma_chunk_bits(mw[i], i - (i / NW) * NW);
        }
        slot_any[slot] = any;
        mbar_arrive_expect_tx(full + slot, (unsigned)__popc(any) * (unsigned)(a.in_rows * COLS * kInElem));
        for (int k = 0; k < a.in_chunks; ++k)
          if ((any >> k) & 1u)
            tma_load_4d(dst + (size_t)k * a.in_rows * COLS * kInElem, &tin, 0, c1, k * a.in_rows - a.in_lo, c3,
                        full + slot);
      } else if constexpr (SHANNA) {
        const int u0 = (b % a.gu) * a.L, vi = b / a.gu;
        const int nl = min(a.L, a.du - u0);  // lines inside the volume (>= 1)
        const unsigned xbytes = (unsigned)(nl * a.img_len) * 8u;
        mbar_arrive_expect_tx(full + slot, kBuf + xbytes);
        for (int k = 0; k < a.in_chunks; ++k)
          tma_load_4d(dst + (size_t)k * a.in_rows * COLS * kInElem, &tin, 0, c1, k * a.in_rows - a.in_lo, c3,
                      full + slot);
        bulk_load(xbuf + (size_t)slot * a.L * a.img_len, a.img + (long long)a.img_len * (u0 + (long long)a.du * vi),
                  xbytes, full + slot);
      } else {
        if constexpr (MASK_OUT) {
          uint32_t keep = 0;  // bit k: output chunk k holds an occupied row of some line
#pragma unroll
          for (int i = 0; i < kTmaMaskWords; ++i)
            keep |= tma_chunk_bits(mw[i], i - (i / NW) * NW);
          slot_any[slot] = keep;
          if (keep == 0) {  // nothing of this bundle is stored: no load, no transform
            mbar_arrive(full + slot);
            return;
          }
        }
        mbar_arrive_expect_tx(full + slot, IN_H ? kBuf / 2 : kBuf);
        for (int k = 0; k < a.in_chunks; ++k)
          tma_load_4d(dst + (size_t)k * a.in_rows * COLS * kInElem, &tin, 0, c1, k * a.in_rows - a.in_lo, c3,
                      full + slot);
      }
    };
    auto store = [&](int slot, int b) {
      const unsigned char* src = base + slot * kBuf + (size_t)a.out_lo * COLS * kOutElem;
      const int c1 = (b % a.gu) * a.L, c3 = b / a.gu;
      uint32_t keep = ~0u;  // MASK_OUT: bit k = chunk k holds an occupied row of some line
      if constexpr (MASK_OUT) keep = slot_any[slot];
      for (int k = 0; k < a.out_chunks; ++k)
        if ((keep >> k) & 1u)
          tma_store_4d(&tout, 0, c1, k * a.out_rows, c3, src + (size_t)k * a.out_rows * COLS * kOutElem);
      bulk_commit();
    };
    int it = 0;
    bool ok = true;
    for (int b = blockIdx.x; b < a.nbundles; b += G, ++it) {
      const int slot = it % NSLOT;
      fetch_masks(b);  // in flight during the wait below
      if (it >= NSLOT) {  // the slot held bundle it - NSLOT: store it first
        if (!mbar_wait(done + slot, (unsigned)((it / NSLOT) - 1) & 1u, abort, a.err)) {
          ok = false;
          break;
        }
        store(slot, b - NSLOT * G);
        bulk_wait_read_all();  // the store has read the buffer
      }
      if (!(a.test_stall && blockIdx.x == 0 && it == 0)) load(slot, b);
    }
    const int issued = it;
    if (ok) {  // the last NSLOT bundles
      for (int k = issued > NSLOT ? issued - NSLOT : 0; k < issued; ++k) {
        const int slot = k % NSLOT;
        if (!mbar_wait(done + slot, (unsigned)(k / NSLOT) & 1u, abort, a.err)) {
          ok = false;
          break;
        }
        store(slot, blockIdx.x + k * G);
      }
    }
    if (!ok) {  // let every load already issued land before the CTA leaves
      for (int k = issued > NSLOT ? issued - NSLOT : 0; k < issued; ++k)
        mbar_wait_bounded(full + k % NSLOT, (unsigned)(k / NSLOT) & 1u);
    }
    bulk_wait_all();
    return;
  }
  // transform threads
  float hs_in = 1.f, hs_out = 1.f;  // FP16 load / store factors (powers of two)
  if constexpr (IN_H) hs_in = 1.f / half_store_scale(a.h_amax, a.h_len);
  if constexpr (OUT_H) hs_out = half_store_scale(a.h_amax, a.h_len_out > 0 ? a.h_len_out : a.h_len);
  float amax = 0.f;  // AMAX: largest output component this thread wrote
  int it = 0;
  for (int b = blockIdx.x; b < a.nbundles; b += G, ++it) {
    const int slot = it % NSLOT;
    const bool ok = mbar_wait(full + slot, (unsigned)(it / NSLOT) & 1u, abort, a.err);
    if (bar_transform_or<NT>(!ok)) return;  // all transform threads leave together
    const uint32_t* lbits = nullptr;
    if constexpr (MASKED) lbits = masks + slot * kTmaMaskWords + ((tid % COLS) / (COLS / a.L)) * NW;
    if constexpr (SHANNA) {  // x .* KFC with the modulation, in place (bmShanna_MATLAB.m:28-54)
      const int col = tid % COLS, l = col / (COLS / a.L);
      const int ui = (b % a.gu) * a.L + l, vi = b / a.gu;
      if (ui < a.du) {  // lines past the volume edge: zero KFC rows, no image values
        const int par = (a.par0 + ui + vi) & 1;
        const float2* const xl = xbuf + (size_t)slot * a.L * a.img_len + l * a.img_len - a.in_lo;
        float2* const sb = reinterpret_cast<float2*>(base + slot * kBuf);
        for (int n = a.in_lo + tid / COLS; n < a.in_lo + a.img_len; n += NT / COLS) {
          float2 p = cmulf_rn(xl[n], sb[n * COLS + col]);
          if ((n + par) & 1) p = make_float2(-p.x, -p.y);
          sb[n * COLS + col] = p;
        }
      }
      bar_transform<NT>();  // every product written before the transform reads it
    }
    // an empty bundle (uniform over the CTA: one slot word)
    const bool empty = (MASKED || MASK_OUT) && slot_any[slot] == 0;
    if (!empty) {
      smem_fft_natural<N1, N2, DIR, COLS, NT, IN_H, OUT_H, MASKED, AMAX>(
          reinterpret_cast<float2*>(base + slot * kBuf), tws, hs_in, hs_out, lbits, &amax);
    } else if constexpr (MASKED) {  // all-zero input: its kept rows are zeros
      const int col = tid % COLS;
      for (int k = a.out_lo + tid / COLS; k < a.out_lo + a.out_rows * a.out_chunks; k += NT / COLS) {
        if constexpr (OUT_H)
          reinterpret_cast<__half2*>(base + slot * kBuf)[k * COLS + col] = __floats2half2_rn(0.f, 0.f);
        else
          reinterpret_cast<float2*>(base + slot * kBuf)[k * COLS + col] = make_float2(0.f, 0.f);
      }
    }
    fence_proxy_async_smem();  // the transform's writes become visible to the store
    mbar_arrive(done + slot);
  }
  if constexpr (AMAX) warp_amax(a.amax, amax);  // the transform threads are whole warps
}

// Host: 4-D tensor map of a coil-fastest volume seen as the line boxes of
// one pass (mlg_fft.cu).  Strides in complex units; box = (2C floats, box_L
// lines, box_rows rows, 1); half: FP16 values (2C halves per cell).
int tma_line_map(CUtensorMap* map, const void* base, int C, int dim_u, long long st_u, int len, long long st_ax,
                 int dim_v, long long st_v, int box_L, int box_rows, bool half = false);
// Whether the TMA passes are enabled (MLG_FFT_TMA=0 turns them off).
bool tma_passes_enabled();
// The timeout test hook (MLG_TEST_WAIT_TIMEOUT=1), read once per process.
bool tma_test_stall();

}  // namespace mlg
