// Error plumbing, device selection, stream-ordered allocation, CSR upload
// from the jump format, and the deterministic FP64 reduction used by the
// solvers.
#include <cub/device/device_radix_sort.cuh>

#include <cstdarg>
#include <cstring>
#include <mutex>
#include <vector>

#include "mlg_internal.cuh"

namespace mlg {

std::atomic<long long> g_launches{0};
static thread_local std::string t_last_error;
static thread_local int t_device = -1;

void set_error(const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  t_last_error = buf;
}

int fail(int status, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  t_last_error = buf;
  return status;
}

int ensure_device() {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    cudaGetLastError();
    return fail(MLG_ERR_NO_DEVICE, "no CUDA device visible (%s)", cudaGetErrorString(e));
  }
  if (t_device >= 0) MLG_CUDA(cudaSetDevice(t_device));
  int dev = 0;
  MLG_CUDA(cudaGetDevice(&dev));
  static std::mutex mu;
  static std::vector<bool> pool_ready;
  std::lock_guard<std::mutex> lk(mu);
  if ((int)pool_ready.size() <= dev) pool_ready.resize(dev + 1, false);
  if (!pool_ready[dev]) {
    // Keep freed blocks in the default pool: repeated per-call work buffers
    // then cost no cudaMalloc after the first call.
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
      uint64_t thr = UINT64_MAX;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    cudaGetLastError();
    pool_ready[dev] = true;
  }
  return MLG_OK;
}

int dev_alloc(void** p, size_t bytes, cudaStream_t s) {
  *p = nullptr;
  cudaError_t e = cudaMallocAsync(p, bytes, s);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return fail(e == cudaErrorMemoryAllocation ? MLG_ERR_OOM : MLG_ERR_CUDA,
                "device allocation of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
  }
  return MLG_OK;
}

void dev_free(void* p, cudaStream_t s) {
  if (p) cudaFreeAsync(p, s);
}

void csr_free(Csr& c) {
  cudaFree(c.row_ptr);
  cudaFree(c.col);
  cudaFree(c.val);
  cudaFree(c.long_rows);
  cudaFree(c.seg_lo);
  cudaFree(c.seg_hi);
  cudaFree(c.long_seg0);
  cudaFree(c.nz_rows);
  cudaFree(c.nz_mask);
  cudaFree(c.ord_rows);
  cudaFree(c.ord_bounds);
  cudaFree(c.val_h);
  cudaFree(c.ord_rec);
  c = Csr();
}

// bit r set <=> row r non-empty; one thread per 32-row word
__global__ void nz_mask_kernel(const uint32_t* __restrict__ row_ptr, int l_size, uint32_t* __restrict__ mask,
                               int* __restrict__ word_count) {
  const int nw = (l_size + 31) / 32;
  for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < nw; w += gridDim.x * blockDim.x) {
    uint32_t m = 0;
    for (int b = 0; b < 32; ++b) {
      const long long r = (long long)w * 32 + b;
      if (r < l_size && row_ptr[r + 1] > row_ptr[r]) m |= 1u << b;
    }
    mask[w] = m;
    word_count[w] = __popc(m);
  }
}

__global__ void nz_rows_kernel(const uint32_t* __restrict__ mask, const int* __restrict__ word_off, int nw,
                               int* __restrict__ rows) {
  for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < nw; w += gridDim.x * blockDim.x) {
    uint32_t m = mask[w];
    int o = word_off[w];
    while (m) {
      const int b = __ffs(m) - 1;
      rows[o++] = w * 32 + b;
      m &= m - 1;
    }
  }
}

// brick key of row i (rows[i], or i): its cell (the row itself, or the
// column of its first entry when by_first_col; empty rows sort last)
// split: rows with more than kMidRow entries get the key's top bit (they
// sort after the others, each group in brick order) and are counted in
// n_mid.
__global__ void order_keys_kernel(const uint32_t* __restrict__ row_ptr, const int* __restrict__ col,
                                  const int* __restrict__ rows, int n, int by_first_col, int N0, int N1, int nbx,
                                  int nby, bool split, uint32_t* __restrict__ keys, int* __restrict__ vals,
                                  int* __restrict__ n_mid) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int r = rows ? rows[i] : i;
    vals[i] = r;
    long long cell = r;
    if (by_first_col) {
      const uint32_t b = row_ptr[r];
      if (b == row_ptr[r + 1]) {
        keys[i] = 0xffffffffu;
        continue;
      }
      cell = col[b];
    }
    const long long x = cell % N0, t = cell / N0, y = t % N1, z = t / N1;
    const long long brick = (x >> 3) + nbx * ((y >> 3) + (long long)nby * (z >> 3));
    uint32_t key = (uint32_t)(brick * 512 + (x & 7) + 8 * ((y & 7) + 8 * (z & 7)));
    if (split && row_ptr[r + 1] - row_ptr[r] > (uint32_t)kMidRow) {
      key |= 0x80000000u;
      atomicAdd(n_mid, 1);
    }
    keys[i] = key;
  }
}

__global__ void order_bounds_kernel(const uint32_t* __restrict__ row_ptr, const int* __restrict__ rows, int n,
                                    uint2* __restrict__ bounds) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int r = rows[i];
    bounds[i] = make_uint2(row_ptr[r], row_ptr[r + 1]);
  }
}

int csr_build_order(Csr& c, const int* N, bool nonempty, cudaStream_t s) {
  if (c.ord_rows) return MLG_OK;
  MLG_CHECK(!nonempty || c.nz_rows, "ordered non-empty rows need the row list");
  const int n = nonempty ? c.n_nonempty : c.l_size;
  const int nbx = (N[0] + 7) / 8, nby = (N[1] + 7) / 8, nbz = (N[2] + 7) / 8;
  const double nkeys = (double)nbx * nby * nbz * 512.0;
  if (nkeys >= 4294967295.0) return MLG_OK;  // keys would not fit: keep row order
  // non-empty rows: short rows first when the keys leave the top bit free
  const bool split = nonempty && nkeys < 2147483648.0;
  DevBuf<uint32_t> keys, keys_out;
  DevBuf<int> vals, n_mid;
  MLG_TRY(keys.alloc((size_t)std::max(1, n), s));
  MLG_TRY(keys_out.alloc((size_t)std::max(1, n), s));
  MLG_TRY(vals.alloc((size_t)std::max(1, n), s));
  MLG_TRY(n_mid.alloc(1, s));
  MLG_CUDA(cudaMemsetAsync(n_mid.p, 0, sizeof(int), s));
  const int g = std::max(1, std::min(4096, (n + 255) / 256));
  order_keys_kernel<<<g, 256, 0, s>>>(c.row_ptr, c.col, nonempty ? c.nz_rows : nullptr, n, nonempty ? 0 : 1, N[0],
                                      N[1], nbx, nby, split, keys.p, vals.p, n_mid.p);
  count_launch();
  int h_mid = 0;
  MLG_CUDA(cudaMemcpyAsync(&h_mid, n_mid.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  int* ord = nullptr;
  uint2* bounds = nullptr;
  MLG_CUDA(cudaMalloc(&ord, sizeof(int) * (size_t)std::max(1, n)));
  if (cudaMalloc(&bounds, sizeof(uint2) * (size_t)std::max(1, n)) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(ord);
    return fail(MLG_ERR_OOM, "row order: device allocation failed");
  }
  size_t tb = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tb, keys.p, keys_out.p, vals.p, ord, n);
  DevBuf<char> tmp;
  int st = tmp.alloc(std::max<size_t>(tb, 1), s);
  if (st == MLG_OK && cub::DeviceRadixSort::SortPairs(tmp.p, tb, keys.p, keys_out.p, vals.p, ord, n, 0, 32, s) !=
                          cudaSuccess)
    st = fail(MLG_ERR_CUDA, "row order: sort failed");
  if (st != MLG_OK) {
    cudaFree(ord);
    cudaFree(bounds);
    return st;
  }
  order_bounds_kernel<<<g, 256, 0, s>>>(c.row_ptr, ord, n, bounds);
  count_launch();
  MLG_CUDA(cudaStreamSynchronize(s));
  c.ord_rows = ord;
  c.ord_bounds = bounds;
  c.n_ord = n;
  c.ord_nonempty = nonempty;
  c.ord_short = split ? n - h_mid : -1;
  return MLG_OK;
}

int csr_build_nonempty(Csr& c, cudaStream_t s) {
  if (c.nz_mask) return MLG_OK;
  const int nw = (c.l_size + 31) / 32;
  int *cnt = nullptr, *off = nullptr;
  MLG_CUDA(cudaMalloc(&c.nz_mask, sizeof(uint32_t) * (size_t)std::max(1, nw)));
  MLG_CUDA(cudaMalloc(&cnt, sizeof(int) * (size_t)(nw + 1)));
  MLG_CUDA(cudaMalloc(&off, sizeof(int) * (size_t)(nw + 1)));
  const int g = std::max(1, std::min(4096, (nw + 255) / 256));
  nz_mask_kernel<<<g, 256, 0, s>>>(c.row_ptr, c.l_size, c.nz_mask, cnt);
  count_launch();
  // exclusive scan of the word counts on the host (nw is small: l_size/32)
  std::vector<int> h(nw + 1, 0);
  MLG_CUDA(cudaMemcpyAsync(h.data(), cnt, sizeof(int) * nw, cudaMemcpyDeviceToHost, s));
  MLG_CUDA(cudaStreamSynchronize(s));
  int run = 0;
  for (int w = 0; w < nw; ++w) {
    const int v = h[w];
    h[w] = run;
    run += v;
  }
  h[nw] = run;
  c.n_nonempty = run;
  MLG_CUDA(cudaMemcpyAsync(off, h.data(), sizeof(int) * (nw + 1), cudaMemcpyHostToDevice, s));
  MLG_CUDA(cudaMalloc(&c.nz_rows, sizeof(int) * (size_t)std::max(1, run)));
  nz_rows_kernel<<<g, 256, 0, s>>>(c.nz_mask, off, nw, c.nz_rows);
  count_launch();
  MLG_CUDA(cudaStreamSynchronize(s));
  cudaFree(cnt);
  cudaFree(off);
  return MLG_OK;
}

__global__ void long_bounds_kernel(const uint32_t* __restrict__ row_ptr, const int* __restrict__ rows, int n,
                                   uint32_t* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    out[2 * i] = row_ptr[rows[i]];
    out[2 * i + 1] = row_ptr[rows[i] + 1];
  }
}

int csr_build_segments(Csr& c, cudaStream_t s) {
  c.n_seg = 0;
  if (c.n_long == 0) return MLG_OK;
  uint32_t* d_b = nullptr;
  MLG_CUDA(cudaMalloc(&d_b, sizeof(uint32_t) * 2 * (size_t)c.n_long));
  long_bounds_kernel<<<(c.n_long + 255) / 256, 256, 0, s>>>(c.row_ptr, c.long_rows, c.n_long, d_b);
  count_launch();
  std::vector<uint32_t> b(2 * (size_t)c.n_long);
  cudaError_t e = cudaMemcpyAsync(b.data(), d_b, sizeof(uint32_t) * b.size(), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(d_b);
  if (e != cudaSuccess) return fail(MLG_ERR_CUDA, "segment bounds: %s", cudaGetErrorString(e));
  std::vector<uint32_t> lo, hi;
  std::vector<int> seg0(c.n_long + 1);
  for (int j = 0; j < c.n_long; ++j) {
    seg0[j] = (int)lo.size();
    for (uint32_t a = b[2 * j]; a < b[2 * j + 1]; a += kSegLen) {
      lo.push_back(a);
      hi.push_back(std::min<uint32_t>(a + kSegLen, b[2 * j + 1]));
    }
  }
  seg0[c.n_long] = (int)lo.size();
  c.n_seg = (int)lo.size();
  MLG_CUDA(cudaMalloc(&c.seg_lo, sizeof(uint32_t) * lo.size()));
  MLG_CUDA(cudaMalloc(&c.seg_hi, sizeof(uint32_t) * hi.size()));
  MLG_CUDA(cudaMalloc(&c.long_seg0, sizeof(int) * seg0.size()));
  MLG_CUDA(cudaMemcpyAsync(c.seg_lo, lo.data(), sizeof(uint32_t) * lo.size(), cudaMemcpyHostToDevice, s));
  MLG_CUDA(cudaMemcpyAsync(c.seg_hi, hi.data(), sizeof(uint32_t) * hi.size(), cudaMemcpyHostToDevice, s));
  MLG_CUDA(cudaMemcpyAsync(c.long_seg0, seg0.data(), sizeof(int) * seg0.size(), cudaMemcpyHostToDevice, s));
  MLG_CUDA(cudaStreamSynchronize(s));
  return MLG_OK;
}

// Decodes the jump format on the host (one pass, 64-bit running indices,
// every index range-checked), then uploads.  bmSparseMat.m:135-166 defines
// the format: r_jump/l_jump hold deltas whose first entry is absolute.
int csr_from_jump(int r_size, const int* r_jump, const int* r_nJump, const float* m_val, int l_size,
                  const int* l_jump, int l_nJump, Csr& out, cudaStream_t s, int nBlock, const int* block_length,
                  const int* l_block_start, const long long* m_block_start) {
  MLG_CHECK(r_size > 0 && l_size > 0, "matrix sizes must be positive (r_size=%d l_size=%d)", r_size, l_size);
  MLG_CHECK(l_nJump >= 0 && r_nJump != nullptr, "r_nJump missing");
  MLG_CHECK(l_jump != nullptr || l_nJump == l_size,
            "without l_jump the matrix must store every row (l_nJump=%d, l_size=%d)", l_nJump, l_size);
  long long nnz = 0;
  for (int i = 0; i < l_nJump; ++i) {
    MLG_CHECK(r_nJump[i] >= 0, "negative r_nJump at row %d", i);
    nnz += r_nJump[i];
  }
  MLG_CHECK(nnz < (1LL << 32) - 1, "nnz=%lld exceeds the 32-bit row pointer", nnz);
  MLG_CHECK(nnz == 0 || (r_jump && m_val), "r_jump / m_val missing");

  // block starts: stored rows and entries where the running sums restart
  // (one block: row 0 and entry 0); the blocks must tile the stored rows and
  // m_block_start must count the entries before each block
  std::vector<char> row_start((size_t)l_nJump + 1, 0), ent_start((size_t)nnz + 1, 0);
  row_start[0] = ent_start[0] = 1;
  if (nBlock > 0) {
    MLG_CHECK(block_length && l_block_start && m_block_start, "block arrays missing (nBlock=%d)", nBlock);
    long long next_row = 0, entries = 0;
    int ri = 0;
    for (int b = 0; b < nBlock; ++b) {
      MLG_CHECK(l_block_start[b] == next_row && block_length[b] >= 1 &&
                    (long long)l_block_start[b] + block_length[b] <= l_nJump,
                "block %d: l_block_start=%d / block_length=%d do not tile the stored rows", b, l_block_start[b],
                block_length[b]);
      for (; ri < l_block_start[b]; ++ri) entries += r_nJump[ri];
      MLG_CHECK(m_block_start[b] == entries, "block %d: m_block_start=%lld, expected %lld", b, m_block_start[b],
                entries);
      row_start[(size_t)l_block_start[b]] = 1;
      ent_start[(size_t)entries] = 1;
      next_row = (long long)l_block_start[b] + block_length[b];
    }
    MLG_CHECK(next_row == l_nJump, "blocks cover %lld of %d stored rows", next_row, l_nJump);
  }

  std::vector<uint32_t> row_ptr((size_t)l_size + 1, 0);
  long long row = -1;
  for (int i = 0; i < l_nJump; ++i) {
    // l_jump holds row deltas, absolute 0-based at a block's first row
    long long r = l_jump ? (row_start[i] ? (long long)l_jump[i] : row + l_jump[i]) : i;
    MLG_CHECK(r > row && r < l_size, "row index %lld out of order or range at stored row %d", r, i);
    row = r;
    row_ptr[(size_t)r + 1] = (uint32_t)r_nJump[i];
  }
  for (int r = 0; r < l_size; ++r) row_ptr[(size_t)r + 1] += row_ptr[r];

  std::vector<int> col((size_t)nnz);
  long long c = 0;
  for (long long e = 0; e < nnz; ++e) {
    c = ent_start[(size_t)e] ? (long long)r_jump[e] : c + r_jump[e];
    MLG_CHECK(c >= 0 && c < r_size, "column index %lld out of range [0,%d) at entry %lld", c, r_size, e);
    col[(size_t)e] = (int)c;
  }

  Csr m;
  m.r_size = r_size;
  m.l_size = l_size;
  m.nnz = nnz;
  cudaError_t e1 = cudaMalloc(&m.row_ptr, sizeof(uint32_t) * ((size_t)l_size + 1));
  cudaError_t e2 = cudaMalloc(&m.col, sizeof(int) * (size_t)(nnz ? nnz : 1));
  cudaError_t e3 = cudaMalloc(&m.val, sizeof(float) * (size_t)(nnz ? nnz : 1));
  if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess) {
    cudaGetLastError();
    csr_free(m);
    return fail(MLG_ERR_OOM, "matrix upload: device allocation failed (nnz=%lld)", nnz);
  }
  MLG_CUDA(cudaMemcpyAsync(m.row_ptr, row_ptr.data(), sizeof(uint32_t) * row_ptr.size(), cudaMemcpyHostToDevice, s));
  if (nnz) {
    MLG_CUDA(cudaMemcpyAsync(m.col, col.data(), sizeof(int) * (size_t)nnz, cudaMemcpyHostToDevice, s));
    MLG_CUDA(cudaMemcpyAsync(m.val, m_val, sizeof(float) * (size_t)nnz, cudaMemcpyHostToDevice, s));
  }
  std::vector<int> longs;
  int nonempty = 0;
  for (int r = 0; r < l_size; ++r) {
    uint32_t len = row_ptr[(size_t)r + 1] - row_ptr[r];
    nonempty += len > 0;
    if (len > (uint32_t)kLongRow) longs.push_back(r);
  }
  m.n_long = (int)longs.size();
  m.n_nonempty = nonempty;
  if (!longs.empty()) {
    MLG_CUDA(cudaMalloc(&m.long_rows, sizeof(int) * longs.size()));
    MLG_CUDA(cudaMemcpyAsync(m.long_rows, longs.data(), sizeof(int) * longs.size(), cudaMemcpyHostToDevice, s));
  }
  MLG_CUDA(cudaStreamSynchronize(s));  // host vectors go out of scope
  {
    const int st = csr_build_segments(m, s);
    if (st != MLG_OK) {
      csr_free(m);
      return st;
    }
  }
  out = m;
  return MLG_OK;
}

// ---- deterministic reduction ---------------------------------------------
__global__ void reduce_partials_kernel(const double* __restrict__ partial, int n, double* out) {
  // One CTA; fixed per-thread strided order, fixed tree: bitwise
  // reproducible for a given n.
  __shared__ double sh[256];
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) acc += partial[i];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = sh[0];
}

int reduce_partials(const double* partial, int n, double* out, cudaStream_t s) {
  reduce_partials_kernel<<<1, 256, 0, s>>>(partial, n, out);
  MLG_LAUNCHED();
  return MLG_OK;
}

}  // namespace mlg

// ---- C ABI: library ---------------------------------------------------------
extern "C" {

int mlg_version(void) { return 10000; }

const char* mlg_status_string(int status) {
  switch (status) {
    case MLG_OK: return "ok";
    case MLG_ERR_ARG: return "invalid argument";
    case MLG_ERR_OOM: return "out of device memory";
    case MLG_ERR_CUDA: return "CUDA error";
    case MLG_ERR_TIMEOUT: return "timeout";
    case MLG_ERR_STATE: return "invalid state";
    case MLG_ERR_UNSUPPORTED: return "unsupported";
    case MLG_ERR_NO_DEVICE: return "no CUDA device";
    default: return "unknown status";
  }
}

const char* mlg_last_error(void) { return mlg::t_last_error.c_str(); }

int mlg_set_device(int device) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
    cudaGetLastError();
    return mlg::fail(MLG_ERR_ARG, "device %d not available (%d visible)", device, n);
  }
  mlg::t_device = device;
  MLG_CUDA(cudaSetDevice(device));
  return MLG_OK;
}

long long mlg_kernel_launch_count(void) { return mlg::g_launches.load(); }

}  // extern "C"
