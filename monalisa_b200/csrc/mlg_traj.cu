// Gridding-matrix construction on the device: the semantics of
// src/gridding123/m/bmTraj2SparseMat.m:58-297 (Gu and Gut outputs).
//
// One thread per sample forms the sample's nNb window entries in FP64
// (isotropic distance, Gaussian or Kaiser-Bessel weight, periodic wrap),
// sorts them by cell, sums duplicate cells (MATLAB's sparse() does), drops
// zeros and normalises the row to sum 1 (value * (1/sum), as myDiag*A does).
// Samples outside the grid keep empty rows.  Gu is the compacted row-major
// result (columns ascending within a row); Gut = Gu^T comes from a stable
// radix sort of the entries by cell, which keeps each cell's samples in
// ascending order -- the CSR of MATLAB's transpose.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>

#include "mlg_internal.cuh"

namespace mlg {

// window cells per sample held in registers/local memory: nWin <= 5 in 3-D,
// <= 11 in 2-D (the reference's default is 3)
constexpr int kMaxNb = 128;

struct TrajGeom {
  int imDim;
  int N[3];
  double dK[3];
  double shift[3];   // fix(N/2 + 1)
  double floor_shift;
  int nWin, nRange, lo;  // window offsets lo .. lo + nRange - 1 per dimension
  int nNb;
  int kernel;
  double kp[3];
  double I0a;        // I0(alpha) for Kaiser-Bessel
  double Du;
  // deformation-field matrices (bmImDeformField2sparseMat_ind_weight.m):
  // the input is a displacement per pixel, the position pixel (1-based) +
  // displacement, the window the 2^imDim cells floor(t) + {0, 1}, the weight
  // the bump exp(-1/(1-d^2)) for d < 1; torus keeps displaced pixels that
  // leave the image (wrapped) instead of emptying their rows
  int deform = 0;
  int torus = 0;
};

__device__ double bessel_i0_dev(double x) {
  const double q = 0.25 * x * x;
  double term = 1.0, sum = 1.0;
  for (int k = 1; k < 500; ++k) {
    term *= q / ((double)k * (double)k);
    sum += term;
    if (term < sum * 1e-17) break;
  }
  return sum;
}

static double bessel_i0_host(double x) {
  const double q = 0.25 * x * x;
  double term = 1.0, sum = 1.0;
  for (int k = 1; k < 500; ++k) {
    term *= q / ((double)k * (double)k);
    sum += term;
    if (term < sum * 1e-17) break;
  }
  return sum;
}

// Entries of one sample: returns the count (0 for deleted samples), writes
// sorted unique cells and normalised FP32 values (and, when traw is given,
// the raw FP64 weights the Gn output needs).
__global__ void traj_rows_kernel(TrajGeom g, const double* __restrict__ t, int nPt, int* __restrict__ cnt,
                                 int* __restrict__ tcol, float* __restrict__ tval, double* __restrict__ traw) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < nPt; p += gridDim.x * blockDim.x) {
    double tg[3], tf[3], tr[3];
    bool del = false;
    int q = p;  // pixel coordinates (deformation fields), x fastest
    for (int d = 0; d < 3; ++d) {
      if (d < g.imDim) {
        if (g.deform) {
          // bmImDeformField2sparseMat_ind_weight.m:36-60: t = ndgrid(1:N) + v,
          // deleted when outside [1, N] unless torus
          tg[d] = (double)(q % g.N[d] + 1) + t[(long long)p * g.imDim + d];
          q /= g.N[d];
          del = del || (!g.torus && (!(tg[d] >= 1.0) || !(tg[d] <= (double)g.N[d])));
        } else {
          tg[d] = t[(long long)p * g.imDim + d] / g.dK[d] + g.shift[d];
          del = del || !(tg[d] >= 1.0) || !(tg[d] <= (double)g.N[d]);  // bmTraj2SparseMat.m:117-126
        }
        tf[d] = floor(tg[d] + g.floor_shift);
        tr[d] = tg[d] - tf[d];
      } else {
        tg[d] = tf[d] = tr[d] = 0.0;
      }
    }
    if (del) {
      cnt[p] = 0;
      continue;
    }
    int cols[kMaxNb];
    double ws[kMaxNb];
    int n = 0;
    for (int k = 0; k < g.nNb; ++k) {
      // ndgrid order: x fastest
      int off[3] = {k % g.nRange + g.lo, (k / g.nRange) % g.nRange + g.lo, k / (g.nRange * g.nRange) + g.lo};
      double d2 = 0.0;
      long long lin = 0, stride = 1;
      for (int d = 0; d < g.imDim; ++d) {
        const double dd = tr[d] - off[d];
        d2 += dd * dd;
        // mod(n - 1, N) + 1, 1-based -> 0-based cell coordinate
        long long c = (long long)(tf[d] + off[d]) - 1;
        c %= g.N[d];
        if (c < 0) c += g.N[d];
        lin += c * stride;
        stride *= g.N[d];
      }
      const double dist = sqrt(d2);
      double w;
      if (g.deform) {
        // bump function (ind_weight.m:97-99): exp(-1/(1-d^2)), infinities
        // to 0, zero unless |d| < 1
        w = exp(-1.0 / (1.0 - dist * dist));
        if (isinf(w) || !(fabs(dist) < 1.0)) w = 0.0;
      } else if (g.kernel == MLG_KERNEL_GAUSS) {
        const double z = dist / g.kp[0];
        w = exp(-0.5 * (z * z)) / (sqrt(2 * M_PI) * g.kp[0]);
      } else {
        const double z = dist / g.kp[0];  // tau
        double u = 1 - z * z;
        if (u < 0) u = 0;
        w = bessel_i0_dev(g.kp[1] * sqrt(u)) / g.I0a;
      }
      w *= g.Du;
      // insert sorted by cell, merging duplicates (sparse() sums them)
      int j = n - 1;
      bool merged = false;
      for (int q = 0; q < n; ++q)
        if (cols[q] == (int)lin) {
          ws[q] += w;
          merged = true;
          break;
        }
      if (merged) continue;
      while (j >= 0 && cols[j] > (int)lin) {
        cols[j + 1] = cols[j];
        ws[j + 1] = ws[j];
        --j;
      }
      cols[j + 1] = (int)lin;
      ws[j + 1] = w;
      ++n;
    }
    // drop exact zeros, row sum in ascending column order
    double s = 0.0;
    int m = 0;
    for (int q = 0; q < n; ++q) {
      if (ws[q] == 0.0) continue;
      cols[m] = cols[q];
      ws[m] = ws[q];
      s += ws[q];
      ++m;
    }
    const double inv = s != 0.0 ? 1.0 / s : 0.0;
    for (int q = 0; q < m; ++q) {
      tcol[(long long)p * g.nNb + q] = cols[q];
      tval[(long long)p * g.nNb + q] = (float)(ws[q] * inv);
      if (traw) traw[(long long)p * g.nNb + q] = ws[q];
    }
    cnt[p] = m;
  }
}

__global__ void traj_compact_kernel(int nNb, int nPt, const int* __restrict__ cnt, const int* __restrict__ off,
                                    const int* __restrict__ tcol, const float* __restrict__ tval,
                                    int* __restrict__ col, float* __restrict__ val, int* __restrict__ erow) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < nPt; p += gridDim.x * blockDim.x) {
    const int o = off[p];
    for (int q = 0; q < cnt[p]; ++q) {
      col[o + q] = tcol[(long long)p * nNb + q];
      val[o + q] = tval[(long long)p * nNb + q];
      erow[o + q] = p;
    }
  }
}

__global__ void traj_compact_raw_kernel(int nNb, int nPt, const int* __restrict__ cnt, const int* __restrict__ off,
                                        const double* __restrict__ traw, double* __restrict__ raw) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < nPt; p += gridDim.x * blockDim.x)
    for (int q = 0; q < cnt[p]; ++q) raw[off[p] + q] = traw[(long long)p * nNb + q];
}

// Dn = ve / prod(dK_u), the divisions in dimension order (bmTraj2SparseMat.m:81-106)
__global__ void traj_dn_kernel(const double* __restrict__ ve, int nPt, double dk0, double dk1, double dk2, int imDim,
                               double* __restrict__ Dn) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < nPt; p += gridDim.x * blockDim.x) {
    double v = ve[p] / dk0;
    if (imDim > 1) v /= dk1;
    if (imDim > 2) v /= dk2;
    Dn[p] = v;
  }
}

// Gn (bmTraj2SparseMat.m:245-256): per grid cell, over its entries in
// ascending sample order (the transposed order), w * Dn with zeros dropped;
// count and FP64 row sum ...
__global__ void gn_count_kernel(const int* __restrict__ toff, long long Nu, const int* __restrict__ perm,
                                const int* __restrict__ erow, const double* __restrict__ raw,
                                const double* __restrict__ Dn, int* __restrict__ cnt, double* __restrict__ sum) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < Nu; c += (long long)gridDim.x * blockDim.x) {
    int n = 0;
    double s = 0.0;
    for (int i = toff[c]; i < toff[c + 1]; ++i) {
      const int k = perm[i];
      const double v = raw[k] * Dn[erow[k]];
      if (v != 0.0) {
        ++n;
        s += v;
      }
    }
    cnt[c] = n;
    sum[c] = s;
  }
}

// ... then the row normalised to sum 1 (value * (1/sum), as myDiag * A)
__global__ void gn_fill_kernel(const int* __restrict__ toff, long long Nu, const int* __restrict__ perm,
                               const int* __restrict__ erow, const double* __restrict__ raw,
                               const double* __restrict__ Dn, const double* __restrict__ sum,
                               const uint32_t* __restrict__ row_ptr, int* __restrict__ col, float* __restrict__ val) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < Nu; c += (long long)gridDim.x * blockDim.x) {
    const double inv = sum[c] != 0.0 ? 1.0 / sum[c] : 0.0;
    uint32_t o = row_ptr[c];
    for (int i = toff[c]; i < toff[c + 1]; ++i) {
      const int k = perm[i];
      const double v = raw[k] * Dn[erow[k]];
      if (v != 0.0) {
        col[o] = erow[k];
        val[o] = (float)(v * inv);
        ++o;
      }
    }
  }
}

__global__ void iota_i32_kernel(int* a, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    a[i] = (int)i;
}

__global__ void cell_count_kernel(const int* __restrict__ col, long long n, int* __restrict__ cnt) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    atomicAdd(cnt + col[i], 1);
}

__global__ void transpose_fill_kernel(const int* __restrict__ perm, const int* __restrict__ erow,
                                      const float* __restrict__ val, long long n, int* __restrict__ tcol,
                                      float* __restrict__ tv) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int k = perm[i];
    tcol[i] = erow[k];
    tv[i] = val[k];
  }
}

__global__ void to_u32_kernel(const int* __restrict__ a, uint32_t* __restrict__ b, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    b[i] = (uint32_t)a[i];
}

__global__ void list_long_rows_kernel(const uint32_t* __restrict__ row_ptr, int l_size, int* __restrict__ list,
                                      int* __restrict__ n_long, int* __restrict__ n_nonempty) {
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < l_size; r += (long long)gridDim.x * blockDim.x) {
    const uint32_t len = row_ptr[r + 1] - row_ptr[r];
    if (len > (uint32_t)kLongRow) list[atomicAdd(n_long, 1)] = (int)r;
    if (len > 0) atomicAdd(n_nonempty, 1);
  }
}

static int g1d(long long n) { return (int)std::max<long long>(1, std::min<long long>((n + 255) / 256, 148LL * 32)); }

// Row pointer (uint32) from per-row counts, and the long-row list.
static int finish_csr(Csr& m, int* counts, cudaStream_t s) {
  size_t tmp_bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, counts, counts, m.l_size + 1);
  DevBuf<char> tmp;
  MLG_TRY(tmp.alloc(tmp_bytes, s));
  MLG_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, tmp_bytes, counts, counts, m.l_size + 1, s));
  to_u32_kernel<<<g1d(m.l_size + 1LL), 256, 0, s>>>(counts, m.row_ptr, m.l_size + 1LL);
  MLG_LAUNCHED();
  DevBuf<int> nl;
  MLG_TRY(nl.alloc(2, s));
  MLG_CUDA(cudaMemsetAsync(nl.p, 0, 8, s));
  int* list = nullptr;
  MLG_CUDA(cudaMalloc(&list, sizeof(int) * (size_t)std::max(1, m.l_size)));
  list_long_rows_kernel<<<g1d(m.l_size), 256, 0, s>>>(m.row_ptr, m.l_size, list, nl.p, nl.p + 1);
  MLG_LAUNCHED();
  int h[2];
  MLG_CUDA(cudaMemcpyAsync(h, nl.p, 8, cudaMemcpyDeviceToHost, s));
  MLG_CUDA(cudaStreamSynchronize(s));
  m.long_rows = list;
  m.n_long = h[0];
  m.n_nonempty = h[1];
  MLG_TRY(csr_build_segments(m, s));
  return MLG_OK;
}

static int build_sparsemats(const TrajGeom& g, int nPt, const double* t_host, Csr* Gu, Csr* Gut, cudaStream_t s,
                            const double* ve_host, Csr* Gn);

// src/gridding123/m/bmImDeformField2SparseMat.m:14-146 with the weights of
// bmImDeformField2sparseMat_ind_weight.m: one row per pixel (deleted pixels
// keep empty rows), Gu/Gut row-normalised, Gn = rows of cells with values
// w * Dn normalised per cell (Dn given per pixel; dK = 1 so Dn passes
// through the volume-element scaling unchanged).
int deform2sparsemat(int imDim, const int* N_u, const double* v_host, const double* dn_host, bool torus, Csr* Gu,
                     Csr* Gut, Csr* Gn, cudaStream_t s) {
  TrajGeom g;
  g.imDim = imDim;
  g.deform = 1;
  g.torus = torus ? 1 : 0;
  long long Nu = 1;
  for (int d = 0; d < 3; ++d) {
    g.N[d] = d < imDim ? N_u[d] : 1;
    g.dK[d] = 1.0;
    g.shift[d] = 0.0;
    if (d < imDim) Nu *= g.N[d];
  }
  MLG_CHECK(Nu < (1LL << 31), "image too large");
  g.floor_shift = 0.0;
  g.nWin = 2;
  g.nRange = 2;
  g.lo = 0;
  g.nNb = 1 << imDim;
  g.kernel = -1;
  for (int i = 0; i < 3; ++i) g.kp[i] = 0.0;
  g.I0a = 1.0;
  g.Du = 1.0;
  return build_sparsemats(g, (int)Nu, v_host, Gu, Gut, s, dn_host, Gn);
}

int traj2sparsemat(int imDim, int nPt, const double* t_host, const int* N_u, const double* dK_u, int kernelType,
                   int nWin, const double* kp, Csr* Gu, Csr* Gut, cudaStream_t s, const double* ve_host = nullptr,
                   Csr* Gn = nullptr) {
  MLG_CHECK(!Gn || ve_host, "Gn needs the volume elements ve");
  TrajGeom g;
  g.imDim = imDim;
  g.nWin = nWin;
  g.kernel = kernelType;
  long long Nu = 1;
  g.Du = 1.0;
  for (int d = 0; d < 3; ++d) {
    g.N[d] = d < imDim ? (int)(float)N_u[d] : 1;
    g.dK[d] = d < imDim ? (double)(float)dK_u[d] : 1.0;  // double(single(dK_u))
    g.shift[d] = d < imDim ? std::floor(g.N[d] / 2.0 + 1.0) : 0.0;
    if (d < imDim) {
      Nu *= g.N[d];
      g.Du *= (1.0 / g.dK[d]) / g.N[d];
    }
  }
  MLG_CHECK(Nu < (1LL << 31), "grid too large");
  // bmTraj2SparseMat.m:134-156: even widths use offsets -nWin/2-1 .. nWin/2
  if (nWin % 2 == 0) {
    g.lo = -nWin / 2 - 1;
    g.nRange = nWin + 2;
    g.floor_shift = 0.0;
  } else {
    g.lo = -(nWin / 2);
    g.nRange = nWin;
    g.floor_shift = 0.5;
  }
  g.nNb = g.nRange;
  for (int d = 1; d < imDim; ++d) g.nNb *= g.nRange;
  MLG_CHECK(g.nNb <= kMaxNb, "window of %d cells exceeds %d", g.nNb, kMaxNb);
  for (int i = 0; i < 3; ++i) g.kp[i] = (double)(float)kp[i];  // double(single(kernelParam))
  g.I0a = kernelType == MLG_KERNEL_KAISER ? bessel_i0_host(g.kp[1]) : 1.0;
  return build_sparsemats(g, nPt, t_host, Gu, Gut, s, ve_host, Gn);
}

// Rows of every sample (or pixel), then the CSR outputs: Gu, its transpose
// Gut, and Gn (rows = cells, values w * Dn with Dn = ve / prod(dK),
// normalised per cell).
static int build_sparsemats(const TrajGeom& g, int nPt, const double* t_host, Csr* Gu, Csr* Gut, cudaStream_t s,
                            const double* ve_host, Csr* Gn) {
  const int imDim = g.imDim;
  long long Nu = 1;
  for (int d = 0; d < imDim; ++d) Nu *= g.N[d];
  const long long cap = (long long)nPt * g.nNb;
  MLG_CHECK(cap < (1LL << 31), "nPt * nNb too large");
  DevBuf<double> dt;
  DevBuf<int> cnt, tcol;
  DevBuf<float> tval;
  MLG_TRY(dt.alloc((size_t)imDim * nPt + 1, s));
  MLG_TRY(cnt.alloc((size_t)nPt + 1, s));
  MLG_TRY(tcol.alloc((size_t)cap + 1, s));
  MLG_TRY(tval.alloc((size_t)cap + 1, s));
  MLG_CUDA(cudaMemcpyAsync(dt.p, t_host, sizeof(double) * imDim * nPt, cudaMemcpyHostToDevice, s));
  MLG_CUDA(cudaMemsetAsync(cnt.p + nPt, 0, sizeof(int), s));
  DevBuf<double> traw;
  if (Gn) MLG_TRY(traw.alloc((size_t)cap + 1, s));
  traj_rows_kernel<<<g1d(nPt), 128, 0, s>>>(g, dt.p, nPt, cnt.p, tcol.p, tval.p, Gn ? traw.p : nullptr);
  MLG_LAUNCHED();
  DevBuf<int> off;
  MLG_TRY(off.alloc((size_t)nPt + 1, s));
  size_t tb = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt.p, off.p, nPt + 1);
  DevBuf<char> tmp;
  MLG_TRY(tmp.alloc(tb, s));
  MLG_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, tb, cnt.p, off.p, nPt + 1, s));
  int nnz = 0;
  MLG_CUDA(cudaMemcpyAsync(&nnz, off.p + nPt, sizeof(int), cudaMemcpyDeviceToHost, s));
  MLG_CUDA(cudaStreamSynchronize(s));

  Csr u;
  u.r_size = (int)Nu;
  u.l_size = nPt;
  u.nnz = nnz;
  MLG_CUDA(cudaMalloc(&u.row_ptr, sizeof(uint32_t) * ((size_t)nPt + 1)));
  MLG_CUDA(cudaMalloc(&u.col, sizeof(int) * (size_t)std::max(1, nnz)));
  MLG_CUDA(cudaMalloc(&u.val, sizeof(float) * (size_t)std::max(1, nnz)));
  DevBuf<int> erow;
  MLG_TRY(erow.alloc((size_t)nnz + 1, s));
  traj_compact_kernel<<<g1d(nPt), 256, 0, s>>>(g.nNb, nPt, cnt.p, off.p, tcol.p, tval.p, u.col, u.val, erow.p);
  MLG_LAUNCHED();
  DevBuf<double> raw;
  if (Gn) {
    MLG_TRY(raw.alloc((size_t)nnz + 1, s));
    traj_compact_raw_kernel<<<g1d(nPt), 256, 0, s>>>(g.nNb, nPt, cnt.p, off.p, traw.p, raw.p);
    MLG_LAUNCHED();
  }
  // Gu row pointer: counts -> scan (reuse cnt with a trailing zero)
  MLG_TRY(finish_csr(u, cnt.p, s));

  if (Gut || Gn) {
    // entries grouped by cell, samples ascending within a cell (stable sort)
    DevBuf<int> keys_out, perm_in, perm_out, ccnt;
    MLG_TRY(keys_out.alloc((size_t)nnz + 1, s));
    MLG_TRY(perm_in.alloc((size_t)nnz + 1, s));
    MLG_TRY(perm_out.alloc((size_t)nnz + 1, s));
    MLG_TRY(ccnt.alloc((size_t)Nu + 1, s));
    iota_i32_kernel<<<g1d(nnz), 256, 0, s>>>(perm_in.p, nnz);
    MLG_LAUNCHED();
    int end_bit = 1;
    while ((1LL << end_bit) < Nu) ++end_bit;
    size_t sb = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, sb, u.col, keys_out.p, perm_in.p, perm_out.p, nnz, 0, end_bit);
    DevBuf<char> stmp;
    MLG_TRY(stmp.alloc(sb, s));
    MLG_CUDA(cub::DeviceRadixSort::SortPairs(stmp.p, sb, u.col, keys_out.p, perm_in.p, perm_out.p, nnz, 0, end_bit, s));
    MLG_CUDA(cudaMemsetAsync(ccnt.p, 0, sizeof(int) * ((size_t)Nu + 1), s));
    cell_count_kernel<<<g1d(nnz), 256, 0, s>>>(u.col, nnz, ccnt.p);
    MLG_LAUNCHED();
    if (Gut) {
      Csr v;
      v.r_size = nPt;
      v.l_size = (int)Nu;
      v.nnz = nnz;
      MLG_CUDA(cudaMalloc(&v.row_ptr, sizeof(uint32_t) * ((size_t)Nu + 1)));
      MLG_CUDA(cudaMalloc(&v.col, sizeof(int) * (size_t)std::max(1, nnz)));
      MLG_CUDA(cudaMalloc(&v.val, sizeof(float) * (size_t)std::max(1, nnz)));
      transpose_fill_kernel<<<g1d(nnz), 256, 0, s>>>(perm_out.p, erow.p, u.val, nnz, v.col, v.val);
      MLG_LAUNCHED();
      MLG_TRY(finish_csr(v, ccnt.p, s));  // leaves the cell offsets in ccnt
      *Gut = v;
    } else {
      size_t tb2 = 0;
      cub::DeviceScan::ExclusiveSum(nullptr, tb2, ccnt.p, ccnt.p, Nu + 1);
      DevBuf<char> tmp2;
      MLG_TRY(tmp2.alloc(tb2, s));
      MLG_CUDA(cub::DeviceScan::ExclusiveSum(tmp2.p, tb2, ccnt.p, ccnt.p, Nu + 1, s));
    }
    if (Gn) {
      DevBuf<double> dve, Dn, gsum;
      DevBuf<int> gcnt;
      MLG_TRY(dve.alloc((size_t)nPt, s));
      MLG_TRY(Dn.alloc((size_t)nPt, s));
      MLG_TRY(gsum.alloc((size_t)Nu, s));
      MLG_TRY(gcnt.alloc((size_t)Nu + 1, s));
      MLG_CUDA(cudaMemcpyAsync(dve.p, ve_host, sizeof(double) * nPt, cudaMemcpyHostToDevice, s));
      traj_dn_kernel<<<g1d(nPt), 256, 0, s>>>(dve.p, nPt, g.dK[0], g.dK[1], g.dK[2], imDim, Dn.p);
      MLG_LAUNCHED();
      MLG_CUDA(cudaMemsetAsync(gcnt.p + Nu, 0, sizeof(int), s));
      gn_count_kernel<<<g1d(Nu), 256, 0, s>>>(ccnt.p, Nu, perm_out.p, erow.p, raw.p, Dn.p, gcnt.p, gsum.p);
      MLG_LAUNCHED();
      Csr w;
      w.r_size = nPt;
      w.l_size = (int)Nu;
      MLG_CUDA(cudaMalloc(&w.row_ptr, sizeof(uint32_t) * ((size_t)Nu + 1)));
      const int st = finish_csr(w, gcnt.p, s);
      uint32_t nnz_n = 0;
      if (st == MLG_OK) {
        MLG_CUDA(cudaMemcpyAsync(&nnz_n, w.row_ptr + Nu, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        MLG_CUDA(cudaStreamSynchronize(s));
      }
      w.nnz = nnz_n;
      if (st != MLG_OK || cudaMalloc(&w.col, sizeof(int) * (size_t)std::max<uint32_t>(1, nnz_n)) != cudaSuccess ||
          cudaMalloc(&w.val, sizeof(float) * (size_t)std::max<uint32_t>(1, nnz_n)) != cudaSuccess) {
        cudaGetLastError();
        csr_free(w);
        if (Gu) *Gu = u;  // the caller frees what it asked for
        else csr_free(u);
        return st != MLG_OK ? st : fail(MLG_ERR_OOM, "Gn: device allocation failed");
      }
      gn_fill_kernel<<<g1d(Nu), 256, 0, s>>>(ccnt.p, Nu, perm_out.p, erow.p, raw.p, Dn.p, gsum.p, w.row_ptr, w.col,
                                             w.val);
      MLG_LAUNCHED();
      *Gn = w;
    }
  }
  if (Gu) {
    *Gu = u;
  } else {
    csr_free(u);
  }
  MLG_CUDA(cudaStreamSynchronize(s));
  return MLG_OK;
}

}  // namespace mlg

extern "C" int mlg_traj2sparsemat3(int imDim, int nPt, const double* t, const double* ve, const int* N_u,
                                   const double* dK_u, int kernelType, int nWin, const double* kernelParam,
                                   mlg_matrix_t* Gn, mlg_matrix_t* Gu, mlg_matrix_t* Gut) {
  mlg::NvtxRange range("bmTraj2SparseMat (Gn, Gu, Gut)");
  MLG_CHECK(imDim >= 1 && imDim <= 3 && nPt >= 1 && t && N_u && dK_u && kernelParam, "invalid argument");
  MLG_CHECK(kernelType == MLG_KERNEL_GAUSS || kernelType == MLG_KERNEL_KAISER, "unknown kernel type");
  MLG_CHECK(nWin >= 1, "nWin must be >= 1");
  MLG_CHECK(Gn || Gu || Gut, "no output requested");
  MLG_CHECK(!Gn || ve, "Gn needs the volume elements ve");
  for (int d = 0; d < imDim; ++d) MLG_CHECK(N_u[d] >= 1 && dK_u[d] > 0, "invalid N_u / dK_u");
  MLG_TRY(mlg::ensure_device());
  if (Gn) *Gn = nullptr;
  if (Gu) *Gu = nullptr;
  if (Gut) *Gut = nullptr;
  mlg::Csr u, v, w;
  int st = mlg::traj2sparsemat(imDim, nPt, t, N_u, dK_u, kernelType, nWin, kernelParam, Gu ? &u : nullptr,
                               Gut ? &v : nullptr, nullptr, ve, Gn ? &w : nullptr);
  if (st != MLG_OK) {
    mlg::csr_free(u);
    mlg::csr_free(v);
    mlg::csr_free(w);
    return st;
  }
  int dev = 0;
  cudaGetDevice(&dev);
  mlg_matrix_t* outs[3] = {Gn, Gu, Gut};
  mlg::Csr* csrs[3] = {&w, &u, &v};
  for (int i = 0; i < 3; ++i)
    if (outs[i]) {
      *outs[i] = new mlg_matrix_s();
      (*outs[i])->csr = *csrs[i];
      (*outs[i])->device = dev;
    }
  return MLG_OK;
}

extern "C" int mlg_traj2sparsemat(int imDim, int nPt, const double* t, const double* ve, const int* N_u,
                                  const double* dK_u, int kernelType, int nWin, const double* kernelParam,
                                  mlg_matrix_t* Gu, mlg_matrix_t* Gut) {
  // Gu / Gut are row-normalised: the volume elements cancel (bmTraj2SparseMat.m:271-281)
  MLG_CHECK(Gu || Gut, "no output requested");
  return mlg_traj2sparsemat3(imDim, nPt, t, ve, N_u, dK_u, kernelType, nWin, kernelParam, nullptr, Gu, Gut);
}

extern "C" int mlg_deform2sparsemat(int imDim, const int* N_u, const double* v, const double* Dn, int torus_flag,
                                    mlg_matrix_t* Gn, mlg_matrix_t* Gu, mlg_matrix_t* Gut) {
  MLG_CHECK(imDim >= 1 && imDim <= 3 && N_u && v, "invalid argument");
  MLG_CHECK(Gn || Gu || Gut, "no output requested");
  MLG_CHECK(!Gn || Dn, "Gn needs Dn");
  for (int d = 0; d < imDim; ++d) MLG_CHECK(N_u[d] >= 1, "invalid N_u");
  MLG_TRY(mlg::ensure_device());
  if (Gn) *Gn = nullptr;
  if (Gu) *Gu = nullptr;
  if (Gut) *Gut = nullptr;
  mlg::Csr u, t, w;
  const int st = mlg::deform2sparsemat(imDim, N_u, v, Dn, torus_flag != 0, Gu ? &u : nullptr, Gut ? &t : nullptr,
                                       Gn ? &w : nullptr, nullptr);
  if (st != MLG_OK) {
    mlg::csr_free(u);
    mlg::csr_free(t);
    mlg::csr_free(w);
    return st;
  }
  int dev = 0;
  cudaGetDevice(&dev);
  mlg_matrix_t* outs[3] = {Gn, Gu, Gut};
  mlg::Csr* csrs[3] = {&w, &u, &t};
  for (int i = 0; i < 3; ++i)
    if (outs[i]) {
      *outs[i] = new mlg_matrix_s();
      (*outs[i])->csr = *csrs[i];
      (*outs[i])->device = dev;
    }
  return MLG_OK;
}
