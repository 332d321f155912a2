// Setup-time computations on the device: the deapodisation K of
// src/fourier123/prep_function/bmK.m:6-156 and the volume elements of full
// radial trajectories (geom3/bmVolumeElement_full_radial3.m,
// geom2/bmVolumeElement_voronoi_full_radial2.m).
//
// Deapodisation: the same separable FP64 passes and summation order as the
// host computation in mlg_deapod.cpp (tables from deapod_tables), with
// explicit round-to-nearest multiplies and adds, so the two agree bit for
// bit.  Volume elements: FP64, the restatement's steps (line directions,
// projected radii, 1-D Voronoi lengths along the lines in the first line's
// order, radial or angular-Voronoi area factors, the centre sample).
#include <cub/device/device_radix_sort.cuh>

#include <cmath>

#include "mlg_internal.cuh"

namespace mlg {
namespace {

constexpr int kThreads = 256;

int grid_of(long long n) { return (int)std::max<long long>(1, std::min<long long>((n + kThreads - 1) / kThreads, 148LL * 32)); }

// ---- deapodisation -----------------------------------------------------------
struct DeapodDims {
  int N0, N1, N2, S, Sy, Sz, imDim;
};

// A2[az][jy][jx] = sum_ay cy[jy][ay] * (sum_ax w[az][ay][ax] * cx[jx][ax]):
// the host's passes x then y, same order per sum
__global__ void deapod_xy_kernel(DeapodDims D, const double* __restrict__ w, const double* __restrict__ cx,
                                 const double* __restrict__ cy, double* __restrict__ A2) {
  const long long total = (long long)D.Sz * D.N1 * D.N0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int jx = (int)(i % D.N0);
    const long long q = i / D.N0;
    const int jy = (int)(q % D.N1), az = (int)(q / D.N1);
    double acc2 = 0.0;
    for (int ay = 0; ay < D.Sy; ++ay) {
      double acc1 = 0.0;
      for (int ax = 0; ax < D.S; ++ax)
        acc1 = __dadd_rn(acc1, __dmul_rn(w[((long long)az * D.Sy + ay) * D.S + ax], cx[(long long)jx * D.S + ax]));
      acc2 = __dadd_rn(acc2, __dmul_rn(acc1, D.imDim > 1 ? cy[(long long)jy * D.S + ay] : 1.0));
    }
    A2[i] = acc2;
  }
}

__device__ __forceinline__ double deapod_z(const DeapodDims& D, const double* A2, const double* cz, int jz, int jy,
                                           int jx) {
  double acc = 0.0;
  for (int az = 0; az < D.Sz; ++az)
    acc = __dadd_rn(acc, __dmul_rn(A2[((long long)az * D.N1 + jy) * D.N0 + jx], D.imDim > 2 ? cz[(long long)jz * D.S + az] : 1.0));
  return fabs(acc);
}

// the maximum of |Re K| (non-negative doubles order as their bit patterns)
__global__ void deapod_max_kernel(DeapodDims D, const double* __restrict__ A2, const double* __restrict__ cz,
                                  unsigned long long* __restrict__ kmax) {
  const long long total = (long long)D.N0 * D.N1 * D.N2;
  unsigned long long m = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int jx = (int)(i % D.N0);
    const long long q = i / D.N0;
    const unsigned long long b = (unsigned long long)__double_as_longlong(deapod_z(D, A2, cz, (int)(q / D.N1), (int)(q % D.N1), jx));
    m = b > m ? b : m;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long t = __shfl_xor_sync(0xffffffffu, m, o);
    m = t > m ? t : m;
  }
  if ((threadIdx.x & 31) == 0) atomicMax(kmax, m);
}

// K = min(1 / (|Re K| / max), K_max), as bmK.m:148-151
__global__ void deapod_final_kernel(DeapodDims D, const double* __restrict__ A2, const double* __restrict__ cz,
                                    const unsigned long long* __restrict__ kmax_bits, double K_max,
                                    float* __restrict__ K) {
  const double kmax = __longlong_as_double((long long)*kmax_bits);
  const long long total = (long long)D.N0 * D.N1 * D.N2;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int jx = (int)(i % D.N0);
    const long long q = i / D.N0;
    const double v = deapod_z(D, A2, cz, (int)(q / D.N1), (int)(q % D.N1), jx);
    const double k = __ddiv_rn(1.0, __ddiv_rn(v, kmax));
    K[i] = (float)(k < K_max ? k : K_max);
  }
}

// ---- volume elements -----------------------------------------------------------
// t [imDim][nPt] (row-major (imDim, nPt)); line l holds samples l*N .. l*N+N-1.

// e[d][l]: mean over samples n >= ceil(N/2) - 1 of the unit vector from the
// line's first sample, samples at zero distance left out (nanmean)
__global__ void ve_direction_kernel(const double* __restrict__ t, int imDim, int nPt, int N, int nLine,
                                    double* __restrict__ e) {
  for (int l = blockIdx.x * blockDim.x + threadIdx.x; l < nLine; l += gridDim.x * blockDim.x) {
    double s[3] = {0.0, 0.0, 0.0};
    int cnt = 0;
    const long long p0 = (long long)l * N;
    for (int n = (N + 1) / 2 - 1; n < N; ++n) {
      double v[3], r2 = 0.0;
      for (int d = 0; d < imDim; ++d) {
        v[d] = t[(long long)d * nPt + p0 + n] - t[(long long)d * nPt + p0];
        r2 += v[d] * v[d];
      }
      const double r = sqrt(r2);
      if (r > 0.0) {
        for (int d = 0; d < imDim; ++d) s[d] += v[d] / r;
        ++cnt;
      }
    }
    for (int d = 0; d < imDim; ++d) e[(long long)d * nLine + l] = cnt ? s[d] / cnt : 0.0;
  }
}

// dr[i] = t_i . e_line(i); keys of the first line for its sort
__global__ void ve_radius_kernel(const double* __restrict__ t, const double* __restrict__ e, int imDim, int nPt, int N,
                                 int nLine, double* __restrict__ dr, int* __restrict__ idx) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nPt; i += gridDim.x * blockDim.x) {
    const int l = i / N;
    double acc = 0.0;
    for (int d = 0; d < imDim; ++d) acc += t[(long long)d * nPt + i] * e[(long long)d * nLine + l];
    dr[i] = acc;
    if (i < N) idx[i] = i;
  }
}

// bmVolumeElement1 over every line in the first line's order perm: sorted
// values s_k, midpoints, end cells mirrored, lengths back at perm[k]
__global__ void ve_voronoi1_kernel(const double* __restrict__ dr, const int* __restrict__ perm, int N, int nLine,
                                   double* __restrict__ len) {
  const long long total = (long long)N * nLine;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int l = (int)(i / N), k = (int)(i % N);
    const double* col = dr + (long long)l * N;
    const double s = col[perm[k]];
    double lo, hi;
    if (N == 1) {
      lo = hi = s;
    } else {
      const double sp = k > 0 ? col[perm[k - 1]] : 0.0, sn = k < N - 1 ? col[perm[k + 1]] : 0.0;
      const double mp = k > 0 ? (s + sp) / 2 : 0.0, mn = k < N - 1 ? (sn + s) / 2 : 0.0;
      lo = k > 0 ? mp : s - (mn - s);
      hi = k < N - 1 ? mn : s + (s - mp);
    }
    len[(long long)l * N + perm[k]] = hi - lo;
  }
}

// angles of the directions e and -e (2 nLine), for the 2-D angular Voronoi
__global__ void ve_angle_kernel(const double* __restrict__ e, int nLine, double* __restrict__ ang, int* __restrict__ idx) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < 2 * nLine; k += gridDim.x * blockDim.x) {
    const int l = k < nLine ? k : k - nLine;
    const double sg = k < nLine ? 1.0 : -1.0;
    ang[k] = atan2(sg * e[nLine + l], sg * e[l]);
    idx[k] = k;
  }
}

// angular Voronoi width of line l: half the gap between its sorted
// neighbours, the wrap-around gap shared by the two ends
__global__ void ve_angvor_kernel(const double* __restrict__ a, const int* __restrict__ perm, int M, int nLine,
                                 double* __restrict__ vor) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < M; k += gridDim.x * blockDim.x) {
    const double cut = (M_PI - a[M - 1]) + (a[0] + M_PI);
    double v;
    if (k == 0)
      v = (a[1] - a[0]) / 2 + cut / 2;
    else if (k == M - 1)
      v = (a[M - 1] - a[M - 2]) / 2 + cut / 2;
    else
      v = (a[k + 1] - a[k - 1]) / 2;
    const int orig = perm[k];
    if (orig < nLine) vor[orig] = v;
  }
}

// v_i = len_i * ds_i: 3-D 4 pi |t|^2 / (2 nLine), 2-D |t| * vor_line
__global__ void ve_combine_kernel(const double* __restrict__ t, const double* __restrict__ len,
                                  const double* __restrict__ vor, int imDim, int nPt, int N, int nLine,
                                  double* __restrict__ v) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nPt; i += gridDim.x * blockDim.x) {
    double r2 = 0.0;
    for (int d = 0; d < imDim; ++d) r2 += t[(long long)d * nPt + i] * t[(long long)d * nPt + i];
    const double ds = imDim == 3 ? 4 * M_PI * r2 / (2.0 * nLine) : sqrt(r2) * vor[i / N];
    v[i] = len[i] * ds;
  }
}

// the centre samples: dr0 = mean over lines of len[N/2] / 2, one block, lines
// summed in order
__global__ void ve_centre_kernel(const double* __restrict__ len, int imDim, int N, int nLine, double* __restrict__ v) {
  __shared__ double part[kThreads];
  double s = 0.0;
  for (int l = threadIdx.x; l < nLine; l += blockDim.x) s += len[(long long)l * N + N / 2];
  part[threadIdx.x] = s;
  __syncthreads();
  __shared__ double v0;
  if (threadIdx.x == 0) {
    double tot = 0.0;
    for (int k = 0; k < (int)blockDim.x; ++k) tot += part[k];
    const double dr0 = tot / nLine / 2;
    v0 = imDim == 3 ? (4.0 / 3.0) * M_PI * dr0 * dr0 * dr0 / (2.0 * nLine) : M_PI * dr0 * dr0 / (2.0 * nLine);
  }
  __syncthreads();
  for (int l = threadIdx.x; l < nLine; l += blockDim.x) v[(long long)l * N + N / 2] = v0;
}

}  // namespace
}  // namespace mlg

using namespace mlg;

extern "C" int mlg_deapodization_dev(int imDim, const int* N_u, const double* dK_u, int kernelType, int nWin,
                                     const double* kernelParam, float* K, void* stream) {
  (void)dK_u;  // only scales the DFT, which cancels in the normalisation
  MLG_TRY(ensure_device());
  MLG_CHECK(K, "NULL output");
  DeapodTables T;
  MLG_TRY(deapod_tables(imDim, N_u, kernelType, nWin, kernelParam, T));
  cudaStream_t s = (cudaStream_t)stream;
  const DeapodDims D{T.N[0], T.N[1], T.N[2], T.S, T.Sy, T.Sz, imDim};
  DevBuf<double> w, cx, cy, cz, A2;
  DevBuf<unsigned long long> kmax;
  MLG_TRY(w.alloc(T.w.size(), s));
  MLG_TRY(cx.alloc(T.cx.size(), s));
  MLG_TRY(cy.alloc(T.cy.size(), s));
  MLG_TRY(cz.alloc(T.cz.size(), s));
  MLG_TRY(A2.alloc((size_t)D.Sz * D.N1 * D.N0, s));
  MLG_TRY(kmax.alloc(1, s));
  MLG_CUDA(cudaMemcpyAsync(w.p, T.w.data(), T.w.size() * 8, cudaMemcpyHostToDevice, s));
  MLG_CUDA(cudaMemcpyAsync(cx.p, T.cx.data(), T.cx.size() * 8, cudaMemcpyHostToDevice, s));
  MLG_CUDA(cudaMemcpyAsync(cy.p, T.cy.data(), T.cy.size() * 8, cudaMemcpyHostToDevice, s));
  MLG_CUDA(cudaMemcpyAsync(cz.p, T.cz.data(), T.cz.size() * 8, cudaMemcpyHostToDevice, s));
  MLG_CUDA(cudaMemsetAsync(kmax.p, 0, 8, s));
  const long long total = (long long)D.N0 * D.N1 * D.N2;
  deapod_xy_kernel<<<grid_of((long long)D.Sz * D.N1 * D.N0), kThreads, 0, s>>>(D, w.p, cx.p, cy.p, A2.p);
  MLG_LAUNCHED();
  deapod_max_kernel<<<grid_of(total), kThreads, 0, s>>>(D, A2.p, cz.p, kmax.p);
  MLG_LAUNCHED();
  deapod_final_kernel<<<grid_of(total), kThreads, 0, s>>>(D, A2.p, cz.p, kmax.p, T.K_max, K);
  MLG_LAUNCHED();
  // the tables are released in stream order; the host vectors must live
  // until their copies have been made
  MLG_CUDA(cudaStreamSynchronize(s));
  unsigned long long h = 0;
  MLG_CUDA(cudaMemcpy(&h, kmax.p, 8, cudaMemcpyDeviceToHost));
  MLG_CHECK(h != 0, "kernel transform vanishes (check kernel parameters)");
  return MLG_OK;
}

extern "C" int mlg_volume_element_radial_dev(int imDim, int nPt, int N, const double* t, double* v, void* stream) {
  MLG_TRY(ensure_device());
  MLG_CHECK(imDim == 2 || imDim == 3, "imDim must be 2 or 3");
  MLG_CHECK(N >= 2 && nPt >= N && nPt % N == 0, "nPt=%d must be a positive multiple of the line length N=%d", nPt, N);
  MLG_CHECK(t && v, "NULL argument");
  cudaStream_t s = (cudaStream_t)stream;
  const int nLine = nPt / N;
  DevBuf<double> e, dr, len, keys_out, ang, ang_out, vor;
  DevBuf<int> idx, perm, aidx, aperm;
  DevBuf<char> tmp;
  MLG_TRY(e.alloc((size_t)imDim * nLine, s));
  MLG_TRY(dr.alloc((size_t)nPt, s));
  MLG_TRY(len.alloc((size_t)nPt, s));
  MLG_TRY(keys_out.alloc((size_t)N, s));
  MLG_TRY(idx.alloc((size_t)N, s));
  MLG_TRY(perm.alloc((size_t)N, s));
  MLG_TRY(vor.alloc((size_t)nLine, s));
  ve_direction_kernel<<<grid_of(nLine), kThreads, 0, s>>>(t, imDim, nPt, N, nLine, e.p);
  MLG_LAUNCHED();
  ve_radius_kernel<<<grid_of(nPt), kThreads, 0, s>>>(t, e.p, imDim, nPt, N, nLine, dr.p, idx.p);
  MLG_LAUNCHED();
  // the first line's order (a stable sort of its radii)
  size_t tb = 0, tb2 = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tb, (const double*)nullptr, (double*)nullptr, (const int*)nullptr,
                                  (int*)nullptr, N);
  if (imDim == 2)
    cub::DeviceRadixSort::SortPairs(nullptr, tb2, (const double*)nullptr, (double*)nullptr, (const int*)nullptr,
                                    (int*)nullptr, 2 * nLine);
  MLG_TRY(tmp.alloc(std::max<size_t>(std::max(tb, tb2), 1), s));
  MLG_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tb, dr.p, keys_out.p, idx.p, perm.p, N, 0, 64, s));
  ve_voronoi1_kernel<<<grid_of((long long)N * nLine), kThreads, 0, s>>>(dr.p, perm.p, N, nLine, len.p);
  MLG_LAUNCHED();
  if (imDim == 2) {
    MLG_TRY(ang.alloc((size_t)2 * nLine, s));
    MLG_TRY(ang_out.alloc((size_t)2 * nLine, s));
    MLG_TRY(aidx.alloc((size_t)2 * nLine, s));
    MLG_TRY(aperm.alloc((size_t)2 * nLine, s));
    ve_angle_kernel<<<grid_of(2 * nLine), kThreads, 0, s>>>(e.p, nLine, ang.p, aidx.p);
    MLG_LAUNCHED();
    tb2 = tmp.n;
    MLG_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tb2, ang.p, ang_out.p, aidx.p, aperm.p, 2 * nLine, 0, 64, s));
    ve_angvor_kernel<<<grid_of(2 * nLine), kThreads, 0, s>>>(ang_out.p, aperm.p, 2 * nLine, nLine, vor.p);
    MLG_LAUNCHED();
  }
  ve_combine_kernel<<<grid_of(nPt), kThreads, 0, s>>>(t, len.p, vor.p, imDim, nPt, N, nLine, v);
  MLG_LAUNCHED();
  ve_centre_kernel<<<1, kThreads, 0, s>>>(len.p, imDim, N, nLine, v);
  MLG_LAUNCHED();
  return MLG_OK;
}
