// The transform tail of the gridded reconstructions on the device:
// src/fourier123/map_function/nonCartesian/bmMathilda.m:76-121 and
// bmNasha.m:48-88 after their gridding step (leight gridder or Gn product):
//   x = coil_pinv( crop( K .* bmIDF(grid) ) )
// bmIDF = fftshift(ifft(ifftshift(.))) * prod(N_u) * prod(dK_u) per coil
// (src/fourier3/bmIDF3.m), K the deapodisation (bmK.m), crop to n_u
// (bmImCrope.m), coil_pinv = sum_c conj(C) x / sum_c |C|^2
// (src/coilSense/map/bmCoilSense_pinv.m:10); without C every coil's image is
// returned.
//
// The centred inverse transform is a plain inverse DFT between two
// (-1)^(x+y+z) modulations (even N, as bmIDF requires); the input modulation
// is fused into the gather of the gridded data into coil-major order, the
// output one, the scale, K, the crop and the coil combination into one tail
// kernel.  The transform itself is cuFFT (batched over coils): a one-shot
// step of a non-iterative reconstruction.
#include <cufft.h>

#include "mlg_internal.cuh"

namespace mlg {

constexpr int kGtThreads = 256;

static int gt_grid(long long n) {
  return (int)std::max<long long>(1, std::min<long long>((n + kGtThreads - 1) / kGtThreads, 148LL * 16));
}

__device__ __forceinline__ int cell_parity(long long cell, int imDim, int Nx, int Ny) {
  long long s = cell % Nx;
  if (imDim > 1) {
    const long long q = cell / Nx;
    s += q % Ny;
    if (imDim > 2) s += q / Ny;
  }
  return (int)(s & 1);
}

// point layout [Nu][nCh] (interleaved complex, or split re / im) ->
// coil-major [nCh][Nu] with the (-1)^cell input modulation
__global__ void gt_gather_kernel(const void* __restrict__ a, const float* __restrict__ b, int split, long long Nu,
                                 int nCh, int imDim, int Nx, int Ny, float2* __restrict__ out) {
  const long long n = Nu * nCh;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const long long c = i / Nu, cell = i - c * Nu;
    const long long src = cell * nCh + c;
    float2 v = split ? make_float2(reinterpret_cast<const float*>(a)[src], b[src])
                     : reinterpret_cast<const float2*>(a)[src];
    if (cell_parity(cell, imDim, Nx, Ny)) v = make_float2(-v.x, -v.y);
    out[i] = v;
  }
}

struct TailGeom {
  int imDim;
  int N[3], n[3], off[3];
  long long Nu, nu;
  int nCh;
  float fac;  // shift sign * single(prod(N_u) prod(dK_u)) / prod(N_u)
};

// one thread per image pixel p of the n_u block
__global__ void gt_tail_kernel(const float2* __restrict__ g, TailGeom t, const float* __restrict__ K,
                               const float2* __restrict__ C, float2* __restrict__ x) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < t.nu;
       p += (long long)gridDim.x * blockDim.x) {
    const long long px = p % t.n[0], q = p / t.n[0];
    const long long py = q % t.n[1], pz = q / t.n[1];
    const long long cell =
        (px + t.off[0]) + (long long)t.N[0] * ((py + t.off[1]) + (long long)t.N[1] * (pz + t.off[2]));
    const float f = cell_parity(cell, t.imDim, t.N[0], t.N[1]) ? -t.fac : t.fac;
    const float k = K[cell];
    if (C) {
      float2 num = make_float2(0.f, 0.f);
      float den = 0.f;
      for (int c = 0; c < t.nCh; ++c) {
        const float2 gv = g[(long long)c * t.Nu + cell];
        const float2 v = make_float2(__fmul_rn(__fmul_rn(gv.x, f), k), __fmul_rn(__fmul_rn(gv.y, f), k));
        const float2 cc = C[p * t.nCh + c];
        // conj(C) .* x
        num.x = __fadd_rn(num.x, __fadd_rn(__fmul_rn(cc.x, v.x), __fmul_rn(cc.y, v.y)));
        num.y = __fadd_rn(num.y, __fsub_rn(__fmul_rn(cc.x, v.y), __fmul_rn(cc.y, v.x)));
        den = __fadd_rn(den, __fadd_rn(__fmul_rn(cc.x, cc.x), __fmul_rn(cc.y, cc.y)));
      }
      x[p] = make_float2(__fdiv_rn(num.x, den), __fdiv_rn(num.y, den));
    } else {
      for (int c = 0; c < t.nCh; ++c) {
        const float2 gv = g[(long long)c * t.Nu + cell];
        x[(long long)c * t.nu + p] = make_float2(__fmul_rn(__fmul_rn(gv.x, f), k), __fmul_rn(__fmul_rn(gv.y, f), k));
      }
    }
  }
}

}  // namespace mlg

using namespace mlg;

extern "C" int mlg_gridded_tail_dev(int imDim, const int* N_u, const int* n_u, const float* dK_u, int nCh,
                                    int grid_split, const void* grid_a, const void* grid_b, const float* K,
                                    const void* C, void* x, void* stream) {
  MLG_TRY(ensure_device());
  MLG_CHECK(imDim >= 1 && imDim <= 3 && N_u && dK_u && nCh >= 1, "invalid argument");
  MLG_CHECK(grid_a && (!grid_split || grid_b) && K && x, "NULL buffer");
  TailGeom t;
  t.imDim = imDim;
  t.nCh = nCh;
  t.Nu = t.nu = 1;
  float sc = 1.f;
  double dk = 1.0;
  for (int d = 0; d < 3; ++d) {
    t.N[d] = d < imDim ? N_u[d] : 1;
    t.n[d] = d < imDim ? (n_u ? n_u[d] : N_u[d]) : 1;
    if (d < imDim) {
      MLG_CHECK(t.N[d] >= 2 && !(t.N[d] & 1), "N_u must be even and >= 2 (dim %d: %d)", d, t.N[d]);
      MLG_CHECK(t.n[d] >= 1 && t.n[d] <= t.N[d], "n_u must lie in [1, N_u] (dim %d: %d)", d, t.n[d]);
      MLG_CHECK(dK_u[d] > 0, "dK_u must be > 0");
      dk *= dK_u[d];
      if ((t.N[d] / 2) & 1) sc = -sc;
    }
    t.off[d] = t.N[d] / 2 - t.n[d] / 2;  // bmImCrope.m: the centred n_u block
    t.Nu *= t.N[d];
    t.nu *= t.n[d];
  }
  // ifft's 1/prod(N) times single(prod(N_u) * prod(dK_u)) of bmIDF
  const float F = (float)((double)t.Nu * dk);
  t.fac = (float)(sc * (double)F / (double)t.Nu);
  cudaStream_t s = (cudaStream_t)stream;
  DevBuf<float2> cm;
  MLG_TRY(cm.alloc((size_t)(t.Nu * nCh), s));
  gt_gather_kernel<<<gt_grid(t.Nu * nCh), kGtThreads, 0, s>>>(grid_a, (const float*)grid_b, grid_split, t.Nu, nCh,
                                                               imDim, t.N[0], t.N[1], cm.p);
  MLG_LAUNCHED();
  cufftHandle h;
  int nn[3];
  for (int d = 0; d < imDim; ++d) nn[d] = t.N[imDim - 1 - d];
  MLG_CUFFT(cufftPlanMany(&h, imDim, nn, nullptr, 1, (int)t.Nu, nullptr, 1, (int)t.Nu, CUFFT_C2C, nCh));
  cufftSetStream(h, s);
  const cufftResult r = cufftExecC2C(h, (cufftComplex*)cm.p, (cufftComplex*)cm.p, CUFFT_INVERSE);
  count_launch();
  if (r != CUFFT_SUCCESS) {
    cufftDestroy(h);
    return fail(MLG_ERR_CUDA, "gridded tail: cufftExecC2C failed (%d)", (int)r);
  }
  gt_tail_kernel<<<gt_grid(t.nu), kGtThreads, 0, s>>>(cm.p, t, K, (const float2*)C, (float2*)x);
  MLG_LAUNCHED();
  // the plan's work area belongs to the calls queued on s: wait before freeing it
  const cudaError_t e = cudaStreamSynchronize(s);
  cufftDestroy(h);
  if (e != cudaSuccess) return fail(MLG_ERR_CUDA, "gridded tail failed: %s", cudaGetErrorString(e));
  return MLG_OK;
}
