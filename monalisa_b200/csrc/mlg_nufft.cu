// Fused NUFFT operators around cuFFT.
//
// bmShanna (src/fourier123/map_function/nonCartesian/bmShanna_MATLAB.m:28-54):
//   x .* KFC -> zero-fill n_u -> N_u -> fftshift(fft(ifftshift)) -> Gu
// bmNakatsha (bmNakatsha_MATLAB.m:32-56):
//   Gut -> fftshift(ifft(ifftshift)) -> crop -> .* KFC_conj -> coil sum
//
// For even N the centred transform is a modulated plain DFT:
//   fftshift(F(ifftshift(v)))[k] = (-1)^k (-1)^(N/2) F((-1)^n v)[k]
// (same for the inverse).  The input modulation is fused into the
// pre-kernel (Shanna) or folded into the row signs of Gut (Nakatsha); the
// output modulation is folded into the column signs of Gu (Shanna) or fused
// into the post-kernel (Nakatsha).  So a Shanna is three kernels
// (pre, cuFFT, SpMM) and a Nakatsha three (SpMM, cuFFT, post), with every
// elementwise stage of the reference fused into one of them.
#include <algorithm>
#include <vector>

#include "mlg_plan.cuh"

namespace mlg {

constexpr int kEwThreads = 256;

struct Geo {
  int imDim;
  int N[3], n[3], off[3];  // off = N/2 - n/2 (zero-fill / crop origin)
  long long Nu, nu;
  int nCh;
};

static Geo geo_of(const mlg_plan_s* p) {
  Geo g;
  g.imDim = p->imDim;
  for (int d = 0; d < 3; ++d) {
    g.N[d] = p->N[d];
    g.n[d] = p->n[d];
    g.off[d] = p->N[d] / 2 - p->n[d] / 2;
  }
  g.Nu = p->Nu_tot;
  g.nu = p->nu_tot;
  g.nCh = p->nCh;
  return g;
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(__fsub_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)),
                     __fadd_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x)));
}

// grid[c][cell] = (cell in image block ? x[m] * KFC[c][m] : 0) * (-1)^(x+y+z)
__global__ void __launch_bounds__(kEwThreads) shanna_pre_kernel(Geo g, const float2* __restrict__ x, int x_per_coil,
                                                                const float2* __restrict__ KFC,
                                                                float2* __restrict__ grid) {
  const long long total = g.Nu * g.nCh;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(i / g.Nu);
    const long long cell = i - (long long)c * g.Nu;
    const int cx = (int)(cell % g.N[0]);
    const long long q = cell / g.N[0];
    const int cy = (int)(q % g.N[1]);
    const int cz = (int)(q / g.N[1]);
    const int bx = cx - g.off[0], by = cy - g.off[1], bz = cz - g.off[2];
    float2 v = make_float2(0.f, 0.f);
    if (bx >= 0 && bx < g.n[0] && by >= 0 && by < g.n[1] && bz >= 0 && bz < g.n[2]) {
      const long long m = bx + (long long)g.n[0] * (by + (long long)g.n[1] * bz);
      const float2 xv = __ldg(x + (x_per_coil ? (long long)c * g.nu + m : m));
      v = cmul(xv, __ldg(KFC + (long long)c * g.nu + m));
      if ((cx + cy + cz) & 1) v = make_float2(-v.x, -v.y);
    }
    grid[i] = v;
  }
}

// x[m] = scale * sum_c KFCc[c][m] * s(n) * grid[c][n(m)],
// s(n) = (-1)^(x+y+z) * shift_const / prod(N); optional FP64 |x|^2 partials.
__global__ void __launch_bounds__(kEwThreads) nakatsha_post_kernel(Geo g, const float2* __restrict__ grid,
                                                                   const float2* __restrict__ KFCc, float sfac,
                                                                   float2* __restrict__ x, double* partial) {
  __shared__ double sh[kEwThreads / 32];
  double sq = 0.0;
  for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < g.nu;
       m += (long long)gridDim.x * blockDim.x) {
    const int bx = (int)(m % g.n[0]);
    const long long q = m / g.n[0];
    const int by = (int)(q % g.n[1]);
    const int bz = (int)(q / g.n[1]);
    const int cx = bx + g.off[0], cy = by + g.off[1], cz = bz + g.off[2];
    const long long cell = cx + (long long)g.N[0] * (cy + (long long)g.N[1] * cz);
    const float s = ((cx + cy + cz) & 1) ? -sfac : sfac;
    float2 acc = make_float2(0.f, 0.f);
    for (int c = 0; c < g.nCh; ++c) {
      float2 v = __ldg(grid + (long long)c * g.Nu + cell);
      v = make_float2(__fmul_rn(v.x, s), __fmul_rn(v.y, s));
      const float2 t = cmul(v, __ldg(KFCc + (long long)c * g.nu + m));
      acc = make_float2(__fadd_rn(acc.x, t.x), __fadd_rn(acc.y, t.y));
    }
    x[m] = acc;
    sq += (double)acc.x * acc.x + (double)acc.y * acc.y;
  }
  if (partial) {
    for (int o = 16; o > 0; o >>= 1) sq += __shfl_down_sync(0xffffffffu, sq, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = sq;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int i = 0; i < kEwThreads / 32; ++i) t += sh[i];
      partial[blockIdx.x] = t;
    }
  }
}

static int ew_grid(long long n) {
  return (int)std::max<long long>(1, std::min<long long>((n + kEwThreads - 1) / kEwThreads, 148LL * 16));
}

int post_partial_count(const mlg_plan_s* p) { return ew_grid(p->nu_tot); }

int shanna_pre(mlg_plan_s* p, const float2* x, bool x_per_coil, cudaStream_t s) {
  const Geo g = geo_of(p);
  shanna_pre_kernel<<<ew_grid(g.Nu * g.nCh), kEwThreads, 0, s>>>(g, x, x_per_coil ? 1 : 0, p->KFC, p->grid);
  MLG_LAUNCHED();
  return MLG_OK;
}

int fft_exec(mlg_plan_s* p, bool forward, cudaStream_t s) {
  MLG_CUFFT(cufftSetStream(p->fft, s));
  MLG_CUFFT(cufftExecC2C(p->fft, (cufftComplex*)p->grid, (cufftComplex*)p->grid,
                         forward ? CUFFT_FORWARD : CUFFT_INVERSE));
  count_launch();
  return MLG_OK;
}

int shanna_run(mlg_plan_s* p, const float2* x, bool x_per_coil, float2* y, const float* sqn_w, double* partial,
               int* n_partial, cudaStream_t s) {
  MLG_TRY(shanna_pre(p, x, x_per_coil, s));
  MLG_TRY(fft_exec(p, true, s));
  return shanna_spmm(p, y, sqn_w, partial, n_partial, s);
}

int shanna_spmm(mlg_plan_s* p, float2* y, const float* sqn_w, double* partial, int* n_partial, cudaStream_t s) {
  SpmmArgs a;
  a.m = &p->Gu_s;
  a.nCh = p->nCh;
  a.in.layout = Layout::kCoilC64;
  a.in.a = p->grid;
  a.in.rows = p->Nu_tot;
  a.out.layout = Layout::kPointC64;
  a.out.a = y;
  a.out.rows = p->nPt;
  a.sqn_row_weight = sqn_w;
  a.partial = partial;
  if (n_partial) *n_partial = partial ? spmm_partial_count(a) : 0;
  return spmm(a, s);
}

int nakatsha_run(mlg_plan_s* p, const float2* y, const float* HY, float scale, float2* x, double* partial,
                 int* n_partial, cudaStream_t s) {
  MLG_TRY(nakatsha_spmm(p, y, HY, s));
  MLG_TRY(fft_exec(p, false, s));
  return nakatsha_post(p, scale, x, partial, n_partial, s);
}

int nakatsha_post(mlg_plan_s* p, float scale, float2* x, double* partial, int* n_partial, cudaStream_t s) {
  const Geo g = geo_of(p);
  const float sfac = (float)((double)p->shift_const / (double)p->Nu_tot * (double)scale);
  nakatsha_post_kernel<<<ew_grid(g.nu), kEwThreads, 0, s>>>(g, p->grid, p->KFCc, sfac, x, partial);
  MLG_LAUNCHED();
  if (n_partial) *n_partial = partial ? ew_grid(g.nu) : 0;
  return MLG_OK;
}

int nakatsha_spmm(mlg_plan_s* p, const float2* y, const float* HY, cudaStream_t s) {
  SpmmArgs a;
  a.m = &p->Gut_s;
  a.nCh = p->nCh;
  a.in.layout = Layout::kPointC64;
  a.in.a = const_cast<float2*>(y);
  a.in.rows = p->nPt;
  a.in_row_scale = HY;
  a.out.layout = Layout::kCoilC64;
  a.out.a = p->grid;
  a.out.rows = p->Nu_tot;
  return spmm(a, s);
}

// ---- layout conversion kernels ----------------------------------------------
// split [rows, nCh] column layout <-> float2 point layout [rows][nCh]
__global__ void pack_col_to_point_kernel(const float* __restrict__ re, const float* __restrict__ im, long long rows,
                                         int nCh, float2* __restrict__ out) {
  const long long n = rows * nCh;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const long long r = i / nCh;
    const int c = (int)(i - r * nCh);
    out[i] = make_float2(re[(long long)c * rows + r], im ? im[(long long)c * rows + r] : 0.f);
  }
}

__global__ void unpack_point_to_col_kernel(const float2* __restrict__ in, long long rows, int nCh,
                                           float* __restrict__ re, float* __restrict__ im) {
  const long long n = rows * nCh;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(i / rows);
    const long long r = i - (long long)c * rows;
    const float2 v = in[r * nCh + c];
    re[i] = v.x;
    im[i] = v.y;
  }
}

// split -> interleaved (same element order)
__global__ void interleave_kernel(const float* __restrict__ re, const float* __restrict__ im, long long n,
                                  float2* __restrict__ out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = make_float2(re[i], im ? im[i] : 0.f);
}

__global__ void deinterleave_kernel(const float2* __restrict__ in, long long n, float* __restrict__ re,
                                    float* __restrict__ im) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float2 v = in[i];
    re[i] = v.x;
    im[i] = v.y;
  }
}

int pack_col_to_point(const float* re, const float* im, long long rows, int nCh, float2* out, cudaStream_t s) {
  pack_col_to_point_kernel<<<ew_grid(rows * nCh), kEwThreads, 0, s>>>(re, im, rows, nCh, out);
  MLG_LAUNCHED();
  return MLG_OK;
}
int unpack_point_to_col(const float2* in, long long rows, int nCh, float* re, float* im, cudaStream_t s) {
  unpack_point_to_col_kernel<<<ew_grid(rows * nCh), kEwThreads, 0, s>>>(in, rows, nCh, re, im);
  MLG_LAUNCHED();
  return MLG_OK;
}
int interleave(const float* re, const float* im, long long n, float2* out, cudaStream_t s) {
  interleave_kernel<<<ew_grid(n), kEwThreads, 0, s>>>(re, im, n, out);
  MLG_LAUNCHED();
  return MLG_OK;
}
int deinterleave(const float2* in, long long n, float* re, float* im, cudaStream_t s) {
  deinterleave_kernel<<<ew_grid(n), kEwThreads, 0, s>>>(in, n, re, im);
  MLG_LAUNCHED();
  return MLG_OK;
}

// ---- plan lifecycle ---------------------------------------------------------
static void plan_free(mlg_plan_s* p) {
  if (!p) return;
  cudaSetDevice(p->device);
  if (p->cg_graph) cudaGraphExecDestroy(p->cg_graph);
  if (p->fft_ready) cufftDestroy(p->fft);
  csr_free_sign_copy(p->Gu_s);
  csr_free_sign_copy(p->Gut_s);
  cudaFree(p->KFC);
  cudaFree(p->KFCc);
  cudaFree(p->grid);
  cudaFree(p->partial);
  cudaFree(p->scalars);
  cudaFree(p->x_p);
  cudaFree(p->x_dagM);
  cudaFree(p->k_res);
  cudaFree(p->k_Mp);
  cudaFree(p->HY);
  if (p->ev_in) cudaEventDestroy(p->ev_in);
  if (p->ev_out) cudaEventDestroy(p->ev_out);
  if (p->stream) cudaStreamDestroy(p->stream);
  delete p;
}

static int plan_create_impl(int imDim, const int* N_u, const int* n_u, int nCh, const Csr* Gu, const Csr* Gut,
                            const float* KFC_re, const float* KFC_im, const float* KFCc_re, const float* KFCc_im,
                            bool kfc_on_device, mlg_plan_s** out) {
  MLG_CHECK(out, "NULL output");
  *out = nullptr;
  MLG_CHECK(imDim >= 1 && imDim <= 3, "imDim must be 1, 2 or 3");
  MLG_CHECK(N_u && nCh >= 1, "invalid N_u / nCh");
  MLG_CHECK(Gu || Gut, "at least one of Gu / Gut is needed");
  MLG_TRY(ensure_device());
  mlg_plan_s* p = new mlg_plan_s();
  cudaGetDevice(&p->device);
  p->imDim = imDim;
  p->nCh = nCh;
  long long Nu = 1, nu = 1;
  float sc = 1.0f;
  for (int d = 0; d < 3; ++d) {
    p->N[d] = d < imDim ? N_u[d] : 1;
    p->n[d] = d < imDim ? (n_u ? n_u[d] : N_u[d]) : 1;
    if (d < imDim) {
      if (p->N[d] < 2 || (p->N[d] & 1) || p->n[d] < 2 || (p->n[d] & 1) || p->n[d] > p->N[d]) {
        plan_free(p);
        return fail(MLG_ERR_ARG, "N_u and n_u must be even, >= 2, with n_u <= N_u (dim %d: N=%d n=%d)", d,
                    N_u[d], n_u ? n_u[d] : N_u[d]);
      }
      if ((p->N[d] / 2) & 1) sc = -sc;
    }
    Nu *= p->N[d];
    nu *= p->n[d];
  }
  p->Nu_tot = Nu;
  p->nu_tot = nu;
  p->shift_const = sc;
  p->HX = 1.0;  // dK_u = 1 until mlg_plan_set_dk
  for (int d = 0; d < imDim; ++d) p->HX = (double)((float)p->HX * (1.0f / (float)p->N[d]));
  if (Gu && (Gu->r_size != Nu)) {
    plan_free(p);
    return fail(MLG_ERR_ARG, "Gu has %d columns, prod(N_u) = %lld", Gu->r_size, Nu);
  }
  if (Gut && (Gut->l_size != Nu)) {
    plan_free(p);
    return fail(MLG_ERR_ARG, "Gut has %d rows, prod(N_u) = %lld", Gut->l_size, Nu);
  }
  if (Gu && Gut && Gu->l_size != Gut->r_size) {
    plan_free(p);
    return fail(MLG_ERR_ARG, "Gu rows (%d) and Gut columns (%d) differ", Gu->l_size, Gut->r_size);
  }
  p->nPt = Gu ? Gu->l_size : Gut->r_size;
  p->Gu = Gu;
  p->Gut = Gut;
  int st = MLG_OK;
  auto bail = [&](int status) {
    plan_free(p);
    return status;
  };
  if (cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&p->ev_in, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&p->ev_out, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    return bail(fail(MLG_ERR_CUDA, "stream/event creation failed"));
  }
  cudaStream_t s = p->stream;
  if (Gu && (st = csr_sign_copy(*Gu, false, imDim, p->N, sc, p->Gu_s, s)) != MLG_OK) return bail(st);
  if (Gut && (st = csr_sign_copy(*Gut, true, imDim, p->N, 1.0f, p->Gut_s, s)) != MLG_OK) return bail(st);
  const size_t kbytes = sizeof(float2) * (size_t)nu * nCh;
  if (cudaMalloc(&p->KFC, kbytes) != cudaSuccess || cudaMalloc(&p->KFCc, kbytes) != cudaSuccess ||
      cudaMalloc(&p->grid, sizeof(float2) * (size_t)Nu * nCh) != cudaSuccess) {
    cudaGetLastError();
    return bail(fail(MLG_ERR_OOM, "plan: device allocation failed"));
  }
  // KFC / KFC_conj: [prod(n_u), nCh] column layout = coil-major
  const long long nk = nu * nCh;
  if (kfc_on_device) {
    if ((st = interleave(KFC_re, KFC_im, nk, p->KFC, s)) != MLG_OK) return bail(st);
    if ((st = interleave(KFCc_re, KFCc_im, nk, p->KFCc, s)) != MLG_OK) return bail(st);
  } else {
    float* tmp = nullptr;
    if (cudaMalloc(&tmp, sizeof(float) * 2 * (size_t)nk) != cudaSuccess) {
      cudaGetLastError();
      return bail(fail(MLG_ERR_OOM, "plan: staging allocation failed"));
    }
    const float* srcs[2][2] = {{KFC_re, KFC_im}, {KFCc_re, KFCc_im}};
    float2* dsts[2] = {p->KFC, p->KFCc};
    for (int k = 0; k < 2; ++k) {
      if (!srcs[k][0]) {
        cudaMemsetAsync(dsts[k], 0, sizeof(float2) * (size_t)nk, s);
        continue;
      }
      cudaMemcpyAsync(tmp, srcs[k][0], sizeof(float) * nk, cudaMemcpyHostToDevice, s);
      if (srcs[k][1]) cudaMemcpyAsync(tmp + nk, srcs[k][1], sizeof(float) * nk, cudaMemcpyHostToDevice, s);
      if ((st = interleave(tmp, srcs[k][1] ? tmp + nk : nullptr, nk, dsts[k], s)) != MLG_OK) {
        cudaFree(tmp);
        return bail(st);
      }
    }
    cudaStreamSynchronize(s);
    cudaFree(tmp);
  }
  int n[3];
  for (int d = 0; d < imDim; ++d) n[d] = p->N[imDim - 1 - d];  // cuFFT: slowest dimension first
  if (cufftPlanMany(&p->fft, imDim, n, nullptr, 1, (int)Nu, nullptr, 1, (int)Nu, CUFFT_C2C, nCh) != CUFFT_SUCCESS)
    return bail(fail(MLG_ERR_CUDA, "cufftPlanMany failed for N=(%d,%d,%d) batch %d", p->N[0], p->N[1], p->N[2], nCh));
  p->fft_ready = true;
  size_t fft_bytes = 0;
  cufftGetSize(p->fft, &fft_bytes);
  // partial-sum buffer: the largest CTA count any fused reduction uses
  int cap = post_partial_count(p) + 8;
  if (Gu) {
    SpmmArgs a;
    a.m = &p->Gu_s;
    a.nCh = nCh;
    cap = std::max(cap, spmm_partial_count(a));
  }
  cap = std::max(cap, ew_grid((long long)p->nPt * nCh) + 8);
  p->partial_cap = cap;
  if (cudaMalloc(&p->partial, sizeof(double) * (size_t)cap) != cudaSuccess ||
      cudaMalloc(&p->scalars, sizeof(double) * 64) != cudaSuccess) {
    cudaGetLastError();
    return bail(fail(MLG_ERR_OOM, "plan: partial buffer allocation failed"));
  }
  if (cudaStreamSynchronize(s) != cudaSuccess) return bail(fail(MLG_ERR_CUDA, "plan creation failed"));
  p->bytes = 2 * kbytes + sizeof(float2) * (size_t)Nu * nCh + fft_bytes +
             sizeof(float) * (size_t)((Gu ? Gu->nnz : 0) + (Gut ? Gut->nnz : 0)) + sizeof(double) * (cap + 64);
  *out = p;
  return MLG_OK;
}

// Orders `work` on the plan's stream after the caller's stream and back.
struct StreamJoin {
  mlg_plan_s* p;
  cudaStream_t user;
  StreamJoin(mlg_plan_s* plan, cudaStream_t u) : p(plan), user(u) {
    cudaEventRecord(p->ev_in, user);
    cudaStreamWaitEvent(p->stream, p->ev_in, 0);
  }
  ~StreamJoin() {
    cudaEventRecord(p->ev_out, p->stream);
    cudaStreamWaitEvent(user, p->ev_out, 0);
  }
};

}  // namespace mlg

using namespace mlg;

extern "C" {

int mlg_plan_create(int imDim, const int* N_u, const int* n_u, int nCh, mlg_matrix_t Gu, mlg_matrix_t Gut,
                    const float* KFC_re, const float* KFC_im, const float* KFCc_re, const float* KFCc_im,
                    mlg_plan_t* out) {
  MLG_CHECK(Gu || Gut, "at least one of Gu / Gut is needed");
  return plan_create_impl(imDim, N_u, n_u, nCh, Gu ? &Gu->csr : nullptr, Gut ? &Gut->csr : nullptr, KFC_re, KFC_im,
                          KFCc_re, KFCc_im, false, out);
}

int mlg_plan_destroy(mlg_plan_t p) {
  plan_free(p);
  return MLG_OK;
}

int mlg_plan_device_bytes(mlg_plan_t p, long long* bytes) {
  MLG_CHECK(p && bytes, "NULL argument");
  *bytes = (long long)p->bytes;
  return MLG_OK;
}

int mlg_shanna_dev(mlg_plan_t p, const void* x, int x_per_coil, void* y, void* stream) {
  MLG_CHECK(p && x && y, "NULL argument");
  MLG_CHECK(p->Gu, "plan has no Gu");
  MLG_CUDA(cudaSetDevice(p->device));
  StreamJoin j(p, (cudaStream_t)stream);
  return shanna_run(p, (const float2*)x, x_per_coil != 0, (float2*)y, nullptr, nullptr, nullptr, p->stream);
}

int mlg_nakatsha_dev(mlg_plan_t p, const void* y, const float* HY, float scale, void* x, void* stream) {
  MLG_CHECK(p && x && y, "NULL argument");
  MLG_CHECK(p->Gut, "plan has no Gut");
  MLG_CUDA(cudaSetDevice(p->device));
  StreamJoin j(p, (cudaStream_t)stream);
  return nakatsha_run(p, (const float2*)y, HY, scale, (float2*)x, nullptr, nullptr, p->stream);
}

// Stateless host-buffer operators (drop-ins for the CUFFT MEX files).
int mlg_shanna(int imDim, const int* N_u, const int* n_u, int nCh, const float* xR, const float* xI, int x_nCol,
               const float* KFC_R, const float* KFC_I, int r_size, const int* r_jump, const int* r_nJump,
               const float* m_val, int l_size, const int* l_jump, int l_nJump, float* yR, float* yI) {
  MLG_TRY(ensure_device());
  MLG_CHECK(xR && KFC_R && yR && yI, "NULL buffer");
  MLG_CHECK(x_nCol == 1 || x_nCol == nCh, "x must have 1 or nCh columns (got %d, nCh=%d)", x_nCol, nCh);
  mlg_matrix_t G = nullptr;
  MLG_TRY(mlg_matrix_create(r_size, r_jump, r_nJump, m_val, l_size, l_jump, l_nJump, &G));
  mlg_plan_s* p = nullptr;
  int st = plan_create_impl(imDim, N_u, n_u, nCh, &G->csr, nullptr, KFC_R, KFC_I, nullptr, nullptr, false, &p);
  if (st != MLG_OK) {
    mlg_matrix_destroy(G);
    return st;
  }
  cudaStream_t s = p->stream;
  const long long nx = p->nu_tot * x_nCol, ny = (long long)p->nPt * nCh;
  float *dx = nullptr, *dy = nullptr;
  float2 *x2 = nullptr, *y2 = nullptr;
  if (cudaMalloc(&dx, sizeof(float) * 2 * nx) != cudaSuccess || cudaMalloc(&x2, sizeof(float2) * nx) != cudaSuccess ||
      cudaMalloc(&y2, sizeof(float2) * ny) != cudaSuccess || cudaMalloc(&dy, sizeof(float) * 2 * ny) != cudaSuccess) {
    cudaGetLastError();
    st = fail(MLG_ERR_OOM, "shanna: device allocation failed");
  }
  if (st == MLG_OK) {
    cudaMemcpyAsync(dx, xR, sizeof(float) * nx, cudaMemcpyHostToDevice, s);
    if (xI) cudaMemcpyAsync(dx + nx, xI, sizeof(float) * nx, cudaMemcpyHostToDevice, s);
    st = interleave(dx, xI ? dx + nx : nullptr, nx, x2, s);
  }
  if (st == MLG_OK) st = shanna_run(p, x2, x_nCol > 1, y2, nullptr, nullptr, nullptr, s);
  if (st == MLG_OK) st = unpack_point_to_col(y2, p->nPt, nCh, dy, dy + ny, s);
  if (st == MLG_OK) {
    cudaMemcpyAsync(yR, dy, sizeof(float) * ny, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(yI, dy + ny, sizeof(float) * ny, cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) st = fail(MLG_ERR_CUDA, "shanna failed: %s",
                                                           cudaGetErrorString(cudaGetLastError()));
  }
  cudaStreamSynchronize(s);
  cudaFree(dx);
  cudaFree(dy);
  cudaFree(x2);
  cudaFree(y2);
  plan_free(p);
  mlg_matrix_destroy(G);
  return st;
}

int mlg_nakatsha(int imDim, const int* N_u, const int* n_u, int nCh, const float* yR, const float* yI,
                 const float* KFCc_R, const float* KFCc_I, int r_size, const int* r_jump, const int* r_nJump,
                 const float* m_val, int l_size, const int* l_jump, int l_nJump, float* xR, float* xI) {
  MLG_TRY(ensure_device());
  MLG_CHECK(yR && yI && KFCc_R && xR && xI, "NULL buffer");
  mlg_matrix_t G = nullptr;
  MLG_TRY(mlg_matrix_create(r_size, r_jump, r_nJump, m_val, l_size, l_jump, l_nJump, &G));
  mlg_plan_s* p = nullptr;
  int st = plan_create_impl(imDim, N_u, n_u, nCh, nullptr, &G->csr, nullptr, nullptr, KFCc_R, KFCc_I, false, &p);
  if (st != MLG_OK) {
    mlg_matrix_destroy(G);
    return st;
  }
  cudaStream_t s = p->stream;
  const long long ny = (long long)p->nPt * nCh, nx = p->nu_tot;
  float *dy = nullptr, *dx = nullptr;
  float2 *y2 = nullptr, *x2 = nullptr;
  if (cudaMalloc(&dy, sizeof(float) * 2 * ny) != cudaSuccess || cudaMalloc(&y2, sizeof(float2) * ny) != cudaSuccess ||
      cudaMalloc(&x2, sizeof(float2) * nx) != cudaSuccess || cudaMalloc(&dx, sizeof(float) * 2 * nx) != cudaSuccess) {
    cudaGetLastError();
    st = fail(MLG_ERR_OOM, "nakatsha: device allocation failed");
  }
  if (st == MLG_OK) {
    cudaMemcpyAsync(dy, yR, sizeof(float) * ny, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dy + ny, yI, sizeof(float) * ny, cudaMemcpyHostToDevice, s);
    st = pack_col_to_point(dy, dy + ny, p->nPt, nCh, y2, s);
  }
  if (st == MLG_OK) st = nakatsha_run(p, y2, nullptr, 1.0f, x2, nullptr, nullptr, s);
  if (st == MLG_OK) st = deinterleave(x2, nx, dx, dx + nx, s);
  if (st == MLG_OK) {
    cudaMemcpyAsync(xR, dx, sizeof(float) * nx, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(xI, dx + nx, sizeof(float) * nx, cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) st = fail(MLG_ERR_CUDA, "nakatsha failed: %s",
                                                           cudaGetErrorString(cudaGetLastError()));
  }
  cudaStreamSynchronize(s);
  cudaFree(dx);
  cudaFree(dy);
  cudaFree(x2);
  cudaFree(y2);
  plan_free(p);
  mlg_matrix_destroy(G);
  return st;
}

}  // extern "C"

// ---- inverse DFT (bmIDF{1,2,3}) ----------------------------------------------
namespace mlg {

__global__ void idf_modulate_kernel(const float* __restrict__ re, const float* __restrict__ im, long long Nu,
                                    long long total, int imDim, int Nx, int Ny, float2* __restrict__ out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long cell = i % Nu;
    long long s = cell % Nx;
    if (imDim > 1) {
      const long long q = cell / Nx;
      s += q % Ny;
      if (imDim > 2) s += q / Ny;
    }
    const float sg = (s & 1) ? -1.f : 1.f;
    out[i] = make_float2(re[i] * sg, (im ? im[i] : 0.f) * sg);
  }
}

__global__ void idf_demodulate_kernel(const float2* __restrict__ in, long long Nu, long long total, int imDim, int Nx,
                                      int Ny, float fac, float* __restrict__ re, float* __restrict__ im) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long cell = i % Nu;
    long long s = cell % Nx;
    if (imDim > 1) {
      const long long q = cell / Nx;
      s += q % Ny;
      if (imDim > 2) s += q / Ny;
    }
    const float f = (s & 1) ? -fac : fac;
    re[i] = in[i].x * f;
    im[i] = in[i].y * f;
  }
}

}  // namespace mlg

extern "C" int mlg_idf(int imDim, const int* N_u, const float* dK_u, int nCol, const float* xR, const float* xI,
                       float* yR, float* yI) {
  MLG_TRY(ensure_device());
  MLG_CHECK(imDim >= 1 && imDim <= 3 && N_u && dK_u && nCol >= 1, "invalid argument");
  MLG_CHECK(xR && yR && yI, "NULL buffer");
  long long Nu = 1;
  float sc = 1.f;
  double dk = 1.0;
  int N[3] = {1, 1, 1};
  for (int d = 0; d < imDim; ++d) {
    MLG_CHECK(N_u[d] >= 2 && !(N_u[d] & 1), "N_u must be even and >= 2");
    N[d] = N_u[d];
    Nu *= N_u[d];
    dk *= dK_u[d];
    if ((N_u[d] / 2) & 1) sc = -sc;
  }
  const long long total = Nu * nCol;
  cudaStream_t s = nullptr;
  DevBuf<float> dxs, dys;
  DevBuf<float2> buf;
  MLG_TRY(dxs.alloc(2 * total, s));
  MLG_TRY(buf.alloc(total, s));
  MLG_TRY(dys.alloc(2 * total, s));
  MLG_CUDA(cudaMemcpyAsync(dxs.p, xR, sizeof(float) * total, cudaMemcpyHostToDevice, s));
  if (xI) MLG_CUDA(cudaMemcpyAsync(dxs.p + total, xI, sizeof(float) * total, cudaMemcpyHostToDevice, s));
  idf_modulate_kernel<<<ew_grid(total), kEwThreads, 0, s>>>(dxs.p, xI ? dxs.p + total : nullptr, Nu, total, imDim,
                                                            N[0], N[1], buf.p);
  MLG_LAUNCHED();
  cufftHandle h;
  int n[3];
  for (int d = 0; d < imDim; ++d) n[d] = N[imDim - 1 - d];
  MLG_CUFFT(cufftPlanMany(&h, imDim, n, nullptr, 1, (int)Nu, nullptr, 1, (int)Nu, CUFFT_C2C, nCol));
  cufftSetStream(h, s);
  cufftResult r = cufftExecC2C(h, (cufftComplex*)buf.p, (cufftComplex*)buf.p, CUFFT_INVERSE);
  count_launch();
  if (r != CUFFT_SUCCESS) {
    cufftDestroy(h);
    return fail(MLG_ERR_CUDA, "idf: cufftExecC2C failed (%d)", (int)r);
  }
  // ifft's 1/prod(N) times the reference's single(prod(N_u)*prod(dK_u))
  const float F = (float)((double)Nu * dk);
  const float fac = (float)(sc * (double)F / (double)Nu);
  idf_demodulate_kernel<<<ew_grid(total), kEwThreads, 0, s>>>(buf.p, Nu, total, imDim, N[0], N[1], fac, dys.p,
                                                              dys.p + total);
  MLG_LAUNCHED();
  MLG_CUDA(cudaMemcpyAsync(yR, dys.p, sizeof(float) * total, cudaMemcpyDeviceToHost, s));
  MLG_CUDA(cudaMemcpyAsync(yI, dys.p + total, sizeof(float) * total, cudaMemcpyDeviceToHost, s));
  MLG_CUDA(cudaStreamSynchronize(s));
  cufftDestroy(h);
  return MLG_OK;
}
