// CG-SENSE on the device: the semantics of
// src/fourier123/solver_function/imDim/nonCartesian/bmSensa.m:6-96.
//
// All step sizes live in device memory as FP64 and every dot product is an
// FP64 sum of per-CTA partials reduced in a fixed order, so one CG step is a
// fixed sequence of launches with no host synchronisation: it is captured
// once into a CUDA graph and replayed.  The reference's early exit
// (sqn < 10*eps('single'), bmSensa.m:54) becomes a device flag that freezes
// the updates of x for the rest of the inner loop.
#include <algorithm>
#include <cfloat>
#include <vector>

#include "mlg_plan.cuh"

namespace mlg {

// device scalar slots
enum : int {
  S_SQN_CURR = 0,  // sqn_dagM_res_curr
  S_SQN_MP = 1,
  S_A = 2,
  S_B = 3,
  S_R = 4,         // monitoring residual
  S_DONE = 5,      // 1.0 once sqn_curr < eps (inner loop stopped)
  S_COUNT = 8
};

constexpr int kT = 256;

static int grid1(long long n) {
  return (int)std::max<long long>(1, std::min<long long>((n + kT - 1) / kT, 148LL * 16));
}

__device__ __forceinline__ double block_reduce(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += sh[i];
  return t;
}

// fixed-order sum of n partials (one CTA)
__device__ double sum_partials(const double* __restrict__ partial, int n, double* sh) {
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) acc += partial[i];
  __shared__ double sh2[kT];
  sh2[threadIdx.x] = acc;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) sh2[threadIdx.x] += sh2[threadIdx.x + w];
    __syncthreads();
  }
  (void)sh;
  return sh2[0];
}

// HY = min(ve, ve_max)   (bmSensa.m:29-32)
__global__ void hy_kernel(const float* __restrict__ ve, int n, float ve_max, float* __restrict__ HY) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) HY[i] = fminf(ve[i], ve_max);
}

// max over v[0..n): each CTA reduces a grid-stride slice into out[blockIdx.x];
// run once with many CTAs, then once with one CTA over those partials
__global__ void max_kernel(const float* __restrict__ v, int n, float* out) {
  __shared__ float sh[kT];
  float m = -FLT_MAX;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) m = fmaxf(m, v[i]);
  sh[threadIdx.x] = m;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) sh[threadIdx.x] = fmaxf(sh[threadIdx.x], sh[threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0) out[blockIdx.x] = sh[0];
}

// res = y - Mx (k-space), optional partials of sum HY |res|^2; y is the
// caller's FP32 data, Mx and res (FP32) the work vectors
__global__ void residual_kernel(const float2* __restrict__ y, const float2* __restrict__ Mx, long long n, int nCh,
                                const float* __restrict__ HY, float2* __restrict__ res, double* partial) {
  __shared__ double sh[kT / 32];
  double sq = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float2 a = y[i], b = Mx[i];
    const float2 r = make_float2(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y));
    if (res) res[i] = r;
    sq += (double)HY[i / nCh] * ((double)r.x * r.x + (double)r.y * r.y);
  }
  if (partial) {
    const double t = block_reduce(sq, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = t;
  }
}

// sqn_curr = HX * sum(partials); done = sqn_curr < eps   (bmSensa.m:45,54)
__global__ void cg_init_kernel(const double* __restrict__ partial, int n, double HX, double eps, double* sc) {
  __shared__ double sh[kT / 32];
  const double s = sum_partials(partial, n, sh);
  if (threadIdx.x == 0) {
    sc[S_SQN_CURR] = HX * s;
    sc[S_DONE] = (HX * s < eps) ? 1.0 : 0.0;
  }
}

// sqn_Mp = sum(partials); a = sqn_curr / sqn_Mp   (bmSensa.m:59-61)
__global__ void cg_alpha_kernel(const double* __restrict__ partial, int n, double* sc) {
  __shared__ double sh[kT / 32];
  const double s = sum_partials(partial, n, sh);
  if (threadIdx.x == 0) {
    sc[S_SQN_MP] = s;
    sc[S_A] = sc[S_DONE] != 0.0 ? 0.0 : sc[S_SQN_CURR] / s;
  }
}

// sqn_next = HX * sum; b = sqn_next / sqn_curr; sqn_curr = sqn_next;
// done once sqn_curr < eps   (bmSensa.m:72-75 and the check of :54)
__global__ void cg_beta_kernel(const double* __restrict__ partial, int n, double HX, double eps, double* sc) {
  __shared__ double sh[kT / 32];
  const double s = sum_partials(partial, n, sh);
  if (threadIdx.x == 0) {
    const double next = HX * s;
    if (sc[S_DONE] == 0.0) {
      sc[S_B] = next / sc[S_SQN_CURR];
      sc[S_SQN_CURR] = next;
      if (next < eps) sc[S_DONE] = 1.0;
    }
  }
}

__global__ void sum_to_slot_kernel(const double* __restrict__ partial, int n, double* sc, int slot) {
  __shared__ double sh[kT / 32];
  const double s = sum_partials(partial, n, sh);
  if (threadIdx.x == 0) sc[slot] = s;
}

// x += a p   (bmSensa.m:63)
__global__ void cg_update_x_kernel(float2* __restrict__ x, const float2* __restrict__ p, long long n,
                                   const double* __restrict__ sc) {
  if (sc[S_DONE] != 0.0) return;
  const float a = (float)sc[S_A];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float2 pv = p[i];
    float2 xv = x[i];
    xv.x = __fadd_rn(xv.x, __fmul_rn(a, pv.x));
    xv.y = __fadd_rn(xv.y, __fmul_rn(a, pv.y));
    x[i] = xv;
  }
}

// res -= a Mp   (bmSensa.m:71); the residual and M p are FP32 complex in
// every precision (M p in scaled FP16 was measured: the store slowed the
// latency-bound Gu gather by more than the halved k-space traffic saved, c2
// mixed 97.3 against 95.6 ms, and raised the image error 1.06e-4 -> 1.33e-4)
__global__ void cg_update_res_kernel(float2* __restrict__ res, const float2* __restrict__ Mp, long long n,
                                     const double* __restrict__ sc) {
  if (sc[S_DONE] != 0.0) return;
  const float a = (float)sc[S_A];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float2 m = Mp[i];
    float2 r = res[i];
    r.x = __fsub_rn(r.x, __fmul_rn(a, m.x));
    r.y = __fsub_rn(r.y, __fmul_rn(a, m.y));
    res[i] = r;
  }
}

static void launch_residual(int g, const float2* y, const float2* Mx, long long n, int nCh, const float* HY,
                            float2* res, double* partial, cudaStream_t s) {
  residual_kernel<<<g, kT, 0, s>>>(y, Mx, n, nCh, HY, res, partial);
}

// p = dagM + b p   (bmSensa.m:77)
__global__ void cg_update_p_kernel(float2* __restrict__ p, const float2* __restrict__ dagM, long long n,
                                   const double* __restrict__ sc) {
  if (sc[S_DONE] != 0.0) return;
  const float b = (float)sc[S_B];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float2 d = dagM[i], pv = p[i];
    p[i] = make_float2(__fadd_rn(d.x, __fmul_rn(b, pv.x)), __fadd_rn(d.y, __fmul_rn(b, pv.y)));
  }
}

static int ensure_solver_buffers(mlg_plan_s* p) {
  if (p->x_p && p->solver_nPt == p->nPt) return MLG_OK;
  cudaFree(p->x_p);
  cudaFree(p->x_dagM);
  cudaFree(p->k_res);
  cudaFree(p->k_Mp);
  cudaFree(p->HY);
  const size_t ni = sizeof(float2) * (size_t)p->nu_tot, nk = sizeof(float2) * (size_t)p->nPt * p->nCh;
  cudaFree(p->mix_amax);
  p->mix_amax = nullptr;
  if (cudaMalloc(&p->x_p, ni) != cudaSuccess || cudaMalloc(&p->x_dagM, ni) != cudaSuccess ||
      cudaMalloc(&p->k_res, nk) != cudaSuccess || cudaMalloc(&p->k_Mp, nk) != cudaSuccess ||
      cudaMalloc(&p->HY, sizeof(float) * (size_t)std::max(1, p->nPt)) != cudaSuccess ||
      cudaMalloc(&p->mix_amax, 2 * sizeof(unsigned)) != cudaSuccess) {
    cudaGetLastError();
    return fail(MLG_ERR_OOM, "solver work buffers: device allocation failed");
  }
  p->solver_nPt = p->nPt;
  p->bytes += 2 * ni + 2 * nk + sizeof(float) * (size_t)p->nPt;
  return MLG_OK;
}

// One inner CG step i < nCGD (bmSensa.m:50-77 without the final break).
static int cg_step(mlg_plan_s* p, float2* x, double HX, double eps, cudaStream_t s) {
  const long long nk = (long long)p->nPt * p->nCh;
  int np = 0;
  MLG_TRY(shanna_run(p, p->x_p, false, p->k_Mp, p->HY, p->partial, &np, s));
  cg_alpha_kernel<<<1, kT, 0, s>>>(p->partial, np, p->scalars);
  MLG_LAUNCHED();
  cg_update_x_kernel<<<grid1(p->nu_tot), kT, 0, s>>>(x, p->x_p, p->nu_tot, p->scalars);
  MLG_LAUNCHED();
  cg_update_res_kernel<<<grid1(nk), kT, 0, s>>>(p->k_res, p->k_Mp, nk, p->scalars);
  MLG_LAUNCHED();
  MLG_TRY(nakatsha_run(p, p->k_res, p->HY, (float)(1.0 / HX), p->x_dagM, p->partial, &np, s));
  cg_beta_kernel<<<1, kT, 0, s>>>(p->partial, np, HX, eps, p->scalars);
  MLG_LAUNCHED();
  cg_update_p_kernel<<<grid1(p->nu_tot), kT, 0, s>>>(p->x_p, p->x_dagM, p->nu_tot, p->scalars);
  MLG_LAUNCHED();
  return MLG_OK;
}

static int sensa_body(mlg_plan_s* p, const float2* y, const float* ve, float ve_max, int nIter, int nCGD, float2* x,
                      double* residual, bool use_graph, cudaStream_t s);

int sensa_run(mlg_plan_s* p, const float2* y, const float* ve, float ve_max, int nIter, int nCGD, float2* x,
              double* residual, bool use_graph, cudaStream_t s) {
  NvtxRange range("CG-SENSE (bmSensa)");
  MLG_CHECK(p->Gu && p->Gut, "CG-SENSE needs a plan with both Gu and Gut");
  MLG_CHECK(nIter >= 0 && nCGD >= 0, "nIter / nCGD must be >= 0");
  p->mixed_run = p->precision == MLG_PRECISION_MIXED;
  const int st = sensa_body(p, y, ve, ve_max, nIter, nCGD, x, residual, use_graph, s);
  p->mixed_run = false;
  p->cg_half = false;
  return st;
}

static int sensa_body(mlg_plan_s* p, const float2* y, const float* ve, float ve_max, int nIter, int nCGD, float2* x,
                      double* residual, bool use_graph, cudaStream_t s) {
  MLG_TRY(ensure_solver_buffers(p));
  const long long nk = (long long)p->nPt * p->nCh;
  const double HX = p->HX;
  const double eps = 10.0 * (double)FLT_EPSILON;  // bmSensa.m:11
  // HY = min(ve, ve_max), ve_max = max(ve) when not given (bmSensa.m:29-32)
  float vmax = ve_max;
  if (!(vmax > 0.f)) {
    float* dmax = (float*)(p->scalars + S_COUNT);
    float* dpart = (float*)p->partial;  // >= 128 doubles of room
    max_kernel<<<128, kT, 0, s>>>(ve, p->nPt, dpart);
    MLG_LAUNCHED();
    max_kernel<<<1, kT, 0, s>>>(dpart, 128, dmax);
    MLG_LAUNCHED();
    MLG_CUDA(cudaMemcpyAsync(&vmax, dmax, sizeof(float), cudaMemcpyDeviceToHost, s));
    MLG_CUDA(cudaStreamSynchronize(s));
  }
  hy_kernel<<<grid1(p->nPt), kT, 0, s>>>(ve, p->nPt, vmax, p->HY);
  MLG_LAUNCHED();

  const int full = std::max(0, nCGD - 1);  // inner steps that run to p_next
  // Captured once per solution buffer, after the first init phase has run
  // every kernel of the step at least once (first launches set kernel
  // attributes, which must not happen during capture).
  auto ensure_graph = [&]() -> int {
    if (!use_graph || full == 0 || (p->cg_graph && p->cg_graph_x == x && p->cg_graph_prec == (int)p->mixed_run))
      return MLG_OK;
    if (p->cg_graph) cudaGraphExecDestroy(p->cg_graph);
    p->cg_graph = nullptr;
    cudaGraph_t graph;
    MLG_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    const long long before = g_launches.load();
    const int st = cg_step(p, x, HX, eps, s);
    const cudaError_t ce = cudaStreamEndCapture(s, &graph);
    p->cg_graph_kernels = g_launches.load() - before;
    g_launches.fetch_sub(p->cg_graph_kernels);  // captured, not launched
    if (st != MLG_OK) return st;
    if (ce != cudaSuccess) return fail(MLG_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(ce));
    const cudaError_t ie = cudaGraphInstantiate(&p->cg_graph, graph, 0);
    cudaGraphDestroy(graph);
    if (ie != cudaSuccess) return fail(MLG_ERR_CUDA, "graph instantiate failed: %s", cudaGetErrorString(ie));
    p->cg_graph_x = x;
    p->cg_graph_prec = (int)p->mixed_run;
    return MLG_OK;
  };

  DevBuf<double> hist;
  MLG_TRY(hist.alloc(std::max(1, nIter), s));
  for (int it = 0; it < nIter; ++it) {
    // res = y - M x; dagM = (1/HX) M*(HY res); sqn = HX |dagM|^2; p = dagM
    int np = 0;
    p->cg_half = false;  // M x of the residual and of the monitoring: FP32 transforms
    MLG_TRY(shanna_run(p, x, false, p->k_Mp, nullptr, nullptr, nullptr, s));
    launch_residual(grid1(nk), y, p->k_Mp, nk, p->nCh, p->HY, p->k_res, nullptr, s);
    MLG_LAUNCHED();
    MLG_TRY(nakatsha_run(p, p->k_res, p->HY, (float)(1.0 / HX), p->x_dagM, p->partial, &np, s));
    cg_init_kernel<<<1, kT, 0, s>>>(p->partial, np, HX, eps, p->scalars);
    MLG_LAUNCHED();
    MLG_CUDA(cudaMemcpyAsync(p->x_p, p->x_dagM, sizeof(float2) * (size_t)p->nu_tot, cudaMemcpyDeviceToDevice, s));
    p->cg_half = p->mixed_run;  // the CG steps: FP16 transform intermediate where supported
    if (full > 0) MLG_TRY(ensure_graph());
    for (int i = 0; i < full; ++i) {
      if (use_graph) {
        MLG_CUDA(cudaGraphLaunch(p->cg_graph, s));
        count_launch(p->cg_graph_kernels);
      } else {
        MLG_TRY(cg_step(p, x, HX, eps, s));
      }
    }
    if (nCGD > 0) {  // the last step stops after x += a p (bmSensa.m:67-69)
      MLG_TRY(shanna_run(p, p->x_p, false, p->k_Mp, p->HY, p->partial, &np, s));
      cg_alpha_kernel<<<1, kT, 0, s>>>(p->partial, np, p->scalars);
      MLG_LAUNCHED();
      cg_update_x_kernel<<<grid1(p->nu_tot), kT, 0, s>>>(x, p->x_p, p->nu_tot, p->scalars);
      MLG_LAUNCHED();
    }
    // monitoring: R = |y - Mx|^2_HY   (bmSensa.m:82-83)
    p->cg_half = false;
    MLG_TRY(shanna_run(p, x, false, p->k_Mp, nullptr, nullptr, nullptr, s));
    const int g = grid1(nk);
    launch_residual(g, y, p->k_Mp, nk, p->nCh, p->HY, nullptr, p->partial, s);
    MLG_LAUNCHED();
    sum_to_slot_kernel<<<1, kT, 0, s>>>(p->partial, g, hist.p, it);
    MLG_LAUNCHED();
  }
  if (residual && nIter > 0) {
    MLG_CUDA(cudaMemcpyAsync(residual, hist.p, sizeof(double) * nIter, cudaMemcpyDeviceToHost, s));
    MLG_CUDA(cudaStreamSynchronize(s));
  }
  return MLG_OK;
}

}  // namespace mlg

using namespace mlg;

extern "C" {

int mlg_plan_set_dk(mlg_plan_t p, const double* dK_u) {
  MLG_CHECK(p && dK_u, "NULL argument");
  double hx = 1.0;
  float dx[3] = {1.f, 1.f, 1.f};
  for (int d = 0; d < p->imDim; ++d) {
    MLG_CHECK(dK_u[d] > 0, "dK_u must be > 0");
    // single-precision arithmetic of bmSensa.m:26-27
    dx[d] = (1.0f / (float)dK_u[d]) / (float)p->N[d];
    hx = (double)((float)hx * dx[d]);
  }
  p->HX = hx;
  for (int d = 0; d < 3; ++d) p->dX[d] = dx[d];
  return MLG_OK;
}

int mlg_sensa_dev(mlg_plan_t p, const void* y, const float* ve, float ve_max, int nIter, int nCGD, void* x,
                  double* residual, void* stream) {
  MLG_CHECK(p && y && ve && x, "NULL argument");
  MLG_CUDA(cudaSetDevice(p->device));
  cudaStream_t user = (cudaStream_t)stream;
  MLG_CUDA(cudaEventRecord(p->ev_in, user));
  MLG_CUDA(cudaStreamWaitEvent(p->stream, p->ev_in, 0));
  int st = sensa_run(p, (const float2*)y, ve, ve_max, nIter, nCGD, (float2*)x, residual, true, p->stream);
  cudaEventRecord(p->ev_out, p->stream);
  cudaStreamWaitEvent(user, p->ev_out, 0);
  return st;
}

int mlg_sensa(mlg_plan_t p, const float* yR, const float* yI, const float* ve, float ve_max, int nIter, int nCGD,
              float* xR, float* xI, double* residual) {
  MLG_CHECK(p && yR && yI && ve && xR && xI, "NULL argument");
  MLG_CUDA(cudaSetDevice(p->device));
  cudaStream_t s = p->stream;
  const long long nk = (long long)p->nPt * p->nCh, nx = p->nu_tot;
  DevBuf<float> dy, dve, dx;
  DevBuf<float2> y2, x2;
  MLG_TRY(dy.alloc(2 * nk, s));
  MLG_TRY(dve.alloc(p->nPt, s));
  MLG_TRY(dx.alloc(2 * nx, s));
  MLG_TRY(y2.alloc(nk, s));
  MLG_TRY(x2.alloc(nx, s));
  MLG_CUDA(cudaMemcpyAsync(dy.p, yR, sizeof(float) * nk, cudaMemcpyHostToDevice, s));
  MLG_CUDA(cudaMemcpyAsync(dy.p + nk, yI, sizeof(float) * nk, cudaMemcpyHostToDevice, s));
  MLG_CUDA(cudaMemcpyAsync(dve.p, ve, sizeof(float) * p->nPt, cudaMemcpyHostToDevice, s));
  MLG_CUDA(cudaMemcpyAsync(dx.p, xR, sizeof(float) * nx, cudaMemcpyHostToDevice, s));
  MLG_CUDA(cudaMemcpyAsync(dx.p + nx, xI, sizeof(float) * nx, cudaMemcpyHostToDevice, s));
  MLG_TRY(mlg::pack_col_to_point(dy.p, dy.p + nk, p->nPt, p->nCh, y2.p, s));
  MLG_TRY(mlg::interleave(dx.p, dx.p + nx, nx, x2.p, s));
  MLG_TRY(sensa_run(p, y2.p, dve.p, ve_max, nIter, nCGD, x2.p, residual, true, s));
  MLG_TRY(mlg::deinterleave(x2.p, nx, dx.p, dx.p + nx, s));
  MLG_CUDA(cudaMemcpyAsync(xR, dx.p, sizeof(float) * nx, cudaMemcpyDeviceToHost, s));
  MLG_CUDA(cudaMemcpyAsync(xI, dx.p + nx, sizeof(float) * nx, cudaMemcpyDeviceToHost, s));
  MLG_CUDA(cudaStreamSynchronize(s));
  return mlg::fft_wait_status(p->wait_err, s);
}

}  // extern "C"

// ---- stage timing -------------------------------------------------------------
extern "C" int mlg_plan_profile(mlg_plan_t p, int iters, double* ms) {
  using namespace mlg;
  MLG_CHECK(p && ms && iters >= 1, "invalid argument");
  MLG_CHECK(p->Gu && p->Gut, "profiling needs a plan with both Gu and Gut");
  MLG_CUDA(cudaSetDevice(p->device));
  MLG_TRY(ensure_solver_buffers(p));
  cudaStream_t s = p->stream;
  const long long nk = (long long)p->nPt * p->nCh;
  MLG_CUDA(cudaMemsetAsync(p->x_p, 0, sizeof(float2) * (size_t)p->nu_tot, s));
  MLG_CUDA(cudaMemsetAsync(p->k_res, 0, sizeof(float2) * (size_t)nk, s));
  // a mixed plan's stages as they run inside its CG steps (the FP16
  // transform intermediate, where supported)
  constexpr int S = kShannaStages + kNakatshaStages;
  cudaEvent_t ev[S + 1];
  for (int k = 0; k <= S; ++k) MLG_CUDA(cudaEventCreate(&ev[k]));
  p->cg_half = p->precision == MLG_PRECISION_MIXED;  // reset below on every path
  double acc[S] = {0};
  int st = MLG_OK;
  for (int it = 0; it <= iters && st == MLG_OK; ++it) {
    cudaEventRecord(ev[0], s);
    for (int k = 0; k < kShannaStages && st == MLG_OK; ++k) {
      st = shanna_stage(p, k, p->x_p, false, p->k_Mp, nullptr, nullptr, nullptr, s);
      cudaEventRecord(ev[k + 1], s);
    }
    for (int k = 0; k < kNakatshaStages && st == MLG_OK; ++k) {
      st = nakatsha_stage(p, k, p->k_res, nullptr, 1.0f, p->x_dagM, nullptr, nullptr, s);
      cudaEventRecord(ev[kShannaStages + k + 1], s);
    }
    if (cudaStreamSynchronize(s) != cudaSuccess) st = fail(MLG_ERR_CUDA, "profile run failed");
    if (it == 0 || st != MLG_OK) continue;  // first run is the warm-up
    for (int k = 0; k < S; ++k) {
      float v = 0.f;
      cudaEventElapsedTime(&v, ev[k], ev[k + 1]);
      acc[k] += v;
    }
  }
  p->cg_half = false;
  for (int k = 0; k <= S; ++k) cudaEventDestroy(ev[k]);
  for (int k = 0; k < S; ++k) ms[k] = acc[k] / iters;
  return st;
}

// ---- adjoint strategy and autotuner ------------------------------------------
extern "C" int mlg_plan_set_adjoint(mlg_plan_t p, int mode) {
  using namespace mlg;
  MLG_CHECK(p, "NULL plan");
  MLG_CHECK(adjoint_mode_valid(p, mode), "adjoint strategy %d not available for this plan", mode);
  if (p->adjoint_mode != mode) {
    p->adjoint_mode = mode;
    if (p->cg_graph) cudaGraphExecDestroy(p->cg_graph);  // captured with the old strategy
    p->cg_graph = nullptr;
    p->cg_graph_x = nullptr;
  }
  return MLG_OK;
}

extern "C" int mlg_plan_get_adjoint(mlg_plan_t p, int* mode) {
  MLG_CHECK(p && mode, "NULL argument");
  *mode = p->adjoint_mode;
  return MLG_OK;
}

extern "C" int mlg_plan_autotune(mlg_plan_t p, int reps, double* ms) {
  using namespace mlg;
  MLG_CHECK(p && reps >= 1, "invalid argument");
  MLG_CHECK(p->Gut, "autotuning needs a plan with Gut");
  MLG_CUDA(cudaSetDevice(p->device));
  MLG_TRY(ensure_solver_buffers(p));
  cudaStream_t s = p->stream;
  MLG_CUDA(cudaMemsetAsync(p->k_res, 0, sizeof(float2) * (size_t)p->nPt * p->nCh, s));
  cudaEvent_t a, b;
  MLG_CUDA(cudaEventCreate(&a));
  MLG_CUDA(cudaEventCreate(&b));
  const int orig = p->adjoint_mode;
  int best = orig;
  double best_ms = 1e30;
  int st = MLG_OK;
  for (int mode = 0; mode < 3 && st == MLG_OK; ++mode) {
    double t = -1.0;
    if (adjoint_mode_valid(p, mode)) {
      p->adjoint_mode = mode;
      st = nakatsha_run(p, p->k_res, nullptr, 1.0f, p->x_dagM, nullptr, nullptr, s);  // warm-up
      cudaEventRecord(a, s);
      for (int r = 0; r < reps && st == MLG_OK; ++r)
        st = nakatsha_run(p, p->k_res, nullptr, 1.0f, p->x_dagM, nullptr, nullptr, s);
      cudaEventRecord(b, s);
      if (cudaEventSynchronize(b) != cudaSuccess) st = fail(MLG_ERR_CUDA, "autotune run failed");
      float v = 0.f;
      cudaEventElapsedTime(&v, a, b);
      t = v / reps;
      if (st == MLG_OK && t < best_ms) {
        best_ms = t;
        best = mode;
      }
    }
    if (ms) ms[mode] = t;
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  p->adjoint_mode = orig;
  if (st != MLG_OK) return st;
  return mlg_plan_set_adjoint(p, best);
}

extern "C" int mlg_plan_set_variant(mlg_plan_t p, int pass_buffers, int gut_records, int fwd_masked_store) {
  using namespace mlg;
  MLG_CHECK(p, "NULL plan");
  MLG_CHECK((pass_buffers == 0 || pass_buffers == 2 || pass_buffers == 3) && (gut_records == 0 || gut_records == 1) &&
                (fwd_masked_store == 0 || fwd_masked_store == 1),
            "variants: pass_buffers 0, 2 or 3; gut_records 0 or 1; fwd_masked_store 0 or 1");
  MLG_CHECK(!gut_records || p->Gut_s.ord_rec, "this plan has no Gut row records (masked adjoint, even coil count)");
  MLG_CHECK(!fwd_masked_store || p->gu_covered,
            "this plan cannot mask its forward stores (no line masks, or a Gu column outside Gut's occupied cells)");
  if (p->pass_buffers != pass_buffers || p->gut_records != gut_records || p->fwd_masked_store != fwd_masked_store) {
    p->pass_buffers = pass_buffers;
    p->gut_records = gut_records;
    p->fwd_masked_store = fwd_masked_store;
    if (p->cg_graph) cudaGraphExecDestroy(p->cg_graph);  // captured with the old kernels
    p->cg_graph = nullptr;
    p->cg_graph_x = nullptr;
  }
  return MLG_OK;
}

extern "C" int mlg_plan_get_variant(mlg_plan_t p, int* pass_buffers, int* gut_records, int* fwd_masked_store) {
  MLG_CHECK(p && pass_buffers && gut_records && fwd_masked_store, "NULL argument");
  *pass_buffers = p->pass_buffers;
  *gut_records = p->gut_records;
  *fwd_masked_store = p->fwd_masked_store;
  return MLG_OK;
}

// Times the kernel variants of the plan's current adjoint strategy and keeps
// the fastest: ms[0..2] = forward + adjoint with TMA passes over 2 / 3
// buffers and with cp.async passes (masked forward stores where the plan
// allows them), ms[3..4] = adjoint with Gut from the CSR / from row records,
// ms[5] = forward + adjoint storing every chunk of the grid, at the chosen
// buffer count (-1: not available).
extern "C" int mlg_plan_autotune_variants(mlg_plan_t p, int reps, double* ms) {
  using namespace mlg;
  MLG_CHECK(p && reps >= 1, "invalid argument");
  MLG_CHECK(p->Gu && p->Gut, "variant tuning needs a plan with Gu and Gut");
  MLG_CUDA(cudaSetDevice(p->device));
  MLG_TRY(ensure_solver_buffers(p));
  cudaStream_t s = p->stream;
  MLG_CUDA(cudaMemsetAsync(p->k_res, 0, sizeof(float2) * (size_t)p->nPt * p->nCh, s));
  MLG_CUDA(cudaMemsetAsync(p->x_p, 0, sizeof(float2) * (size_t)p->nu_tot, s));
  cudaEvent_t a, b;
  MLG_CUDA(cudaEventCreate(&a));
  MLG_CUDA(cudaEventCreate(&b));
  int st = MLG_OK;
  auto time_it = [&](bool fwd) {
    auto once = [&] {
      if (fwd && st == MLG_OK) st = shanna_run(p, p->x_p, false, p->k_Mp, nullptr, nullptr, nullptr, s);
      if (st == MLG_OK) st = nakatsha_run(p, p->k_res, nullptr, 1.0f, p->x_dagM, nullptr, nullptr, s);
    };
    once();  // warm-up
    cudaEventRecord(a, s);
    for (int r = 0; r < reps && st == MLG_OK; ++r) once();
    cudaEventRecord(b, s);
    if (cudaEventSynchronize(b) != cudaSuccess) st = fail(MLG_ERR_CUDA, "variant tuning run failed");
    float v = 0.f;
    cudaEventElapsedTime(&v, a, b);
    return (double)v / reps;
  };
  const int buf0 = p->pass_buffers, rec0 = p->gut_records, mask0 = p->fwd_masked_store;
  double t[6] = {-1.0, -1.0, -1.0, -1.0, -1.0, -1.0};
  int best_buf = buf0, best_rec = rec0, best_mask = mask0;
  p->fwd_masked_store = p->gu_covered ? 1 : 0;
  double best_fwd = -1.0;
  if (tma_passes_enabled()) {
    const int opts[3] = {2, 3, 0};
    double best = 1e30;
    for (int i = 0; i < 3 && st == MLG_OK; ++i) {
      p->pass_buffers = opts[i];
      t[i] = time_it(true);
      if (t[i] < best) {
        best = t[i];
        best_buf = opts[i];
      }
    }
    best_fwd = best;
  }
  p->pass_buffers = best_buf;
  best_mask = p->fwd_masked_store;
  if (st == MLG_OK && p->gu_covered && best_buf >= 2 && best_fwd > 0.0) {
    p->fwd_masked_store = 0;
    t[5] = time_it(true);
    best_mask = t[5] < best_fwd ? 0 : 1;
  }
  p->fwd_masked_store = best_mask;
  if (st == MLG_OK && p->Gut_s.ord_rec && p->adjoint_mode == 2) {
    double best = 1e30;
    for (int v = 0; v <= 1 && st == MLG_OK; ++v) {
      p->gut_records = v;
      t[3 + v] = time_it(false);
      if (t[3 + v] < best) {
        best = t[3 + v];
        best_rec = v;
      }
    }
  }
  p->pass_buffers = buf0;
  p->gut_records = rec0;
  p->fwd_masked_store = mask0;
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (ms)
    for (int i = 0; i < 6; ++i) ms[i] = t[i];
  if (st != MLG_OK) return st;
  return mlg_plan_set_variant(p, best_buf, best_rec, best_mask);
}

extern "C" int mlg_plan_set_precision(mlg_plan_t p, int precision) {
  using namespace mlg;
  MLG_CHECK(p, "NULL plan");
  MLG_CHECK(precision == MLG_PRECISION_FP32 || precision == MLG_PRECISION_MIXED ||
                precision == MLG_PRECISION_FP16_VALUES,
            "unknown precision %d", precision);
  MLG_CUDA(cudaSetDevice(p->device));
  if (precision != MLG_PRECISION_FP32) {
    MLG_CHECK(p->Gu && p->Gut, "mixed precision needs a plan with both Gu and Gut");
    MLG_TRY(csr_make_half(p->Gu_s, p->stream));
    MLG_TRY(csr_make_half(p->Gut_s, p->stream));
    MLG_CUDA(cudaStreamSynchronize(p->stream));
  }
  p->precision = precision;
  if (!adjoint_mode_valid(p, p->adjoint_mode))  // the fused gather reads FP32 k-space
    p->adjoint_mode = adjoint_mode_valid(p, 2) ? 2 : 0;
  if (p->cg_graph) cudaGraphExecDestroy(p->cg_graph);
  p->cg_graph = nullptr;
  p->cg_graph_x = nullptr;
  return MLG_OK;
}

extern "C" int mlg_plan_get_precision(mlg_plan_t p, int* precision) {
  MLG_CHECK(p && precision, "NULL argument");
  *precision = p->precision;
  return MLG_OK;
}

extern "C" int mlg_plan_get_half_intermediate(mlg_plan_t p, int* on) {
  MLG_CHECK(p && on, "NULL argument");
  *on = 0;
  if (p->precision == MLG_PRECISION_MIXED && half_intermediate_possible(p)) *on = 1 | (p->half_g_ok ? 2 : 0);
  return MLG_OK;
}
