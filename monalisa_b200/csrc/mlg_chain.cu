// TV-regularised ADMM reconstructions on the device:
//  * temporal TV over frame bins, the semantics of
//    src/fourier123/solver_function/imDim_morphosia/nonCartesian/
//    bmTevaMorphosia_chain.m:6-195 with Tu = Tut = [] (identity deformation);
//  * spatial TV of one image, the semantics of
//    src/fourier123/solver_function/imDim/nonCartesian/bmSteva.m:6-138
//    (a chain of one frame whose sparsifier is the backward gradient,
//    src/optim/bmBackGradient_n.m / bmBackGradient_nT.m).
// Both share the CG/ADMM skeleton below; bmTevaMorphosia_chain.m line
// numbers are cited as ":n", bmSteva.m ones by name.
//
// Frame f has its own trajectory (plan f: Gu{f}, Gut{f}, k-space rows
// y{f}, weights ve{f}); all frames share the grid, image size, coils and KFC.
// Images of all frames are one array [nFr][prod(n_u)] and the k-space rows
// of all frames one array [sum nPt_f][nCh], so every BLAS-1 step, the
// sparsifier F x_f = x_f - x_{f-1} (circular, :266-272) and its adjoint
// (:285-291), the z/u update and every norm run as one launch over all
// frames; only the operators run per frame.
//
// Scalars (step sizes, norms, delta, rho, the early-exit flag) live in
// device memory as FP64, each norm an FP64 sum of per-CTA partials in a
// fixed order.  A CG step therefore needs no host synchronisation; the
// inner step is captured once into a CUDA graph and replayed.
//
// The monitoring residual y - M x computed at the end of an ADMM iteration
// (:174, private_dafi_regul :211-224) is, bit for bit, the residual the next
// iteration starts from (:117): it is computed once and kept.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <vector>

#include "mlg_plan.cuh"

// image geometry of the spatial sparsifier: extents, element strides and
// pixel sizes dX_u along each axis (column-major image)
struct ImGeom {
  int dim = 1;
  int n[3] = {1, 1, 1};
  long long st[3] = {1, 1, 1};
  float dX[3] = {1.f, 1.f, 1.f};
};

struct mlg_chain_s {
  int device = 0;
  int nFr = 0;
  int nCh = 1;
  long long nu = 0;                 // pixels per frame
  ImGeom geom;
  long long nd_cap = 0;             // rows of the dual arrays: max(nFr, imDim)
  bool spatial = false;             // the run in progress: bmSteva (true) or the temporal chain
  std::vector<mlg_plan_s*> fr;      // caller's plans, one per frame
  std::vector<long long> row_off;   // first k-space row of each frame
  long long rows = 0;               // sum of nPt over frames
  double HX = 1.0;
  // work arrays
  float2 *p = nullptr, *dA = nullptr;                                     // [nFr][nu]
  float2 *res_z = nullptr, *Fp = nullptr;                                 // [nd_cap][nu]
  float2 *z = nullptr, *u = nullptr;                                      // host-API z, u [nd_cap][nu]
  float2 *res_y = nullptr, *Mp = nullptr;                                 // [rows][nCh]
  float* HY = nullptr;                                                    // [rows]
  double* partial = nullptr;
  int partial_cap = 0;
  double* sc = nullptr;       // scalar slots
  double* lists = nullptr;    // delta list, rho list [2][nIter_cap]
  int lists_cap = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  cudaGraphExec_t graph = nullptr;
  const void* graph_key[4] = {nullptr, nullptr, nullptr, nullptr};
  std::vector<int> graph_modes;     // sparsifier and the frames' adjoint strategies it was captured with
  long long graph_kernels = 0;
  // deformation fields of the temporal sparsifier (caller's matrices, one
  // per frame, NULL = identity): F x_f = Tu_f x_f - x_{f-1}, F* z_f =
  // (1/HX)(Tut_f (HZ z_f) - HZ z_{f+1})
  std::vector<const mlg::Csr*> Tu, Tut;
  bool deform = false;
  float2 *Dx = nullptr, *Sz = nullptr;  // [nFr][nu]: deformed frames; HZ res_z
  float* dscratch = nullptr;            // long-row segment scratch of those products
};

namespace mlg {

enum : int {
  T_SQ_CURR = 0,  // sqn_dagA_res_curr
  T_SQ_MP = 1,
  T_SQ_FP = 2,
  T_A = 3,
  T_B = 4,
  T_DONE = 5,     // 1 once sqn_curr < eps: the CG loop has stopped
  T_DELTA = 6,
  T_RHO = 7,
  T_DAFI = 8,     // monitoring, latest
  T_REGUL = 9,
  T_ITER = 10,    // ADMM iteration index (0-based) the lists are read at
  T_COUNT = 16
};

constexpr int kT = 256;

static int grid1(long long n) {
  return (int)std::max<long long>(1, std::min<long long>((n + kT - 1) / kT, 148LL * 8));
}

__device__ __forceinline__ double block_sum(double v) {
  __shared__ double sh[kT / 32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += sh[i];
  return t;
}

// fixed-order sum of partial[lo, hi) by one CTA
__device__ double sum_range(const double* __restrict__ partial, int lo, int hi) {
  __shared__ double sh[kT];
  double acc = 0.0;
  for (int i = lo + (int)threadIdx.x; i < hi; i += blockDim.x) acc += partial[i];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  const double r = sh[0];
  __syncthreads();
  return r;
}

__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y)); }
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y)); }
__device__ __forceinline__ double nrm2(float2 a) { return (double)a.x * a.x + (double)a.y * a.y; }

// HY = min(ve, ve_max)   (private_ve_to_HY, :201-209)
__global__ void tv_hy_kernel(const float* __restrict__ ve, long long n, float ve_max, float* __restrict__ HY) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    HY[i] = fminf(ve[i], ve_max);
}

// In the temporal-TV kernels xd is the deformed current frame (Tu_f x_f,
// private_F :262-269 via bmImDeform), x itself without deformation fields.

// z = F x, u = 0   (:75-81)
__global__ void tv_init_zu_kernel(const float2* __restrict__ x, const float2* __restrict__ xd, int nFr, long long nu,
                                  float2* __restrict__ z, float2* __restrict__ u) {
  const long long n = nu * nFr;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const long long f = i / nu, k = i - f * nu;
    const long long prev = ((f + nFr - 1) % nFr) * nu + k;
    z[i] = csub(xd[i], x[prev]);
    u[i] = make_float2(0.f, 0.f);
  }
}

// Sz = HZ res_z (the input of Tut_f in private_dagF :282-289)
__global__ void tv_scale_kernel(const float2* __restrict__ v, long long n, float HZ, float2* __restrict__ out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float2 a = v[i];
    out[i] = make_float2(__fmul_rn(HZ, a.x), __fmul_rn(HZ, a.y));
  }
}

// delta and rho of ADMM iteration T_ITER (:104-110): the lists, or in the
// 'adapt' mode delta = delta_factor * regul / dafi, rho = rho_factor * delta
// (private_adapt_delta_rho, :240-248)
__global__ void tv_params_kernel(const double* __restrict__ lists, int cap, int adapt, double* sc) {
  const int c = (int)sc[T_ITER];
  const float dl = (float)lists[c], rl = (float)lists[cap + c];
  float d = dl, r = rl;
  if (adapt) {
    d = (float)((double)dl * (float)sc[T_REGUL] / (float)sc[T_DAFI]);
    r = rl * d;
  }
  sc[T_DELTA] = d;
  sc[T_RHO] = r;
}

// res_z = (z - u) - F x   (:118)
__global__ void tv_res_z_kernel(const float2* __restrict__ x, const float2* __restrict__ xd,
                                const float2* __restrict__ z, const float2* __restrict__ u, int nFr, long long nu,
                                float2* __restrict__ res_z) {
  const long long n = nu * nFr;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const long long f = i / nu, k = i - f * nu;
    const long long prev = ((f + nFr - 1) % nFr) * nu + k;
    res_z[i] = csub(csub(z[i], u[i]), csub(xd[i], x[prev]));
  }
}

// dA = dA + rho * (1/HX) (HZ res_z_f - HZ res_z_{f+1}), with dA holding
// (1/HX) M*(HY res_y) from the operators (:119-121); partials of |dA|^2.
// ts (optional): Tut_f (HZ res_z_f), taken in place of HZ res_z_f.
__global__ void tv_dA_kernel(float2* __restrict__ dA, const float2* __restrict__ res_z,
                             const float2* __restrict__ ts, int nFr, long long nu, float HZ, float invHX,
                             const double* __restrict__ sc, double* __restrict__ partial) {
  const float rho = (float)sc[T_RHO];
  const long long n = nu * nFr;
  double acc = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const long long f = i / nu, k = i - f * nu;
    const long long next = ((f + 1) % nFr) * nu + k;
    const float2 b = res_z[next];
    float2 a;
    if (ts) {
      a = ts[i];
    } else {
      const float2 r = res_z[i];
      a = make_float2(__fmul_rn(HZ, r.x), __fmul_rn(HZ, r.y));
    }
    float2 t = make_float2(__fsub_rn(a.x, __fmul_rn(HZ, b.x)), __fsub_rn(a.y, __fmul_rn(HZ, b.y)));
    t = make_float2(__fmul_rn(rho, __fmul_rn(invHX, t.x)), __fmul_rn(rho, __fmul_rn(invHX, t.y)));
    const float2 v = cadd(dA[i], t);
    dA[i] = v;
    acc += nrm2(v);
  }
  const double s = block_sum(acc);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// sqn_dagA_res = HX * |dA|^2 (:123); the first CG check (:133-135)
__global__ void tv_sq_init_kernel(const double* __restrict__ partial, int n, double HX, double eps, double* sc) {
  const double s = sum_range(partial, 0, n);
  if (threadIdx.x == 0) {
    sc[T_SQ_CURR] = HX * s;
    sc[T_DONE] = (HX * s < eps) ? 1.0 : 0.0;
  }
}

// Fp = F p with partials of |Fp|^2 (pd: the deformed current frame of p)
__global__ void tv_Fp_kernel(const float2* __restrict__ p, const float2* __restrict__ pd, int nFr, long long nu,
                             float2* __restrict__ Fp, double* __restrict__ partial) {
  const long long n = nu * nFr;
  double acc = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const long long f = i / nu, k = i - f * nu;
    const long long prev = ((f + nFr - 1) % nFr) * nu + k;
    const float2 v = csub(pd[i], p[prev]);
    Fp[i] = v;
    acc += nrm2(v);
  }
  const double s = block_sum(acc);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// a = sqn_curr / (|Mp|^2_HY + rho HZ |Fp|^2)   (:140-146)
__global__ void tv_alpha_kernel(const double* __restrict__ partial, int n_mp, int n_fp, double HZ, double* sc) {
  const double smp = sum_range(partial, 0, n_mp);
  const double sfp = sum_range(partial, n_mp, n_mp + n_fp);
  if (threadIdx.x == 0) {
    const double rhz = (double)((float)sc[T_RHO] * (float)HZ);
    sc[T_SQ_MP] = smp;
    sc[T_SQ_FP] = rhz * sfp;
    sc[T_A] = sc[T_DONE] != 0.0 ? 0.0 : sc[T_SQ_CURR] / (smp + rhz * sfp);
  }
}

// sqn_next = HX |dA|^2; b = sqn_next / sqn_curr (:159-160); stop check (:133)
__global__ void tv_beta_kernel(const double* __restrict__ partial, int n, double HX, double eps, double* sc) {
  const double s = sum_range(partial, 0, n);
  if (threadIdx.x == 0 && sc[T_DONE] == 0.0) {
    const double next = HX * s;
    sc[T_B] = next / sc[T_SQ_CURR];
    sc[T_SQ_CURR] = next;
    if (next < eps) sc[T_DONE] = 1.0;
  }
}

// v += a w   (x update :147; res_y / res_z updates :154-155 with v -= a w)
template <bool MINUS>
__global__ void tv_axpy_kernel(float2* __restrict__ v, const float2* __restrict__ w, long long n,
                               const double* __restrict__ sc) {
  if (sc[T_DONE] != 0.0) return;
  const float a = (float)sc[T_A];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float2 wv = w[i];
    float2 x = v[i];
    if (MINUS) {
      x.x = __fsub_rn(x.x, __fmul_rn(a, wv.x));
      x.y = __fsub_rn(x.y, __fmul_rn(a, wv.y));
    } else {
      x.x = __fadd_rn(x.x, __fmul_rn(a, wv.x));
      x.y = __fadd_rn(x.y, __fmul_rn(a, wv.y));
    }
    v[i] = x;
  }
}

// p = dA + b p   (:161)
__global__ void tv_update_p_kernel(float2* __restrict__ p, const float2* __restrict__ dA, long long n,
                                   const double* __restrict__ sc) {
  if (sc[T_DONE] != 0.0) return;
  const float b = (float)sc[T_B];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float2 d = dA[i], pv = p[i];
    p[i] = make_float2(__fadd_rn(d.x, __fmul_rn(b, pv.x)), __fadd_rn(d.y, __fmul_rn(b, pv.y)));
  }
}

// soft threshold of one part (src/.../linSpace/bmProx_oneNorm.m:24-40)
__device__ __forceinline__ float soft(float w, float s) {
  return w > s ? __fsub_rn(w, s) : (w < -s ? __fadd_rn(w, s) : 0.f);
}

// Fxu = u + F x; z = prox(Fxu, delta/rho); u = Fxu - z   (:167-169)
__global__ void tv_zu_kernel(const float2* __restrict__ x, const float2* __restrict__ xd, int nFr, long long nu,
                             float2* __restrict__ z, float2* __restrict__ u, const double* __restrict__ sc) {
  const float s = fabsf(__fdiv_rn((float)sc[T_DELTA], (float)sc[T_RHO]));
  const long long n = nu * nFr;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const long long f = i / nu, k = i - f * nu;
    const long long prev = ((f + nFr - 1) % nFr) * nu + k;
    const float2 w = cadd(u[i], csub(xd[i], x[prev]));
    const float2 zz = make_float2(soft(w.x, s), soft(w.y, s));
    z[i] = zz;
    u[i] = csub(w, zz);
  }
}

// res = y - Mx over all frames' rows, partials of sum HY |res|^2
__global__ void tv_residual_kernel(const float2* __restrict__ y, const float2* __restrict__ Mx, long long n, int nCh,
                                   const float* __restrict__ HY, float2* __restrict__ res, double* __restrict__ partial) {
  double acc = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float2 r = csub(y[i], Mx[i]);
    res[i] = r;
    acc += (double)HY[i / nCh] * nrm2(r);
  }
  const double s = block_sum(acc);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// partials of sum |Re(x_{f-1} - Tu_f x_f)| + |Im(...)|   (:219-222)
__global__ void tv_regul_kernel(const float2* __restrict__ x, const float2* __restrict__ xd, int nFr, long long nu,
                                double* __restrict__ partial) {
  const long long n = nu * nFr;
  double acc = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const long long f = i / nu, k = i - f * nu;
    const long long prev = ((f + nFr - 1) % nFr) * nu + k;
    const float2 t = csub(x[prev], xd[i]);
    acc += (double)fabsf(t.x) + (double)fabsf(t.y);
  }
  const double s = block_sum(acc);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// dafi, regul; with hstride 3: objective = 0.5 dafi + 0.5 delta regul,
// dafi, regul into hist[3c..3c+2] (:174-179); with hstride 2 (bmSteva.m:
// 117-125): R, TV into hist[2c..2c+1].  Only the slots when hist is NULL
// (the initial monitoring).
__global__ void tv_monitor_kernel(const double* __restrict__ partial, int n_res, int n_reg, double HZ, double* sc,
                                  double* hist, int hstride) {
  const double dafi = sum_range(partial, 0, n_res);
  const double reg = HZ * sum_range(partial, n_res, n_res + n_reg);
  if (threadIdx.x == 0) {
    sc[T_DAFI] = dafi;
    sc[T_REGUL] = reg;
    if (hist) {
      const int c = (int)sc[T_ITER];
      double* h = hist + (size_t)hstride * c;
      if (hstride == 3) *h++ = 0.5 * dafi + 0.5 * sc[T_DELTA] * reg;
      h[0] = dafi;
      h[1] = reg;
      sc[T_ITER] = c + 1;
    }
  }
}

// ---- spatial sparsifier (bmSteva) ---------------------------------------------
// Backward differences along each image axis d (bmBackGradient_n.m:28-46):
//   (G_d v)[i] = (v[i] - v[i - e_d]) / dX_d, 0 on the first slice along d;
// the transposed form the solver uses (bmBackGradient_nT.m:23-44):
//   (T_d h)[i] = (h[i] (0 on the first slice) - h[i + e_d, circular]) / dX_d.
__device__ __forceinline__ int axis_pos(long long i, const ImGeom& g, int d) {
  return (int)((i / g.st[d]) % g.n[d]);
}

__device__ __forceinline__ float2 bgrad(const float2* __restrict__ v, long long i, const ImGeom& g, int d) {
  if (axis_pos(i, g, d) == 0) return make_float2(0.f, 0.f);
  const float2 t = csub(v[i], v[i - g.st[d]]);
  return make_float2(__fdiv_rn(t.x, g.dX[d]), __fdiv_rn(t.y, g.dX[d]));
}

// z_d = G_d x, u = 0   (bmSteva.m:40-45)
__global__ void st_init_zu_kernel(const float2* __restrict__ x, long long nu, ImGeom g, float2* __restrict__ z,
                                  float2* __restrict__ u) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nu; i += (long long)gridDim.x * blockDim.x)
    for (int d = 0; d < g.dim; ++d) {
      z[d * nu + i] = bgrad(x, i, g, d);
      u[d * nu + i] = make_float2(0.f, 0.f);
    }
}

// res_z = (z - u) - G x   (bmSteva.m:58)
__global__ void st_res_z_kernel(const float2* __restrict__ x, const float2* __restrict__ z,
                                const float2* __restrict__ u, long long nu, ImGeom g, float2* __restrict__ res_z) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nu; i += (long long)gridDim.x * blockDim.x)
    for (int d = 0; d < g.dim; ++d) res_z[d * nu + i] = csub(csub(z[d * nu + i], u[d * nu + i]), bgrad(x, i, g, d));
}

// dA = dA + (rho (1/HX)) sum_d T_d(HZ res_z_d), dA holding (1/HX) M*(HY res_y)
// (bmSteva.m:60-63); partials of |dA|^2
__global__ void st_dA_kernel(float2* __restrict__ dA, const float2* __restrict__ res_z, long long nu, ImGeom g,
                             float HZ, float invHX, const double* __restrict__ sc, double* __restrict__ partial) {
  const float s = __fmul_rn((float)sc[T_RHO], invHX);
  double acc = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nu; i += (long long)gridDim.x * blockDim.x) {
    float2 t = make_float2(0.f, 0.f);
    for (int d = 0; d < g.dim; ++d) {
      const int pos = axis_pos(i, g, d);
      const long long nxt = pos == g.n[d] - 1 ? i - (long long)(g.n[d] - 1) * g.st[d] : i + g.st[d];
      const float2 hi = res_z[d * nu + i], hn = res_z[d * nu + nxt];
      const float2 a = pos == 0 ? make_float2(0.f, 0.f) : make_float2(__fmul_rn(HZ, hi.x), __fmul_rn(HZ, hi.y));
      const float2 b = make_float2(__fmul_rn(HZ, hn.x), __fmul_rn(HZ, hn.y));
      const float2 q = csub(a, b);
      t = cadd(t, make_float2(__fdiv_rn(q.x, g.dX[d]), __fdiv_rn(q.y, g.dX[d])));
    }
    const float2 v = cadd(dA[i], make_float2(__fmul_rn(s, t.x), __fmul_rn(s, t.y)));
    dA[i] = v;
    acc += nrm2(v);
  }
  const double r = block_sum(acc);
  if (threadIdx.x == 0) partial[blockIdx.x] = r;
}

// Fp_d = G_d p with partials of |Fp|^2   (bmSteva.m:83)
__global__ void st_Fp_kernel(const float2* __restrict__ p, long long nu, ImGeom g, float2* __restrict__ Fp,
                             double* __restrict__ partial) {
  double acc = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nu; i += (long long)gridDim.x * blockDim.x)
    for (int d = 0; d < g.dim; ++d) {
      const float2 v = bgrad(p, i, g, d);
      Fp[d * nu + i] = v;
      acc += nrm2(v);
    }
  const double r = block_sum(acc);
  if (threadIdx.x == 0) partial[blockIdx.x] = r;
}

// bGx_plus_u = G x + u; z = prox(., delta/rho); u = bGx_plus_u - z   (bmSteva.m:112-114)
__global__ void st_zu_kernel(const float2* __restrict__ x, long long nu, ImGeom g, float2* __restrict__ z,
                             float2* __restrict__ u, const double* __restrict__ sc) {
  const float s = fabsf(__fdiv_rn((float)sc[T_DELTA], (float)sc[T_RHO]));
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nu; i += (long long)gridDim.x * blockDim.x)
    for (int d = 0; d < g.dim; ++d) {
      const float2 w = cadd(bgrad(x, i, g, d), u[d * nu + i]);
      const float2 zz = make_float2(soft(w.x, s), soft(w.y, s));
      z[d * nu + i] = zz;
      u[d * nu + i] = csub(w, zz);
    }
}

// partials of sum_d |Re G_d x| + |Im G_d x|   (bmSteva.m:121-122)
__global__ void st_regul_kernel(const float2* __restrict__ x, long long nu, ImGeom g, double* __restrict__ partial) {
  double acc = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nu; i += (long long)gridDim.x * blockDim.x)
    for (int d = 0; d < g.dim; ++d) {
      const float2 t = bgrad(x, i, g, d);
      acc += (double)fabsf(t.x) + (double)fabsf(t.y);
    }
  const double r = block_sum(acc);
  if (threadIdx.x == 0) partial[blockIdx.x] = r;
}

// max over v[0..n) per CTA (grid-stride), then over the CTA results
__global__ void vmax_kernel(const float* __restrict__ v, long long n, float* out) {
  __shared__ float sh[kT];
  float m = -FLT_MAX;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    m = fmaxf(m, v[i]);
  sh[threadIdx.x] = m;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) sh[threadIdx.x] = fmaxf(sh[threadIdx.x], sh[threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0) out[blockIdx.x] = sh[0];
}

// ---- host side ---------------------------------------------------------------
static void chain_free(mlg_chain_s* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->graph) cudaGraphExecDestroy(c->graph);
  for (void* q : {(void*)c->p, (void*)c->dA, (void*)c->res_z, (void*)c->Fp, (void*)c->z, (void*)c->u,
                  (void*)c->res_y, (void*)c->Mp, (void*)c->HY, (void*)c->partial, (void*)c->sc, (void*)c->lists,
                  (void*)c->Dx, (void*)c->Sz, (void*)c->dscratch})
    cudaFree(q);
  if (c->ev_in) cudaEventDestroy(c->ev_in);
  if (c->ev_out) cudaEventDestroy(c->ev_out);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

// M p for every frame with partials of |Mp_f|^2_HY stored frame after frame
// from partial[0]; returns their count
static int chain_forward(mlg_chain_s* c, const float2* img, float2* out, const float* sqn_w, int* n_part,
                         cudaStream_t s) {
  int off = 0;
  for (int f = 0; f < c->nFr; ++f) {
    int np = 0;
    MLG_TRY(shanna_run(c->fr[f], img + (size_t)f * c->nu, false, out + (size_t)c->row_off[f] * c->nCh, sqn_w ?
                       sqn_w + c->row_off[f] : nullptr, sqn_w ? c->partial + off : nullptr, sqn_w ? &np : nullptr,
                       s));
    off += np;
  }
  if (n_part) *n_part = off;
  return MLG_OK;
}

// dA_f = (1/HX) M_f*(HY_f res_f) for every frame
static int chain_adjoint(mlg_chain_s* c, const float2* res, float2* out, cudaStream_t s) {
  const float invHX = (float)(1.0 / c->HX);
  for (int f = 0; f < c->nFr; ++f)
    MLG_TRY(nakatsha_run(c->fr[f], res + (size_t)c->row_off[f] * c->nCh, c->HY + c->row_off[f], invHX,
                         out + (size_t)f * c->nu, nullptr, nullptr, s));
  return MLG_OK;
}

// dst_f = T_f src_f for every frame (bmImDeform / bmImDeformT with K = []:
// the FP32 sparse product in stored order); dst_f = src_f where T_f is NULL
static int chain_apply(mlg_chain_s* c, const std::vector<const Csr*>& T, const float2* src, float2* dst,
                       cudaStream_t s) {
  for (int f = 0; f < c->nFr; ++f) {
    const float2* a = src + (size_t)f * c->nu;
    float2* b = dst + (size_t)f * c->nu;
    if (!T[f]) {
      MLG_CUDA(cudaMemcpyAsync(b, a, sizeof(float2) * (size_t)c->nu, cudaMemcpyDeviceToDevice, s));
      continue;
    }
    SpmmArgs g;
    g.m = T[f];
    g.nCh = 1;
    g.in.layout = Layout::kPointC64;
    g.in.a = const_cast<float2*>(a);
    g.in.rows = c->nu;
    g.out.layout = Layout::kPointC64;
    g.out.a = b;
    g.out.rows = c->nu;
    g.seg_scratch = c->dscratch;
    MLG_TRY(spmm(g, s));
  }
  return MLG_OK;
}

// the current frames of F applied to v: Tu_f v_f with deformation fields, v itself otherwise
static const float2* chain_deformed(mlg_chain_s* c, const float2* v, cudaStream_t s, int* st) {
  if (!c->deform || c->spatial) return v;
  *st = chain_apply(c, c->Tu, v, c->Dx, s);
  return c->Dx;
}

// dA = dagM res_y + rho dagF res_z and sqn_dagA_res (:119-123 / :156-159)
static int chain_dagA(mlg_chain_s* c, bool first, cudaStream_t s) {
  const long long ni = c->nu * c->nFr;
  const double eps = 10.0 * (double)FLT_EPSILON;
  MLG_TRY(chain_adjoint(c, c->res_y, c->dA, s));
  const int g = grid1(ni);
  if (c->spatial) {
    st_dA_kernel<<<g, kT, 0, s>>>(c->dA, c->res_z, c->nu, c->geom, (float)c->HX, (float)(1.0 / c->HX), c->sc,
                                  c->partial);
  } else {
    const float2* ts = nullptr;
    if (c->deform) {  // Tut_f (HZ res_z_f)
      tv_scale_kernel<<<grid1(ni), kT, 0, s>>>(c->res_z, ni, (float)c->HX, c->Sz);
      MLG_LAUNCHED();
      MLG_TRY(chain_apply(c, c->Tut, c->Sz, c->Dx, s));
      ts = c->Dx;
    }
    tv_dA_kernel<<<g, kT, 0, s>>>(c->dA, c->res_z, ts, c->nFr, c->nu, (float)c->HX, (float)(1.0 / c->HX), c->sc,
                                  c->partial);
  }
  MLG_LAUNCHED();
  if (first)
    tv_sq_init_kernel<<<1, kT, 0, s>>>(c->partial, g, c->HX, eps, c->sc);
  else
    tv_beta_kernel<<<1, kT, 0, s>>>(c->partial, g, c->HX, eps, c->sc);
  MLG_LAUNCHED();
  return MLG_OK;
}

// Le_Midi and Le_Soir: Mp, Fp, a, x += a p   (:138-147)
static int chain_cg_half(mlg_chain_s* c, float2* x, cudaStream_t s) {
  const long long ni = c->nu * c->nFr;
  int n_mp = 0;
  MLG_TRY(chain_forward(c, c->p, c->Mp, c->HY, &n_mp, s));
  const int g = grid1(ni);
  if (c->spatial) {
    st_Fp_kernel<<<g, kT, 0, s>>>(c->p, c->nu, c->geom, c->Fp, c->partial + n_mp);
  } else {
    int st = MLG_OK;
    const float2* pd = chain_deformed(c, c->p, s, &st);
    MLG_TRY(st);
    tv_Fp_kernel<<<g, kT, 0, s>>>(c->p, pd, c->nFr, c->nu, c->Fp, c->partial + n_mp);
  }
  MLG_LAUNCHED();
  tv_alpha_kernel<<<1, kT, 0, s>>>(c->partial, n_mp, g, c->HX, c->sc);
  MLG_LAUNCHED();
  tv_axpy_kernel<false><<<grid1(ni), kT, 0, s>>>(x, c->p, ni, c->sc);
  MLG_LAUNCHED();
  return MLG_OK;
}

// one full CG step j < nCGD (:128-161)
static int chain_cg_step(mlg_chain_s* c, float2* x, cudaStream_t s) {
  const long long ni = c->nu * c->nFr, nk = c->rows * c->nCh, nd = c->nu * (c->spatial ? c->geom.dim : c->nFr);
  MLG_TRY(chain_cg_half(c, x, s));
  tv_axpy_kernel<true><<<grid1(nk), kT, 0, s>>>(c->res_y, c->Mp, nk, c->sc);
  MLG_LAUNCHED();
  tv_axpy_kernel<true><<<grid1(nd), kT, 0, s>>>(c->res_z, c->Fp, nd, c->sc);
  MLG_LAUNCHED();
  MLG_TRY(chain_dagA(c, false, s));
  tv_update_p_kernel<<<grid1(ni), kT, 0, s>>>(c->p, c->dA, ni, c->sc);
  MLG_LAUNCHED();
  return MLG_OK;
}

// y - M x into res_y with dafi, regul of x (private_dafi_regul, :211-224)
static int chain_monitor(mlg_chain_s* c, const float2* y, const float2* x, double* hist, cudaStream_t s) {
  const long long ni = c->nu * c->nFr, nk = c->rows * c->nCh;
  MLG_TRY(chain_forward(c, x, c->Mp, nullptr, nullptr, s));
  const int gk = grid1(nk), gi = grid1(ni);
  tv_residual_kernel<<<gk, kT, 0, s>>>(y, c->Mp, nk, c->nCh, c->HY, c->res_y, c->partial);
  MLG_LAUNCHED();
  if (c->spatial) {
    st_regul_kernel<<<gi, kT, 0, s>>>(x, c->nu, c->geom, c->partial + gk);
  } else {
    int st = MLG_OK;
    const float2* xd = chain_deformed(c, x, s, &st);
    MLG_TRY(st);
    tv_regul_kernel<<<gi, kT, 0, s>>>(x, xd, c->nFr, c->nu, c->partial + gk);
  }
  MLG_LAUNCHED();
  tv_monitor_kernel<<<1, kT, 0, s>>>(c->partial, gk, gi, c->HX, c->sc, hist, c->spatial ? 2 : 3);
  MLG_LAUNCHED();
  return MLG_OK;
}

// spatial: bmSteva (one frame, dual arrays [imDim][nu]); else the temporal
// chain (dual arrays [nFr][nu]).  ve_max <= 0 means max(ve).
static int chain_run(mlg_chain_s* c, bool spatial, const float2* y, const float* ve, float ve_max,
                     const float* delta, const float* rho, int adapt, int nIter, int nCGD, float2* x, float2* z,
                     float2* u, bool init_zu, double* history, cudaStream_t s) {
  NvtxRange range(spatial ? "ADMM spatial TV (bmSteva)" : "ADMM temporal TV (bmTevaMorphosia_chain)");
  MLG_CHECK(nIter >= 0 && nCGD >= 0, "nIter / nCGD must be >= 0");
  MLG_CHECK(delta && rho, "NULL delta / rho");
  MLG_CHECK(!spatial || (c->nFr == 1 && !adapt), "the spatial solver runs on a chain of one frame, 'normal' mode");
  c->spatial = spatial;
  c->HX = c->fr[0]->HX;  // dK_u may have been set after the chain was made
  for (int d = 0; d < c->geom.dim; ++d) c->geom.dX[d] = c->fr[0]->dX[d];
  const long long ni = c->nu * c->nFr;
  const int hstride = spatial ? 2 : 3;
  if (!(ve_max > 0.f)) {  // bmSteva.m:25-27
    float* part = reinterpret_cast<float*>(c->partial);  // >= 64 doubles of room
    float* dmax = part + 64;
    vmax_kernel<<<32, kT, 0, s>>>(ve, c->rows, part);
    MLG_LAUNCHED();
    vmax_kernel<<<1, kT, 0, s>>>(part, 32, dmax);
    MLG_LAUNCHED();
    MLG_CUDA(cudaMemcpyAsync(&ve_max, dmax, sizeof(float), cudaMemcpyDeviceToHost, s));
    MLG_CUDA(cudaStreamSynchronize(s));
  }
  // delta / rho lists: linspace(first, last, nIter) (private_init_regul_param, :226-238)
  if (nIter > c->lists_cap) {
    cudaFree(c->lists);
    c->lists = nullptr;
    MLG_CUDA(cudaMalloc(&c->lists, sizeof(double) * 2 * (size_t)nIter));
    c->lists_cap = nIter;
  }
  std::vector<double> L(2 * (size_t)c->lists_cap, 0.0);
  for (int i = 0; i < nIter; ++i) {
    const double t = nIter > 1 ? (double)i / (double)(nIter - 1) : 0.0;
    const double d0 = std::fabs((double)delta[0]), d1 = std::fabs((double)delta[1]);
    const double r0 = std::fabs((double)rho[0]), r1 = std::fabs((double)rho[1]);
    L[i] = (float)(i == nIter - 1 && nIter > 1 ? d1 : d0 + (d1 - d0) * t);
    L[c->lists_cap + i] = (float)(i == nIter - 1 && nIter > 1 ? r1 : r0 + (r1 - r0) * t);
  }
  if (nIter > 0)
    MLG_CUDA(cudaMemcpyAsync(c->lists, L.data(), sizeof(double) * L.size(), cudaMemcpyHostToDevice, s));
  tv_hy_kernel<<<grid1(c->rows), kT, 0, s>>>(ve, c->rows, ve_max, c->HY);
  MLG_LAUNCHED();
  if (init_zu) {
    if (spatial) {
      st_init_zu_kernel<<<grid1(ni), kT, 0, s>>>(x, c->nu, c->geom, z, u);
    } else {
      int st = MLG_OK;
      const float2* xd = chain_deformed(c, x, s, &st);
      MLG_TRY(st);
      tv_init_zu_kernel<<<grid1(ni), kT, 0, s>>>(x, xd, c->nFr, c->nu, z, u);
    }
    MLG_LAUNCHED();
  }
  MLG_CUDA(cudaMemsetAsync(c->sc, 0, sizeof(double) * T_COUNT, s));
  DevBuf<double> hist;
  MLG_TRY(hist.alloc(hstride * (size_t)std::max(1, nIter), s));
  // initial monitoring: res_y = y - M x, dafi, regul (:86)
  MLG_TRY(chain_monitor(c, y, x, nullptr, s));

  const int full = std::max(0, nCGD - 1);
  auto ensure_graph = [&]() -> int {
    const void* key[4] = {x, z, u, y};
    std::vector<int> modes{spatial ? 1 : 0};
    for (const mlg_plan_s* p : c->fr) modes.push_back(p->adjoint_mode);
    if (full == 0 || (c->graph && std::equal(key, key + 4, c->graph_key) && modes == c->graph_modes)) return MLG_OK;
    if (c->graph) cudaGraphExecDestroy(c->graph);
    c->graph = nullptr;
    cudaGraph_t g;
    MLG_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    const long long before = g_launches.load();
    const int st = chain_cg_step(c, x, s);
    const cudaError_t ce = cudaStreamEndCapture(s, &g);
    c->graph_kernels = g_launches.load() - before;
    g_launches.fetch_sub(c->graph_kernels);  // captured, not launched
    if (st != MLG_OK) return st;
    if (ce != cudaSuccess) return fail(MLG_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(ce));
    const cudaError_t ie = cudaGraphInstantiate(&c->graph, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) return fail(MLG_ERR_CUDA, "graph instantiate failed: %s", cudaGetErrorString(ie));
    std::copy(key, key + 4, c->graph_key);
    c->graph_modes = modes;
    return MLG_OK;
  };

  for (int it = 0; it < nIter; ++it) {
    tv_params_kernel<<<1, 1, 0, s>>>(c->lists, c->lists_cap, adapt, c->sc);
    MLG_LAUNCHED();
    // L_Aube (:116-123): res_y is the kept monitoring residual
    if (spatial) {
      st_res_z_kernel<<<grid1(ni), kT, 0, s>>>(x, z, u, c->nu, c->geom, c->res_z);
    } else {
      int st = MLG_OK;
      const float2* xd = chain_deformed(c, x, s, &st);
      MLG_TRY(st);
      tv_res_z_kernel<<<grid1(ni), kT, 0, s>>>(x, xd, z, u, c->nFr, c->nu, c->res_z);
    }
    MLG_LAUNCHED();
    MLG_TRY(chain_dagA(c, true, s));
    MLG_CUDA(cudaMemcpyAsync(c->p, c->dA, sizeof(float2) * (size_t)ni, cudaMemcpyDeviceToDevice, s));
    if (full > 0) MLG_TRY(ensure_graph());
    for (int j = 0; j < full; ++j) {
      MLG_CUDA(cudaGraphLaunch(c->graph, s));
      count_launch(c->graph_kernels);
    }
    if (nCGD > 0) MLG_TRY(chain_cg_half(c, x, s));  // the last step stops after x += a p (:148-150)
    if (spatial) {
      st_zu_kernel<<<grid1(ni), kT, 0, s>>>(x, c->nu, c->geom, z, u, c->sc);
    } else {
      int st = MLG_OK;
      const float2* xd = chain_deformed(c, x, s, &st);
      MLG_TRY(st);
      tv_zu_kernel<<<grid1(ni), kT, 0, s>>>(x, xd, c->nFr, c->nu, z, u, c->sc);
    }
    MLG_LAUNCHED();
    MLG_TRY(chain_monitor(c, y, x, hist.p, s));
  }
  if (history && nIter > 0) {
    MLG_CUDA(cudaMemcpyAsync(history, hist.p, sizeof(double) * hstride * nIter, cudaMemcpyDeviceToHost, s));
    MLG_CUDA(cudaStreamSynchronize(s));
  }
  return MLG_OK;
}

}  // namespace mlg

using namespace mlg;

extern "C" {

int mlg_chain_create(int nFr, const mlg_plan_t* plans, mlg_chain_t* out) {
  MLG_CHECK(out, "NULL output");
  *out = nullptr;
  MLG_CHECK(nFr >= 1 && plans, "need nFr >= 1 plans");
  const mlg_plan_s* p0 = plans[0];
  MLG_CHECK(p0, "NULL plan 0");
  for (int f = 0; f < nFr; ++f) {
    const mlg_plan_s* p = plans[f];
    MLG_CHECK(p, "NULL plan %d", f);
    MLG_CHECK(p->Gu && p->Gut, "plan %d needs both Gu and Gut", f);
    MLG_CHECK(p->device == p0->device && p->imDim == p0->imDim && p->nCh == p0->nCh,
              "plan %d differs from plan 0 in device, imDim or nCh", f);
    for (int d = 0; d < 3; ++d)
      MLG_CHECK(p->N[d] == p0->N[d] && p->n[d] == p0->n[d], "plan %d differs from plan 0 in N_u / n_u", f);
  }
  MLG_CUDA(cudaSetDevice(p0->device));
  mlg_chain_s* c = new mlg_chain_s();
  c->device = p0->device;
  c->nFr = nFr;
  c->nCh = p0->nCh;
  c->nu = p0->nu_tot;
  c->HX = p0->HX;
  c->geom.dim = p0->imDim;
  for (int d = 0; d < p0->imDim; ++d) {
    c->geom.n[d] = p0->n[d];
    c->geom.st[d] = d == 0 ? 1 : c->geom.st[d - 1] * p0->n[d - 1];
    c->geom.dX[d] = p0->dX[d];
  }
  c->nd_cap = std::max(nFr, p0->imDim);
  int cap = 0;
  for (int f = 0; f < nFr; ++f) {
    c->fr.push_back(plans[f]);
    c->row_off.push_back(c->rows);
    c->rows += plans[f]->nPt;
    cap += plans[f]->partial_cap;
  }
  const long long ni = c->nu * nFr, nk = c->rows * c->nCh;
  cap = std::max(cap, grid1(nk) + grid1(ni)) + grid1(ni) + 64;
  c->partial_cap = cap;
  const size_t bi = sizeof(float2) * (size_t)ni, bk = sizeof(float2) * (size_t)std::max(1LL, nk);
  const size_t bd = sizeof(float2) * (size_t)(c->nu * c->nd_cap);
  bool ok = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreateWithFlags(&c->ev_in, cudaEventDisableTiming) == cudaSuccess &&
            cudaEventCreateWithFlags(&c->ev_out, cudaEventDisableTiming) == cudaSuccess;
  ok = ok && cudaMalloc(&c->p, bi) == cudaSuccess && cudaMalloc(&c->dA, bi) == cudaSuccess &&
       cudaMalloc(&c->res_z, bd) == cudaSuccess && cudaMalloc(&c->Fp, bd) == cudaSuccess &&
       cudaMalloc(&c->res_y, bk) == cudaSuccess && cudaMalloc(&c->Mp, bk) == cudaSuccess &&
       cudaMalloc(&c->HY, sizeof(float) * (size_t)std::max(1LL, c->rows)) == cudaSuccess &&
       cudaMalloc(&c->partial, sizeof(double) * (size_t)cap) == cudaSuccess &&
       cudaMalloc(&c->sc, sizeof(double) * T_COUNT) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    chain_free(c);
    return fail(MLG_ERR_OOM, "chain: device allocation failed");
  }
  c->Tu.assign(nFr, nullptr);
  c->Tut.assign(nFr, nullptr);
  *out = c;
  return MLG_OK;
}

int mlg_chain_set_deform(mlg_chain_t c, const mlg_matrix_t* Tu, const mlg_matrix_t* Tut) {
  MLG_CHECK(c, "NULL chain");
  MLG_CUDA(cudaSetDevice(c->device));
  std::vector<const Csr*> tu(c->nFr, nullptr), tut(c->nFr, nullptr);
  size_t scratch = 0;
  for (int f = 0; f < c->nFr; ++f)
    for (int k = 0; k < 2; ++k) {
      const mlg_matrix_t m = k == 0 ? (Tu ? Tu[f] : nullptr) : (Tut ? Tut[f] : nullptr);
      if (!m) continue;
      MLG_CHECK(m->device == c->device, "deformation matrix of frame %d is on another device", f);
      MLG_CHECK(m->csr.l_size == c->nu && m->csr.r_size == c->nu,
                "deformation matrix of frame %d must be [%lld x %lld] (image pixels), got [%d x %d]", f, c->nu,
                c->nu, m->csr.l_size, m->csr.r_size);
      (k == 0 ? tu : tut)[f] = &m->csr;
      scratch = std::max(scratch, spmm_scratch_floats(m->csr, 1));
    }
  MLG_CUDA(cudaStreamSynchronize(c->stream));
  const bool any = std::any_of(tu.begin(), tu.end(), [](const Csr* m) { return m != nullptr; }) ||
                   std::any_of(tut.begin(), tut.end(), [](const Csr* m) { return m != nullptr; });
  const size_t bi = sizeof(float2) * (size_t)(c->nu * c->nFr);
  if (any && !c->Dx) {
    if (cudaMalloc(&c->Dx, bi) != cudaSuccess || cudaMalloc(&c->Sz, bi) != cudaSuccess) {
      cudaGetLastError();
      return fail(MLG_ERR_OOM, "chain: deformation buffers");
    }
  }
  cudaFree(c->dscratch);
  c->dscratch = nullptr;
  if (scratch > 0 && cudaMalloc(&c->dscratch, sizeof(float) * scratch) != cudaSuccess) {
    cudaGetLastError();
    return fail(MLG_ERR_OOM, "chain: deformation scratch");
  }
  c->Tu = tu;
  c->Tut = tut;
  c->deform = any;
  if (c->graph) cudaGraphExecDestroy(c->graph);  // captured with the previous fields
  c->graph = nullptr;
  return MLG_OK;
}

int mlg_chain_destroy(mlg_chain_t c) {
  chain_free(c);
  return MLG_OK;
}

int mlg_chain_info(mlg_chain_t c, int* nFr, long long* rows, long long* pixels) {
  MLG_CHECK(c, "NULL chain");
  if (nFr) *nFr = c->nFr;
  if (rows) *rows = c->rows;
  if (pixels) *pixels = c->nu;
  return MLG_OK;
}

}  // extern "C"

namespace mlg {

static int run_dev(mlg_chain_t c, bool spatial, const void* y, const float* ve, float ve_max, const float* delta,
                   const float* rho, int adapt, int nIter, int nCGD, void* x, void* z, void* u, int init_zu,
                   double* history, void* stream) {
  MLG_CHECK(c && y && ve && x && z && u, "NULL argument");
  MLG_CUDA(cudaSetDevice(c->device));
  cudaStream_t user = (cudaStream_t)stream;
  MLG_CUDA(cudaEventRecord(c->ev_in, user));
  MLG_CUDA(cudaStreamWaitEvent(c->stream, c->ev_in, 0));
  // the frames' plans may run on their own streams elsewhere: order them
  for (mlg_plan_s* p : c->fr) MLG_CUDA(cudaStreamWaitEvent(c->stream, p->ev_out, 0));
  const int st = chain_run(c, spatial, (const float2*)y, ve, ve_max, delta, rho, adapt, nIter, nCGD, (float2*)x,
                           (float2*)z, (float2*)u, init_zu != 0, history, c->stream);
  cudaEventRecord(c->ev_out, c->stream);
  cudaStreamWaitEvent(user, c->ev_out, 0);
  return st;
}

static int run_host(mlg_chain_t c, bool spatial, const float* yR, const float* yI, const float* ve, float ve_max,
                    const float* delta, const float* rho, int adapt, int nIter, int nCGD, float* xR, float* xI,
                    double* history) {
  MLG_CHECK(c && yR && yI && ve && xR && xI, "NULL argument");
  MLG_CUDA(cudaSetDevice(c->device));
  cudaStream_t s = c->stream;
  const long long nk = c->rows * c->nCh, ni = c->nu * c->nFr;
  if (!c->z) {
    const size_t bd = sizeof(float2) * (size_t)(c->nu * c->nd_cap);
    if (cudaMalloc(&c->z, bd) != cudaSuccess || cudaMalloc(&c->u, bd) != cudaSuccess) {
      cudaGetLastError();
      return fail(MLG_ERR_OOM, "chain: z/u allocation failed");
    }
  }
  DevBuf<float> dy, dve, dx;
  DevBuf<float2> y2, x2;
  MLG_TRY(dy.alloc(2 * (size_t)nk, s));
  MLG_TRY(dve.alloc((size_t)c->rows, s));
  MLG_TRY(dx.alloc(2 * (size_t)ni, s));
  MLG_TRY(y2.alloc((size_t)nk, s));
  MLG_TRY(x2.alloc((size_t)ni, s));
  MLG_CUDA(cudaMemcpyAsync(dy.p, yR, sizeof(float) * nk, cudaMemcpyHostToDevice, s));
  MLG_CUDA(cudaMemcpyAsync(dy.p + nk, yI, sizeof(float) * nk, cudaMemcpyHostToDevice, s));
  MLG_CUDA(cudaMemcpyAsync(dve.p, ve, sizeof(float) * c->rows, cudaMemcpyHostToDevice, s));
  MLG_CUDA(cudaMemcpyAsync(dx.p, xR, sizeof(float) * ni, cudaMemcpyHostToDevice, s));
  MLG_CUDA(cudaMemcpyAsync(dx.p + ni, xI, sizeof(float) * ni, cudaMemcpyHostToDevice, s));
  // frame f's y{f} is [nPt_f, nCh] column-major at row offset row_off[f]
  for (int f = 0; f < c->nFr; ++f) {
    const long long r0 = c->row_off[f], nr = c->fr[f]->nPt;
    MLG_TRY(mlg::pack_col_to_point(dy.p + r0 * c->nCh, dy.p + nk + r0 * c->nCh, nr, c->nCh, y2.p + r0 * c->nCh, s));
  }
  MLG_TRY(mlg::interleave(dx.p, dx.p + ni, ni, x2.p, s));
  for (mlg_plan_s* p : c->fr) MLG_CUDA(cudaStreamWaitEvent(s, p->ev_out, 0));
  MLG_TRY(chain_run(c, spatial, y2.p, dve.p, ve_max, delta, rho, adapt, nIter, nCGD, x2.p, c->z, c->u, true, history,
                    s));
  MLG_TRY(mlg::deinterleave(x2.p, ni, dx.p, dx.p + ni, s));
  MLG_CUDA(cudaMemcpyAsync(xR, dx.p, sizeof(float) * ni, cudaMemcpyDeviceToHost, s));
  MLG_CUDA(cudaMemcpyAsync(xI, dx.p + ni, sizeof(float) * ni, cudaMemcpyDeviceToHost, s));
  if (cudaStreamSynchronize(s) != cudaSuccess)
    return fail(MLG_ERR_CUDA, "ADMM solver failed: %s", cudaGetErrorString(cudaGetLastError()));
  return mlg::fft_wait_status(c->fr[0]->wait_err, s);  // one flag per device: the frames share it
}

}  // namespace mlg

extern "C" {

int mlg_tevamorphosia_dev(mlg_chain_t c, const void* y, const float* ve, float ve_max, const float* delta,
                          const float* rho, int regul_mode, int nIter, int nCGD, void* x, void* z, void* u,
                          int init_zu, double* history, void* stream) {
  MLG_CHECK(regul_mode == MLG_REGUL_NORMAL || regul_mode == MLG_REGUL_ADAPT, "unknown regul_mode %d", regul_mode);
  return run_dev(c, false, y, ve, ve_max, delta, rho, regul_mode == MLG_REGUL_ADAPT, nIter, nCGD, x, z, u, init_zu,
                 history, stream);
}

int mlg_tevamorphosia(mlg_chain_t c, const float* yR, const float* yI, const float* ve, float ve_max,
                      const float* delta, const float* rho, int regul_mode, int nIter, int nCGD, float* xR, float* xI,
                      double* history) {
  MLG_CHECK(regul_mode == MLG_REGUL_NORMAL || regul_mode == MLG_REGUL_ADAPT, "unknown regul_mode %d", regul_mode);
  return run_host(c, false, yR, yI, ve, ve_max, delta, rho, regul_mode == MLG_REGUL_ADAPT, nIter, nCGD, xR, xI,
                  history);
}

int mlg_steva_dev(mlg_chain_t c, const void* y, const float* ve, float ve_max, const float* delta, const float* rho,
                  int nIter, int nCGD, void* x, void* z, void* u, int init_zu, double* history, void* stream) {
  return run_dev(c, true, y, ve, ve_max, delta, rho, 0, nIter, nCGD, x, z, u, init_zu, history, stream);
}

int mlg_steva(mlg_chain_t c, const float* yR, const float* yI, const float* ve, float ve_max, const float* delta,
              const float* rho, int nIter, int nCGD, float* xR, float* xI, double* history) {
  return run_host(c, true, yR, yI, ve, ve_max, delta, rho, 0, nIter, nCGD, xR, xI, history);
}

}  // extern "C"
