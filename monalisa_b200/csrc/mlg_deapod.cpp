// Deapodisation K of src/fourier123/prep_function/bmK.m:6-156.
//
// The reference evaluates the gridding kernel on a 2x oversampled grid of
// step 1/2, zeroes it outside the box |x_d| <= fix(nWin/2) (bmK.m:86-104),
// takes the centred DFT on the oversampled grid, crops the central N_u
// block, and forms min(1/(|Re K| / max|Re K|), K_max) (bmK.m:148-151).
//
// Only (4h+1)^d samples (h = fix(nWin/2)) of the kernel are non-zero, so the
// cropped DFT is evaluated directly: with m_d = j_d - N_d/2 and the sample
// coordinates x_d in {-h, -h+1/2, ..., h},
//   K[j] = sum_x w(|x|) prod_d exp(-2 pi i m_d x_d / N_d),
// as three separable passes (one per dimension) in FP64.  The constant DFT
// scaling of bmDFT{1,2,3} cancels in the normalisation by max |Re K|.
#include <cmath>
#include <vector>

#include "mlg_internal.cuh"

namespace {

double bessel_i0(double x) {
  // power series sum_k ((x/2)^(2k)) / (k!)^2, all terms positive; for the
  // kernel arguments used here (|x| <= alpha ~ 10-20) it converges to full
  // double precision in < 60 terms.
  const double q = 0.25 * x * x;
  double term = 1.0, sum = 1.0;
  for (int k = 1; k < 500; ++k) {
    term *= q / ((double)k * (double)k);
    sum += term;
    if (term < sum * 1e-17) break;
  }
  return sum;
}

double kernel_weight(double d, int type, const double* kp) {
  if (type == MLG_KERNEL_GAUSS) {
    const double s = kp[0];
    return std::exp(-0.5 * (d / s) * (d / s)) / (std::sqrt(2 * M_PI) * s);  // normpdf(d, 0, s)
  }
  const double tau = kp[0], alpha = kp[1];
  double w = 1 - (d / tau) * (d / tau);
  if (w < 0) w = 0;
  return bessel_i0(alpha * std::sqrt(w)) / bessel_i0(alpha);
}

double single(double v) { return (double)(float)v; }

}  // namespace

namespace mlg {

int deapod_tables(int imDim, const int* N_u, int kernelType, int nWin, const double* kernelParam, DeapodTables& T) {
  MLG_CHECK(imDim >= 1 && imDim <= 3 && N_u && kernelParam, "invalid argument");
  MLG_CHECK(kernelType == MLG_KERNEL_GAUSS || kernelType == MLG_KERNEL_KAISER, "unknown kernel type");
  MLG_CHECK(nWin >= 1, "nWin must be >= 1");
  T.imDim = imDim;
  for (int d = 0; d < 3; ++d) T.N[d] = 1;
  for (int d = 0; d < imDim; ++d) {
    MLG_CHECK(N_u[d] >= 2 && (N_u[d] % 2) == 0, "N_u must have all components even");
    T.N[d] = N_u[d];
  }
  // kernel parameters pass through single precision, as bmK.m:19 does
  double kp[3] = {single(kernelParam[0]), single(kernelParam[1]),
                  kernelType == MLG_KERNEL_KAISER ? single(kernelParam[2]) : 0.0};
  T.K_max = kernelType == MLG_KERNEL_GAUSS ? kp[1] : kp[2];
  const int h = nWin / 2;  // fix(nWin/2)
  // support coordinates per dimension: x = -h, -h+1/2, ..., h (4h+1 values)
  const int S = 4 * h + 1;
  T.S = S;
  std::vector<double> xs(S);
  for (int a = 0; a < S; ++a) xs[a] = -h + 0.5 * a;
  // which support coordinates survive the box mask; in 1D the reference's
  // expression (x < h) | (x > h) (bmK.m:88) keeps only x == h
  std::vector<int> keep(S, 1);
  if (imDim == 1)
    for (int a = 0; a < S; ++a) keep[a] = (xs[a] == (double)h);
  const int Sy = imDim > 1 ? S : 1, Sz = imDim > 2 ? S : 1;
  T.Sy = Sy;
  T.Sz = Sz;
  // weights w[az][ay][ax]
  T.w.assign((size_t)S * Sy * Sz, 0.0);
  for (int az = 0; az < Sz; ++az)
    for (int ay = 0; ay < Sy; ++ay)
      for (int ax = 0; ax < S; ++ax) {
        const double x = xs[ax], y = imDim > 1 ? xs[ay] : 0.0, z = imDim > 2 ? xs[az] : 0.0;
        const bool in = keep[ax] && (imDim < 2 || keep[ay]) && (imDim < 3 || keep[az]);
        T.w[((size_t)az * Sy + ay) * S + ax] = in ? kernel_weight(std::sqrt(x * x + y * y + z * z), kernelType, kp) : 0.0;
      }
  // cos tables: c_d[j][a] = cos(2 pi (j - N/2) x_a / N); the support and the
  // weights are symmetric in each x_d, so the DFT is real
  auto table = [&](int n) {
    std::vector<double> t((size_t)n * S);
    for (int j = 0; j < n; ++j)
      for (int a = 0; a < S; ++a) t[(size_t)j * S + a] = std::cos(2 * M_PI * (double)(j - n / 2) * xs[a] / n);
    return t;
  };
  T.cx = table(T.N[0]);
  T.cy = imDim > 1 ? table(T.N[1]) : std::vector<double>(S, 1.0);
  T.cz = imDim > 2 ? table(T.N[2]) : std::vector<double>(S, 1.0);
  return MLG_OK;
}

}  // namespace mlg

extern "C" int mlg_deapodization(int imDim, const int* N_u, const double* dK_u, int kernelType, int nWin,
                                 const double* kernelParam, float* K) {
  (void)dK_u;  // only scales the DFT, which cancels in the normalisation
  MLG_CHECK(K, "invalid argument");
  mlg::DeapodTables T;
  MLG_TRY(mlg::deapod_tables(imDim, N_u, kernelType, nWin, kernelParam, T));
  const int* N = T.N;
  const int S = T.S, Sy = T.Sy, Sz = T.Sz;
  const double K_max = T.K_max;
  const std::vector<double>&w = T.w, &cx = T.cx, &cy = T.cy, &cz = T.cz;
  // pass x: A1[az][ay][jx]
  std::vector<double> A1((size_t)Sz * Sy * N[0], 0.0);
  for (int az = 0; az < Sz; ++az)
    for (int ay = 0; ay < Sy; ++ay)
      for (int jx = 0; jx < N[0]; ++jx) {
        double acc = 0.0;
        for (int ax = 0; ax < S; ++ax) acc += w[((size_t)az * Sy + ay) * S + ax] * cx[(size_t)jx * S + ax];
        A1[((size_t)az * Sy + ay) * N[0] + jx] = acc;
      }
  // pass y: A2[az][jy][jx]
  std::vector<double> A2((size_t)Sz * N[1] * N[0], 0.0);
  for (int az = 0; az < Sz; ++az)
    for (int jy = 0; jy < N[1]; ++jy)
      for (int jx = 0; jx < N[0]; ++jx) {
        double acc = 0.0;
        for (int ay = 0; ay < Sy; ++ay)
          acc += A1[((size_t)az * Sy + ay) * N[0] + jx] * (imDim > 1 ? cy[(size_t)jy * S + ay] : 1.0);
        A2[((size_t)az * N[1] + jy) * N[0] + jx] = acc;
      }
  // pass z, |Re|, and the running maximum
  const size_t total = (size_t)N[0] * N[1] * N[2];
  std::vector<double> Kd(total);
  double kmax = 0.0;
#pragma omp parallel for reduction(max : kmax) schedule(static)
  for (long long jz = 0; jz < N[2]; ++jz)
    for (int jy = 0; jy < N[1]; ++jy)
      for (int jx = 0; jx < N[0]; ++jx) {
        double acc = 0.0;
        for (int az = 0; az < Sz; ++az)
          acc += A2[((size_t)az * N[1] + jy) * N[0] + jx] * (imDim > 2 ? cz[(size_t)jz * S + az] : 1.0);
        const double v = std::fabs(acc);
        Kd[((size_t)jz * N[1] + jy) * N[0] + jx] = v;
        if (v > kmax) kmax = v;
      }
  MLG_CHECK(kmax > 0, "kernel transform vanishes (check kernel parameters)");
  for (size_t i = 0; i < total; ++i) {
    const double k = 1.0 / (Kd[i] / kmax);
    K[i] = (float)(k < K_max ? k : K_max);
  }
  return MLG_OK;
}
