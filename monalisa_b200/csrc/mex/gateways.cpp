// Drop-in MEX gateways: same names and argument layouts as the reference's
// MEX files, computing through libmonalisa_gpu.so.  One translation unit,
// compiled once per gateway with -DMLG_GATEWAY_<name>; it builds against
// MATLAB's mex.h or the project's MEX-API shim.
//
// Unlike the reference gateways (which do no checking), these validate
// argument counts and sizes and report errors through mexErrMsgIdAndTxt.
#include <cmath>
#include <cstdint>
#include <vector>

#include "mex.h"
#include "monalisa_gpu.h"

namespace {

void check(int status, const char* what) {
  if (status != MLG_OK) mexErrMsgIdAndTxt("monalisa_b200:gpu", "%s: %s (%s)", what, mlg_status_string(status),
                                          mlg_last_error());
}

void need(bool cond, const char* msg) {
  if (!cond) mexErrMsgIdAndTxt("monalisa_b200:args", "%s", msg);
}

int scalar_i(const mxArray* a) { return (int)mxGetScalar(a); }

// NULL for empty arrays (MATLAB passes empty l_jump for unsqueezed matrices)
template <typename T>
const T* data(const mxArray* a) {
  return (a && !mxIsEmpty(a)) ? (const T*)mxGetData(a) : nullptr;
}

mxArray* single_matrix(size_t m, size_t n, mxComplexity c = mxREAL) {
  mwSize d[2] = {(mwSize)m, (mwSize)n};
  return mxCreateNumericArray(2, d, mxSINGLE_CLASS, c);
}

// ---- leight gridders (bmGridder_n2u_leight{1,2,3}_mex) ----------------------
// Gateway layout: aR, aI, tx[, ty[, tz]], Dn, nCh, nPt, Nx[, Ny[, Nz]], nWin,
// kp1, kp2 (bmGridder_n2u_leight.m:125-131).  The reference's 1-D gateway
// reads a different, gapped layout (prhs[4] = Dn, prhs[9..11] = nWin, kp1,
// kp2; bmGridder_n2u_leight1_mex.cpp:54-67); 12 arguments select it.
void leight(int imDim, int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  int iDn, iCh, iN, iW;
  if (imDim == 1 && nrhs == 12) {
    iDn = 4, iCh = 5, iN = 7, iW = 9;
  } else {
    need(nrhs == 8 + 2 * imDim, "wrong number of arguments");
    iDn = 2 + imDim, iCh = 3 + imDim, iN = 5 + imDim, iW = 5 + 2 * imDim;
  }
  const int nCh = scalar_i(prhs[iCh]), nPt = scalar_i(prhs[iCh + 1]);
  int N[3] = {1, 1, 1};
  for (int d = 0; d < imDim; ++d) N[d] = scalar_i(prhs[iN + d]);
  need(nCh >= 1 && nPt >= 0, "invalid nCh / nPt");
  need(mxIsSingle(prhs[0]) && mxGetNumberOfElements(prhs[0]) >= (size_t)nCh * nPt, "aReal must be single [nCh, nPt]");
  need(mxIsSingle(prhs[1]) && mxGetNumberOfElements(prhs[1]) >= (size_t)nCh * nPt, "aImag must be single [nCh, nPt]");
  for (int d = 0; d < imDim; ++d)
    need(mxIsSingle(prhs[2 + d]) && mxGetNumberOfElements(prhs[2 + d]) >= (size_t)nPt, "t must be single [1, nPt]");
  need(mxIsSingle(prhs[iDn]) && mxGetNumberOfElements(prhs[iDn]) >= (size_t)nPt, "Dn must be single [1, nPt]");
  const size_t nu = (size_t)N[0] * N[1] * N[2];
  plhs[0] = single_matrix(nCh, nu);
  plhs[1] = single_matrix(nCh, nu);
  (void)nlhs;
  const float* t[3] = {data<float>(prhs[2]), imDim > 1 ? data<float>(prhs[3]) : nullptr,
                       imDim > 2 ? data<float>(prhs[4]) : nullptr};
  check(mlg_gridder_n2u_leight(imDim, data<float>(prhs[0]), data<float>(prhs[1]), t[0], t[1], t[2],
                               data<float>(prhs[iDn]), nCh, nPt, N[0], N[1], N[2], scalar_i(prhs[iW]),
                               (float)mxGetScalar(prhs[iW + 1]), (float)mxGetScalar(prhs[iW + 2]),
                               (float*)mxGetData(plhs[0]), (float*)mxGetData(plhs[1])),
        "bmGridder_n2u_leight");
}

// ---- bmGridder_n2u_mex: aR, aI, w, nJump, nCh, nNb, nPt, Nu_tot -------------
void n2u(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  (void)nlhs;
  need(nrhs == 8, "wrong number of arguments");
  const int nCh = scalar_i(prhs[4]), nNb = scalar_i(prhs[5]), nPt = scalar_i(prhs[6]), Nu = scalar_i(prhs[7]);
  need(mxGetNumberOfElements(prhs[2]) >= (size_t)nNb * nPt, "w must hold nNb*nPt weights");
  need(mxIsInt32(prhs[3]) && mxGetNumberOfElements(prhs[3]) >= (size_t)nNb * nPt, "nJump must be int32 [nNb*nPt]");
  plhs[0] = single_matrix(nCh, Nu);
  plhs[1] = single_matrix(nCh, Nu);
  check(mlg_gridder_n2u(data<float>(prhs[0]), data<float>(prhs[1]), data<float>(prhs[2]), data<int>(prhs[3]), nCh,
                        nNb, nPt, Nu, (float*)mxGetData(plhs[0]), (float*)mxGetData(plhs[1])),
        "bmGridder_n2u");
}

// ---- sparse matrix products --------------------------------------------------
struct Jump {
  int r_size, l_size, l_nJump;
  const int *r_jump, *r_nJump, *l_jump;
  const float* m_val;
};

// prhs[0..7] = r_size, r_jump, r_nJump, m_val, l_size, l_jump, l_nJump, l_jump_flag
Jump jump_args(const mxArray* prhs[], int first = 0) {
  Jump j;
  j.r_size = scalar_i(prhs[first + 0]);
  j.r_jump = data<int>(prhs[first + 1]);
  j.r_nJump = data<int>(prhs[first + 2]);
  j.m_val = data<float>(prhs[first + 3]);
  j.l_size = scalar_i(prhs[first + 4]);
  j.l_jump = data<int>(prhs[first + 5]);
  j.l_nJump = scalar_i(prhs[first + 6]);
  need(mxGetNumberOfElements(prhs[first + 2]) >= (size_t)j.l_nJump, "r_nJump shorter than l_nJump");
  return j;
}

void vec_cC(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  (void)nlhs;
  need(nrhs == 11, "wrong number of arguments");
  Jump j = jump_args(prhs);
  const int nVec = scalar_i(prhs[10]);
  need(mxGetNumberOfElements(prhs[8]) >= (size_t)j.r_size * nVec, "v_real must be [r_size, n_vec]");
  need(mxGetNumberOfElements(prhs[9]) >= (size_t)j.r_size * nVec, "v_imag must be [r_size, n_vec]");
  plhs[0] = single_matrix(j.l_size, nVec);
  plhs[1] = single_matrix(j.l_size, nVec);
  check(mlg_sparsemat_vec_cC(j.r_size, j.r_jump, j.r_nJump, j.m_val, j.l_size, j.l_jump, j.l_nJump,
                             data<float>(prhs[8]), data<float>(prhs[9]), nVec, (float*)mxGetData(plhs[0]),
                             (float*)mxGetData(plhs[1])),
        "bmSparseMat_cC_oBlock");
}

void vec_cR(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  (void)nlhs;
  need(nrhs == 10, "wrong number of arguments");
  Jump j = jump_args(prhs);
  const int nVec = scalar_i(prhs[9]);
  need(mxGetNumberOfElements(prhs[8]) >= (size_t)j.r_size * nVec, "v must be [n_vec, r_size]");
  plhs[0] = single_matrix(nVec, j.l_size, mxCOMPLEX);
  const float* vi = (const float*)mxGetImagData(prhs[8]);
  std::vector<float> zeros;
  if (!vi) {  // a real input vector: imaginary part zero
    zeros.assign((size_t)j.r_size * nVec, 0.f);
    vi = zeros.data();
  }
  check(mlg_sparsemat_vec_cR(j.r_size, j.r_jump, j.r_nJump, j.m_val, j.l_size, j.l_jump, j.l_nJump,
                             data<float>(prhs[8]), vi, nVec, (float*)mxGetData(plhs[0]),
                             (float*)mxGetImagData(plhs[0])),
        "bmSparseMat_cR_oBlock");
}

void vec_rC(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  (void)nlhs;
  need(nrhs == 10, "wrong number of arguments");
  Jump j = jump_args(prhs);
  const int nVec = scalar_i(prhs[9]);
  need(mxGetNumberOfElements(prhs[8]) >= (size_t)j.r_size * nVec, "v must be [r_size, n_vec]");
  plhs[0] = single_matrix(j.l_size, nVec);
  check(mlg_sparsemat_vec_rC(j.r_size, j.r_jump, j.r_nJump, j.m_val, j.l_size, j.l_jump, j.l_nJump,
                             data<float>(prhs[8]), nVec, (float*)mxGetData(plhs[0])),
        "bmSparseMat_rC_oBlock");
}

// rR_oBlock: real row layout v [n_vec, r_size] (prhs[8]), n_vec (prhs[9]) ->
// w [n_vec, l_size] (bmSparseMat_rR_oBlock_mex.cpp:40-62)
void vec_rR(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  (void)nlhs;
  need(nrhs == 10, "wrong number of arguments");
  Jump j = jump_args(prhs);
  const int nVec = scalar_i(prhs[9]);
  need(nVec >= 1 && mxGetNumberOfElements(prhs[8]) >= (size_t)j.r_size * nVec, "v must be [n_vec, r_size]");
  plhs[0] = single_matrix(nVec, j.l_size);
  check(mlg_sparsemat_vec_rR(j.r_size, j.r_jump, j.r_nJump, j.m_val, j.l_size, j.l_jump, j.l_nJump,
                             data<float>(prhs[8]), nVec, (float*)mxGetData(plhs[0])),
        "bmSparseMat_rR_oBlock");
}

// block arrays of the *_nBlock_omp gateways: nBlock, block_length,
// l_block_start (int32), m_block_start (int64) in prhs[8..11]
// (bmSparseMat_cR_nBlock_omp_mex.cpp:63-66)
struct Blocks {
  int n;
  const int* length;
  const int* l_start;
  const long long* m_start;
};

Blocks block_args(const mxArray* prhs[]) {
  Blocks b;
  b.n = scalar_i(prhs[8]);
  need(b.n >= 1, "nBlock must be >= 1");
  need(mxGetNumberOfElements(prhs[9]) >= (size_t)b.n && mxGetNumberOfElements(prhs[10]) >= (size_t)b.n &&
           mxGetNumberOfElements(prhs[11]) >= (size_t)b.n,
       "block arrays shorter than nBlock");
  need(mxIsInt32(prhs[9]) && mxIsInt32(prhs[10]) && mxIsInt64(prhs[11]),
       "block_length / l_block_start must be int32 and m_block_start int64");
  b.length = data<int>(prhs[9]);
  b.l_start = data<int>(prhs[10]);
  b.m_start = data<long long>(prhs[11]);
  return b;
}

// cR_nBlock_omp: the gateway reads one complex v [n_vec, r_size] (prhs[12],
// separate imaginary storage) and n_vec (prhs[13])
// (bmSparseMat_cR_nBlock_omp_mex.cpp:69-71).  bmSparseMat_vec.m:167-172 calls
// it with real(v), imag(v), n_vec instead (15 arguments), which the reference
// gateway misreads; both forms are accepted here.
void vec_cR_nBlock(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  (void)nlhs;
  need(nrhs == 14 || nrhs == 15, "wrong number of arguments");
  Jump j = jump_args(prhs);
  Blocks b = block_args(prhs);
  const int nVec = scalar_i(prhs[nrhs - 1]);
  need(nVec >= 1 && mxGetNumberOfElements(prhs[12]) >= (size_t)j.r_size * nVec, "v must be [n_vec, r_size]");
  const float* vr = data<float>(prhs[12]);
  const float* vi = nrhs == 15 ? data<float>(prhs[13]) : (const float*)mxGetImagData(prhs[12]);
  if (nrhs == 15) need(mxGetNumberOfElements(prhs[13]) >= (size_t)j.r_size * nVec, "imag(v) must be [n_vec, r_size]");
  std::vector<float> zeros;
  if (!vi) {
    zeros.assign((size_t)j.r_size * nVec, 0.f);
    vi = zeros.data();
  }
  plhs[0] = single_matrix(nVec, j.l_size, mxCOMPLEX);
  check(mlg_sparsemat_vec(MLG_LAYOUT_CR, j.r_size, j.r_jump, j.r_nJump, j.m_val, j.l_size, j.l_jump, j.l_nJump, b.n,
                          b.length, b.l_start, b.m_start, vr, vi, nVec, (float*)mxGetData(plhs[0]),
                          (float*)mxGetImagData(plhs[0])),
        "bmSparseMat_cR_nBlock_omp");
}

// rR_nBlock_omp: real v [n_vec, r_size] (prhs[12]), n_vec (prhs[13])
// (bmSparseMat_rR_nBlock_omp_mex.cpp:52-82)
void vec_rR_nBlock(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  (void)nlhs;
  need(nrhs == 14, "wrong number of arguments");
  Jump j = jump_args(prhs);
  Blocks b = block_args(prhs);
  const int nVec = scalar_i(prhs[13]);
  need(nVec >= 1 && mxGetNumberOfElements(prhs[12]) >= (size_t)j.r_size * nVec, "v must be [n_vec, r_size]");
  plhs[0] = single_matrix(nVec, j.l_size);
  check(mlg_sparsemat_vec(MLG_LAYOUT_RR, j.r_size, j.r_jump, j.r_nJump, j.m_val, j.l_size, j.l_jump, j.l_nJump, b.n,
                          b.length, b.l_start, b.m_start, data<float>(prhs[12]), nullptr, nVec,
                          (float*)mxGetData(plhs[0]), nullptr),
        "bmSparseMat_rR_nBlock_omp");
}

// cC_oBlock_2_omp: complex column-layout v [r_size, n_vec] with separate
// imaginary storage (prhs[8]), n_vec (prhs[9]) -> complex w [l_size, n_vec]
// (bmSparseMat_cC_oBlock_2_omp_mex.cpp:44-68)
void vec_cC2(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  (void)nlhs;
  need(nrhs == 10, "wrong number of arguments");
  Jump j = jump_args(prhs);
  const int nVec = scalar_i(prhs[9]);
  need(nVec >= 1 && mxGetNumberOfElements(prhs[8]) >= (size_t)j.r_size * nVec, "v must be [r_size, n_vec]");
  const float* vi = (const float*)mxGetImagData(prhs[8]);
  std::vector<float> zeros;
  if (!vi) {
    zeros.assign((size_t)j.r_size * nVec, 0.f);
    vi = zeros.data();
  }
  plhs[0] = single_matrix(j.l_size, nVec, mxCOMPLEX);
  check(mlg_sparsemat_vec_cC(j.r_size, j.r_jump, j.r_nJump, j.m_val, j.l_size, j.l_jump, j.l_nJump,
                             data<float>(prhs[8]), vi, nVec, (float*)mxGetData(plhs[0]),
                             (float*)mxGetImagData(plhs[0])),
        "bmSparseMat_cC_oBlock_2_omp");
}

void nJump2index(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  need(nrhs == 3, "wrong number of arguments");
  const int l_size = scalar_i(prhs[0]);
  const long long n = (long long)mxGetScalar(prhs[2]);
  mwSize d[2] = {1, (mwSize)n};
  plhs[0] = mxCreateNumericArray(2, d, mxINT32_CLASS, mxREAL);
  mwSize d1[2] = {1, 1};
  if (nlhs > 1) {
    plhs[1] = mxCreateNumericArray(2, d1, mxINT64_CLASS, mxREAL);
    *(long long*)mxGetData(plhs[1]) = (long long)d[1];
  }
  check(mlg_sparsemat_r_nJump2index(l_size, data<int>(prhs[1]), n, (int*)mxGetData(plhs[0])),
        "bmSparseMat_r_nJump2index");
}

// ---- fused operators -----------------------------------------------------------
// Shanna{d}: real(x), imag(x), real(KFC), imag(KFC), int32(N_u), G.r_size,
// G.r_jump, G.r_nJump, G.m_val, G.l_size, G.l_jump, G.l_nJump [, int32(n_u)]
// (bmShanna_CUFFT_omp.m:15-35).  Nakatsha{d} takes y and KFC_conj in the first
// four slots (bmNakatsha_CUFFT_omp.m:17-36).  The trailing n_u extends the
// reference (whose CUFFT path requires n_u == N_u): without it n_u = N_u.
void image_size(int imDim, int nrhs, const mxArray* prhs[], size_t nu_elems, int* N, int* n) {
  const int* Nu = data<int>(prhs[4]);
  need(Nu && mxIsInt32(prhs[4]) && mxGetNumberOfElements(prhs[4]) >= (size_t)imDim, "N_u must be int32 [1, imDim]");
  size_t prodN = 1;
  for (int d = 0; d < imDim; ++d) {
    N[d] = Nu[d];
    prodN *= (size_t)Nu[d];
  }
  if (nrhs == 13) {
    const int* nu = data<int>(prhs[12]);
    need(nu && mxIsInt32(prhs[12]), "n_u must be int32 [1, imDim]");
    for (int d = 0; d < imDim; ++d) n[d] = nu[d];
  } else {
    need(nu_elems == prodN, "without n_u, KFC must have prod(N_u) rows");
    for (int d = 0; d < imDim; ++d) n[d] = N[d];
  }
}

void shanna(int imDim, int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  (void)nlhs;
  need(nrhs == 12 || nrhs == 13, "wrong number of arguments");
  const size_t nu = mxGetM(prhs[2]);
  const int nCh = (int)mxGetN(prhs[2]);
  const int x_nCol = (int)mxGetN(prhs[0]);
  need(mxGetM(prhs[0]) == nu, "x and KFC must have the same number of rows");
  int N[3], n[3];
  image_size(imDim, nrhs, prhs, nu, N, n);
  Jump j = jump_args(prhs, 5);
  plhs[0] = single_matrix(j.l_size, nCh);
  plhs[1] = single_matrix(j.l_size, nCh);
  check(mlg_shanna(imDim, N, n, nCh, data<float>(prhs[0]), data<float>(prhs[1]), x_nCol, data<float>(prhs[2]),
                   data<float>(prhs[3]), j.r_size, j.r_jump, j.r_nJump, j.m_val, j.l_size, j.l_jump, j.l_nJump,
                   (float*)mxGetData(plhs[0]), (float*)mxGetData(plhs[1])),
        "bmShanna_CUFFT");
}

void nakatsha(int imDim, int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  (void)nlhs;
  need(nrhs == 12 || nrhs == 13, "wrong number of arguments");
  const size_t nu = mxGetM(prhs[2]);
  const int nCh = (int)mxGetN(prhs[2]);
  need((int)mxGetN(prhs[0]) == nCh, "y must be [nPt, nCh] with nCh = size(KFC_conj, 2)");
  int N[3], n[3];
  image_size(imDim, nrhs, prhs, nu, N, n);
  Jump j = jump_args(prhs, 5);
  need(mxGetM(prhs[0]) == (size_t)j.r_size, "y must have Gut.r_size rows");
  plhs[0] = single_matrix(nu, 1);
  plhs[1] = single_matrix(nu, 1);
  check(mlg_nakatsha(imDim, N, n, nCh, data<float>(prhs[0]), data<float>(prhs[1]), data<float>(prhs[2]),
                     data<float>(prhs[3]), j.r_size, j.r_jump, j.r_nJump, j.m_val, j.l_size, j.l_jump, j.l_nJump,
                     (float*)mxGetData(plhs[0]), (float*)mxGetData(plhs[1])),
        "bmNakatsha_CUFFT");
}

// IDF{d}: real(x), imag(x), int32(N_u), single(dK_u) (bmMathilda.m:85-102)
void idf(int imDim, int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  (void)nlhs;
  need(nrhs == 4, "wrong number of arguments");
  const int* Nu = data<int>(prhs[2]);
  need(Nu && mxIsInt32(prhs[2]), "N_u must be int32");
  need(mxIsSingle(prhs[3]) && mxGetNumberOfElements(prhs[3]) >= (size_t)imDim, "dK_u must be single [1, imDim]");
  size_t prodN = 1;
  for (int d = 0; d < imDim; ++d) prodN *= (size_t)Nu[d];
  const size_t total = mxGetNumberOfElements(prhs[0]);
  need(prodN > 0 && total % prodN == 0, "x must hold a whole number of N_u blocks");
  const mwSize nd = mxGetNumberOfDimensions(prhs[0]);
  plhs[0] = mxCreateNumericArray(nd, mxGetDimensions(prhs[0]), mxSINGLE_CLASS, mxREAL);
  plhs[1] = mxCreateNumericArray(nd, mxGetDimensions(prhs[0]), mxSINGLE_CLASS, mxREAL);
  check(mlg_idf(imDim, Nu, data<float>(prhs[3]), (int)(total / prodN), data<float>(prhs[0]), data<float>(prhs[1]),
                (float*)mxGetData(plhs[0]), (float*)mxGetData(plhs[1])),
        "bmIDF_CUFFT");
}

}  // namespace

extern "C" void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
#if defined(MLG_GATEWAY_bmGridder_n2u_leight1_mex)
  leight(1, nlhs, plhs, nrhs, prhs);
#elif defined(MLG_GATEWAY_bmGridder_n2u_leight2_mex)
  leight(2, nlhs, plhs, nrhs, prhs);
#elif defined(MLG_GATEWAY_bmGridder_n2u_leight3_mex)
  leight(3, nlhs, plhs, nrhs, prhs);
#elif defined(MLG_GATEWAY_bmGridder_n2u_mex)
  n2u(nlhs, plhs, nrhs, prhs);
#elif defined(MLG_GATEWAY_bmSparseMat_cC_oBlock_omp_mex) || defined(MLG_GATEWAY_bmSparseMat_cC_oBlock_mex)
  vec_cC(nlhs, plhs, nrhs, prhs);
#elif defined(MLG_GATEWAY_bmSparseMat_cR_oBlock_mex)
  vec_cR(nlhs, plhs, nrhs, prhs);
#elif defined(MLG_GATEWAY_bmSparseMat_rC_oBlock_mex) || defined(MLG_GATEWAY_bmSparseMat_rC_oBlock_omp_mex)
  vec_rC(nlhs, plhs, nrhs, prhs);
#elif defined(MLG_GATEWAY_bmSparseMat_rR_oBlock_mex)
  vec_rR(nlhs, plhs, nrhs, prhs);
#elif defined(MLG_GATEWAY_bmSparseMat_cR_nBlock_omp_mex)
  vec_cR_nBlock(nlhs, plhs, nrhs, prhs);
#elif defined(MLG_GATEWAY_bmSparseMat_rR_nBlock_omp_mex)
  vec_rR_nBlock(nlhs, plhs, nrhs, prhs);
#elif defined(MLG_GATEWAY_bmSparseMat_cC_oBlock_2_omp_mex)
  vec_cC2(nlhs, plhs, nrhs, prhs);
#elif defined(MLG_GATEWAY_bmSparseMat_r_nJump2index_mex)
  nJump2index(nlhs, plhs, nrhs, prhs);
#elif defined(MLG_GATEWAY_bmShanna1_CUFFT_omp_mex)
  shanna(1, nlhs, plhs, nrhs, prhs);
#elif defined(MLG_GATEWAY_bmShanna2_CUFFT_omp_mex)
  shanna(2, nlhs, plhs, nrhs, prhs);
#elif defined(MLG_GATEWAY_bmShanna3_CUFFT_omp_mex)
  shanna(3, nlhs, plhs, nrhs, prhs);
#elif defined(MLG_GATEWAY_bmNakatsha1_CUFFT_omp_mex)
  nakatsha(1, nlhs, plhs, nrhs, prhs);
#elif defined(MLG_GATEWAY_bmNakatsha2_CUFFT_omp_mex)
  nakatsha(2, nlhs, plhs, nrhs, prhs);
#elif defined(MLG_GATEWAY_bmNakatsha3_CUFFT_omp_mex)
  nakatsha(3, nlhs, plhs, nrhs, prhs);
#elif defined(MLG_GATEWAY_bmIDF1_CUFFT_mex)
  idf(1, nlhs, plhs, nrhs, prhs);
#elif defined(MLG_GATEWAY_bmIDF2_CUFFT_mex)
  idf(2, nlhs, plhs, nrhs, prhs);
#elif defined(MLG_GATEWAY_bmIDF3_CUFFT_mex)
  idf(3, nlhs, plhs, nrhs, prhs);
#else
#error "define MLG_GATEWAY_<name>"
#endif
}
