/*
 * mex.h -- a small, project-written emulation of the MATLAB MEX C API.
 *
 * MATLAB is not available on the machines this project is built and tested
 * on, so MEX gateways (this project's drop-in gateways and, for parity
 * checks, the Monalisa reference kernels) are compiled against this header
 * and linked with libmexshim.so.  Only the subset of the API that Monalisa's
 * gridding / sparse-matrix MEX files and this project's gateways use is
 * provided.  Storage follows MATLAB's classic "separate complex" model
 * (mxGetPr/mxGetData = real part, mxGetPi/mxGetImagData = imaginary part),
 * column-major, which is what the reference's MEX code assumes.
 *
 * Where real MATLAB exists, the gateways compile unchanged against MATLAB's
 * own mex.h instead.
 */
#ifndef MLG_MEXSHIM_MEX_H
#define MLG_MEXSHIM_MEX_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef size_t mwSize;
typedef size_t mwIndex;
typedef long long mwSignedIndex;

typedef enum {
  mxUNKNOWN_CLASS = 0,
  mxCELL_CLASS,
  mxSTRUCT_CLASS,
  mxLOGICAL_CLASS,
  mxCHAR_CLASS,
  mxVOID_CLASS,
  mxDOUBLE_CLASS,
  mxSINGLE_CLASS,
  mxINT8_CLASS,
  mxUINT8_CLASS,
  mxINT16_CLASS,
  mxUINT16_CLASS,
  mxINT32_CLASS,
  mxUINT32_CLASS,
  mxINT64_CLASS,
  mxUINT64_CLASS
} mxClassID;

typedef enum { mxREAL = 0, mxCOMPLEX = 1 } mxComplexity;

typedef struct mxArray_tag mxArray;

/* data access */
double* mxGetPr(const mxArray* a);
double* mxGetPi(const mxArray* a);
void* mxGetData(const mxArray* a);
void* mxGetImagData(const mxArray* a);
double mxGetScalar(const mxArray* a);

/* shape / type queries */
mwSize mxGetM(const mxArray* a);
mwSize mxGetN(const mxArray* a);
mwSize mxGetNumberOfElements(const mxArray* a);
mwSize mxGetNumberOfDimensions(const mxArray* a);
const mwSize* mxGetDimensions(const mxArray* a);
mxClassID mxGetClassID(const mxArray* a);
int mxIsComplex(const mxArray* a);
int mxIsEmpty(const mxArray* a);
int mxIsSingle(const mxArray* a);
int mxIsDouble(const mxArray* a);
int mxIsInt32(const mxArray* a);
int mxIsInt64(const mxArray* a);

/* creation / destruction (zero-initialised, owned by the caller) */
mxArray* mxCreateNumericArray(mwSize ndim, const mwSize* dims, mxClassID cls,
                              mxComplexity cplx);
mxArray* mxCreateNumericMatrix(mwSize m, mwSize n, mxClassID cls,
                               mxComplexity cplx);
mxArray* mxCreateDoubleScalar(double v);
void mxDestroyArray(mxArray* a);

/* messages; the two error functions abort the running mexFunction and return
 * control to the caller of mxshim_call with a non-zero status */
int mexPrintf(const char* fmt, ...);
void mexErrMsgTxt(const char* msg);
void mexErrMsgIdAndTxt(const char* id, const char* fmt, ...);
void mexWarnMsgTxt(const char* msg);

/* every MEX file exports this */
void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]);

/* ---- shim-only helpers (not part of MATLAB's API) ----------------------- */

/* Wrap caller-owned buffers (no copy, not freed by mxDestroyArray). */
mxArray* mxshim_wrap(mxClassID cls, mwSize ndim, const mwSize* dims,
                     void* real_data, void* imag_data);

typedef void (*mxshim_mexfunc_t)(int, mxArray**, int, const mxArray**);

/* Calls fn(nlhs, plhs, nrhs, prhs), catching mexErrMsgTxt.  Returns 0 on
 * success, 1 if the gateway raised an error (message via mxshim_last_error). */
int mxshim_call(mxshim_mexfunc_t fn, int nlhs, mxArray** plhs, int nrhs,
                const mxArray** prhs);
const char* mxshim_last_error(void);
mwSize mxshim_element_size(const mxArray* a);

#ifdef __cplusplus
}
#endif

#endif /* MLG_MEXSHIM_MEX_H */
