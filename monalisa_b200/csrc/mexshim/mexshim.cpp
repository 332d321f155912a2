// Project-written emulation of the MATLAB MEX C API subset declared in mex.h.
// Arrays are column-major with separate real/imaginary storage, matching the
// layout the Monalisa MEX kernels read through mxGetPr/mxGetPi.
#include "mex.h"

#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>

struct mxArray_tag {
  mxClassID cls;
  mwSize ndim;
  mwSize dims[8];
  void* re;
  void* im;
  bool owns;
};

namespace {

thread_local std::string g_last_error;

struct MexError : std::runtime_error {
  explicit MexError(const std::string& m) : std::runtime_error(m) {}
};

mwSize class_size(mxClassID c) {
  switch (c) {
    case mxDOUBLE_CLASS:
    case mxINT64_CLASS:
    case mxUINT64_CLASS:
      return 8;
    case mxSINGLE_CLASS:
    case mxINT32_CLASS:
    case mxUINT32_CLASS:
      return 4;
    case mxINT16_CLASS:
    case mxUINT16_CLASS:
    case mxCHAR_CLASS:
      return 2;
    case mxINT8_CLASS:
    case mxUINT8_CLASS:
    case mxLOGICAL_CLASS:
      return 1;
    default:
      return 0;
  }
}

mwSize numel(const mxArray* a) {
  mwSize n = 1;
  for (mwSize i = 0; i < a->ndim; ++i) n *= a->dims[i];
  return n;
}

}  // namespace

extern "C" {

double* mxGetPr(const mxArray* a) { return a ? (double*)a->re : nullptr; }
double* mxGetPi(const mxArray* a) { return a ? (double*)a->im : nullptr; }
void* mxGetData(const mxArray* a) { return a ? a->re : nullptr; }
void* mxGetImagData(const mxArray* a) { return a ? a->im : nullptr; }

double mxGetScalar(const mxArray* a) {
  if (!a || !a->re || numel(a) == 0) return 0.0;
  switch (a->cls) {
    case mxDOUBLE_CLASS: return *(const double*)a->re;
    case mxSINGLE_CLASS: return (double)*(const float*)a->re;
    case mxINT32_CLASS: return (double)*(const int32_t*)a->re;
    case mxUINT32_CLASS: return (double)*(const uint32_t*)a->re;
    case mxINT64_CLASS: return (double)*(const int64_t*)a->re;
    case mxUINT64_CLASS: return (double)*(const uint64_t*)a->re;
    case mxINT16_CLASS: return (double)*(const int16_t*)a->re;
    case mxUINT16_CLASS: return (double)*(const uint16_t*)a->re;
    case mxINT8_CLASS: return (double)*(const int8_t*)a->re;
    case mxUINT8_CLASS:
    case mxLOGICAL_CLASS: return (double)*(const uint8_t*)a->re;
    default: return 0.0;
  }
}

mwSize mxGetM(const mxArray* a) { return (a && a->ndim > 0) ? a->dims[0] : 0; }
mwSize mxGetN(const mxArray* a) {
  if (!a || a->ndim < 2) return a && a->ndim == 1 ? 1 : 0;
  mwSize n = 1;
  for (mwSize i = 1; i < a->ndim; ++i) n *= a->dims[i];
  return n;
}
mwSize mxGetNumberOfElements(const mxArray* a) { return a ? numel(a) : 0; }
mwSize mxGetNumberOfDimensions(const mxArray* a) { return a ? a->ndim : 0; }
const mwSize* mxGetDimensions(const mxArray* a) { return a ? a->dims : nullptr; }
mxClassID mxGetClassID(const mxArray* a) { return a ? a->cls : mxUNKNOWN_CLASS; }
int mxIsComplex(const mxArray* a) { return a && a->im != nullptr; }
int mxIsEmpty(const mxArray* a) { return !a || numel(a) == 0; }
int mxIsSingle(const mxArray* a) { return a && a->cls == mxSINGLE_CLASS; }
int mxIsDouble(const mxArray* a) { return a && a->cls == mxDOUBLE_CLASS; }
int mxIsInt32(const mxArray* a) { return a && a->cls == mxINT32_CLASS; }
int mxIsInt64(const mxArray* a) { return a && a->cls == mxINT64_CLASS; }

mxArray* mxCreateNumericArray(mwSize ndim, const mwSize* dims, mxClassID cls,
                              mxComplexity cplx) {
  if (ndim > 8) return nullptr;
  mxArray* a = new mxArray_tag();
  a->cls = cls;
  a->ndim = ndim < 2 ? 2 : ndim;
  a->dims[0] = ndim > 0 ? dims[0] : 0;
  a->dims[1] = ndim > 1 ? dims[1] : 1;
  for (mwSize i = 2; i < ndim; ++i) a->dims[i] = dims[i];
  mwSize bytes = numel(a) * class_size(cls);
  a->re = std::calloc(bytes ? bytes : 1, 1);
  a->im = (cplx == mxCOMPLEX) ? std::calloc(bytes ? bytes : 1, 1) : nullptr;
  a->owns = true;
  return a;
}

mxArray* mxCreateNumericMatrix(mwSize m, mwSize n, mxClassID cls,
                               mxComplexity cplx) {
  mwSize d[2] = {m, n};
  return mxCreateNumericArray(2, d, cls, cplx);
}

mxArray* mxCreateDoubleScalar(double v) {
  mxArray* a = mxCreateNumericMatrix(1, 1, mxDOUBLE_CLASS, mxREAL);
  *(double*)a->re = v;
  return a;
}

void mxDestroyArray(mxArray* a) {
  if (!a) return;
  if (a->owns) {
    std::free(a->re);
    std::free(a->im);
  }
  delete a;
}

int mexPrintf(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  int r = std::vprintf(fmt, ap);
  va_end(ap);
  return r;
}

void mexErrMsgTxt(const char* msg) { throw MexError(msg ? msg : "error"); }

void mexErrMsgIdAndTxt(const char* id, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  std::string m = std::string(id ? id : "") + ": " + buf;
  throw MexError(m);
}

void mexWarnMsgTxt(const char* msg) { std::fprintf(stderr, "Warning: %s\n", msg); }

mxArray* mxshim_wrap(mxClassID cls, mwSize ndim, const mwSize* dims,
                     void* real_data, void* imag_data) {
  if (ndim > 8) return nullptr;
  mxArray* a = new mxArray_tag();
  a->cls = cls;
  a->ndim = ndim < 2 ? 2 : ndim;
  a->dims[0] = ndim > 0 ? dims[0] : 0;
  a->dims[1] = ndim > 1 ? dims[1] : 1;
  for (mwSize i = 2; i < ndim; ++i) a->dims[i] = dims[i];
  // MATLAB hands a NULL data pointer to MEX code for empty arrays.
  a->re = numel(a) ? real_data : nullptr;
  a->im = numel(a) ? imag_data : nullptr;
  a->owns = false;
  return a;
}

int mxshim_call(mxshim_mexfunc_t fn, int nlhs, mxArray** plhs, int nrhs,
                const mxArray** prhs) {
  g_last_error.clear();
  try {
    fn(nlhs, plhs, nrhs, prhs);
  } catch (const std::exception& e) {
    g_last_error = e.what();
    return 1;
  } catch (...) {
    g_last_error = "unknown error";
    return 1;
  }
  return 0;
}

const char* mxshim_last_error(void) { return g_last_error.c_str(); }

mwSize mxshim_element_size(const mxArray* a) { return a ? class_size(a->cls) : 0; }

}  // extern "C"
