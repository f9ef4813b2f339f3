// mxshim.cpp -- headless implementation of the mx/mex subset in mex.h.
// Arrays own a zero-initialised heap block; class tags follow MATLAB's.
#include "mex.h"

#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

struct mxArray_tag {
  mxClassID cls;
  bool complex;
  std::vector<mwSize> dims;
  std::vector<unsigned char> data;
  size_t elsize;
};

namespace {
struct MexError : std::runtime_error {
  std::string id;
  MexError(const char* i, const std::string& m) : std::runtime_error(m), id(i ? i : "") {}
};

size_t class_size(mxClassID c) {
  switch (c) {
    case mxLOGICAL_CLASS: return sizeof(mxLogical);
    case mxDOUBLE_CLASS: return sizeof(double);
    case mxINT32_CLASS: return sizeof(int32_t);
    default: return 0;
  }
}

mxArray* make(mxClassID cls, mwSize ndim, const mwSize* dims, bool cplx) {
  mxArray* a = new mxArray_tag;
  a->cls = cls;
  a->complex = cplx;
  a->dims.assign(dims, dims + ndim);
  while (a->dims.size() < 2) a->dims.push_back(1);
  while (a->dims.size() > 2 && a->dims.back() == 1) a->dims.pop_back();
  a->elsize = class_size(cls);
  size_t n = 1;
  for (mwSize d : a->dims) n *= d;
  a->data.assign(n * a->elsize, 0);
  return a;
}
}  // namespace

extern "C" {

mxArray* mxCreateNumericArray(mwSize ndim, const mwSize* dims, mxClassID cls, mxComplexity flag) {
  return make(cls, ndim, dims, flag == mxCOMPLEX);
}
mxArray* mxCreateNumericMatrix(mwSize m, mwSize n, mxClassID cls, mxComplexity flag) {
  mwSize d[2] = {m, n};
  return make(cls, 2, d, flag == mxCOMPLEX);
}
mxArray* mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity flag) {
  return mxCreateNumericMatrix(m, n, mxDOUBLE_CLASS, flag);
}
mxArray* mxCreateDoubleScalar(double value) {
  mxArray* a = mxCreateDoubleMatrix(1, 1, mxREAL);
  *mxGetDoubles(a) = value;
  return a;
}
mxArray* mxCreateLogicalMatrix(mwSize m, mwSize n) {
  return mxCreateNumericMatrix(m, n, mxLOGICAL_CLASS, mxREAL);
}
void mxDestroyArray(mxArray* a) { delete a; }

void* mxGetData(const mxArray* a) {
  return a->data.empty() ? nullptr : const_cast<unsigned char*>(a->data.data());
}
double* mxGetDoubles(const mxArray* a) {
  return a->cls == mxDOUBLE_CLASS ? static_cast<double*>(mxGetData(a)) : nullptr;
}
double* mxGetPr(const mxArray* a) { return mxGetDoubles(a); }
mxLogical* mxGetLogicals(const mxArray* a) {
  return a->cls == mxLOGICAL_CLASS ? static_cast<mxLogical*>(mxGetData(a)) : nullptr;
}
int32_t* mxGetInt32s(const mxArray* a) {
  return a->cls == mxINT32_CLASS ? static_cast<int32_t*>(mxGetData(a)) : nullptr;
}
double mxGetScalar(const mxArray* a) {
  if (a->data.empty()) return 0.0;
  switch (a->cls) {
    case mxDOUBLE_CLASS: return *reinterpret_cast<const double*>(a->data.data());
    case mxINT32_CLASS: return *reinterpret_cast<const int32_t*>(a->data.data());
    case mxLOGICAL_CLASS: return *reinterpret_cast<const mxLogical*>(a->data.data()) ? 1.0 : 0.0;
    default: return 0.0;
  }
}
size_t mxGetM(const mxArray* a) { return a->dims[0]; }
size_t mxGetN(const mxArray* a) {
  size_t n = 1;
  for (size_t i = 1; i < a->dims.size(); ++i) n *= a->dims[i];
  return n;
}
size_t mxGetNumberOfElements(const mxArray* a) { return a->elsize ? a->data.size() / a->elsize : 0; }
mwSize mxGetNumberOfDimensions(const mxArray* a) { return a->dims.size(); }
const mwSize* mxGetDimensions(const mxArray* a) { return a->dims.data(); }
mxClassID mxGetClassID(const mxArray* a) { return a->cls; }
bool mxIsDouble(const mxArray* a) { return a->cls == mxDOUBLE_CLASS; }
bool mxIsLogical(const mxArray* a) { return a->cls == mxLOGICAL_CLASS; }
bool mxIsInt32(const mxArray* a) { return a->cls == mxINT32_CLASS; }
bool mxIsComplex(const mxArray* a) { return a->complex; }
bool mxIsEmpty(const mxArray* a) { return mxGetNumberOfElements(a) == 0; }

void mexErrMsgIdAndTxt(const char* id, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  throw MexError(id, buf);
}

// MATLAB calls the registered function when the mex file is cleared; the
// headless runtime calls it at process exit.
int mexAtExit(void (*exit_fcn)(void)) {
  static void (*registered)(void) = nullptr;
  static bool hooked = false;
  registered = exit_fcn;
  if (!hooked) {
    hooked = true;
    std::atexit([] {
      if (registered) registered();
    });
  }
  return 0;
}

int mexPrintf(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  int n = std::vprintf(fmt, ap);
  va_end(ap);
  return n;
}

int mxshim_call_mex(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[], char* err,
                    size_t err_len) {
  try {
    mexFunction(nlhs, plhs, nrhs, prhs);
    return 0;
  } catch (const MexError& e) {
    if (err && err_len) std::snprintf(err, err_len, "%s: %s", e.id.c_str(), e.what());
    return 1;
  } catch (const std::exception& e) {
    if (err && err_len) std::snprintf(err, err_len, "exception: %s", e.what());
    return 1;
  }
}

}  // extern "C"
