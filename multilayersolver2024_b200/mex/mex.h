/*
 * mex.h -- headless subset of MATLAB's mex / mx C API.
 *
 * Lets a mex gateway (MATLAB's `mexFunction` entry point) be compiled and
 * driven without MATLAB: arrays are plain heap blocks with MATLAB's
 * column-major layout and class tags, and mexErrMsgIdAndTxt raises a C++
 * exception that mxshim_call_mex() turns into a status code.  Only the calls
 * used by this package's gateway and by the two reference mex files on the
 * layer-builder path are provided.  Builds against a real MATLAB use MATLAB's
 * own mex.h instead of this file.
 */
#ifndef MLX_HEADLESS_MEX_H
#define MLX_HEADLESS_MEX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mxArray_tag mxArray;
typedef size_t mwSize;
typedef size_t mwIndex;
#ifdef __cplusplus
typedef bool mxLogical;
#else
typedef unsigned char mxLogical;
#endif

typedef enum {
  mxUNKNOWN_CLASS = 0,
  mxLOGICAL_CLASS = 3,
  mxDOUBLE_CLASS = 6,
  mxINT32_CLASS = 12
} mxClassID;

typedef enum { mxREAL = 0, mxCOMPLEX = 1 } mxComplexity;

mxArray* mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity flag);
mxArray* mxCreateDoubleScalar(double value);
mxArray* mxCreateLogicalMatrix(mwSize m, mwSize n);
mxArray* mxCreateNumericMatrix(mwSize m, mwSize n, mxClassID cls, mxComplexity flag);
mxArray* mxCreateNumericArray(mwSize ndim, const mwSize* dims, mxClassID cls, mxComplexity flag);
void mxDestroyArray(mxArray* a);

double* mxGetDoubles(const mxArray* a);
double* mxGetPr(const mxArray* a);
mxLogical* mxGetLogicals(const mxArray* a);
int32_t* mxGetInt32s(const mxArray* a);
void* mxGetData(const mxArray* a);
double mxGetScalar(const mxArray* a);

size_t mxGetM(const mxArray* a);
size_t mxGetN(const mxArray* a);
size_t mxGetNumberOfElements(const mxArray* a);
mwSize mxGetNumberOfDimensions(const mxArray* a);
const mwSize* mxGetDimensions(const mxArray* a);
mxClassID mxGetClassID(const mxArray* a);

bool mxIsDouble(const mxArray* a);
bool mxIsLogical(const mxArray* a);
bool mxIsInt32(const mxArray* a);
bool mxIsComplex(const mxArray* a);
bool mxIsEmpty(const mxArray* a);

void mexErrMsgIdAndTxt(const char* id, const char* fmt, ...);
int mexAtExit(void (*exit_fcn)(void));
int mexPrintf(const char* fmt, ...);

/* the gateway every mex file defines */
void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]);

/* ---- harness side (not part of MATLAB's API) --------------------------- */
/* Calls this library's mexFunction; returns 0, or 1 with the error id and
 * message written to `err` when the gateway raised mexErrMsgIdAndTxt. */
int mxshim_call_mex(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[],
                    char* err, size_t err_len);

#ifdef __cplusplus
}
#endif
#endif
