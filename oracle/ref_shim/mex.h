/* Stand-in for MATLAB's mex.h, written for this checker: just enough of the
 * MEX API for the reference's fmex/solve3d.c to compile as a plain C shared
 * library whose GMRES, local matvec and block-Jacobi routines are called
 * directly (never through mexFunction).  Test infrastructure only. */
#ifndef TTG_REF_SHIM_MEX_H
#define TTG_REF_SHIM_MEX_H
#include <math.h>
#include <stddef.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef struct ttg_shim_mxarray mxArray;
typedef enum { mxREAL = 0, mxCOMPLEX = 1 } mxComplexity;
typedef enum { mxDOUBLE_CLASS = 6 } mxClassID;

#define mexPrintf printf

double* mxGetPr(const mxArray* a);
long mxGetNumberOfDimensions(const mxArray* a);
long* mxGetDimensions(const mxArray* a);
size_t mxGetM(const mxArray* a);
size_t mxGetN(const mxArray* a);
mxArray* mxCreateDoubleMatrix(size_t m, size_t n, mxComplexity c);
mxArray* mxCreateNumericArray(long nd, const long* dims, mxClassID id, mxComplexity c);

#endif
