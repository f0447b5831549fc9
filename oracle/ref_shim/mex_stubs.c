/* Definitions behind the mex.h stand-in.  The checker never calls
 * mexFunction, so none of these is reached; they exist only so that the
 * reference file links as a shared library.  Each aborts if called. */
#include "mex.h"

static void not_available(const char* name) {
  fprintf(stderr, "ref shim: %s is not available outside MATLAB\n", name);
  abort();
}

double* mxGetPr(const mxArray* a) { (void)a; not_available("mxGetPr"); return NULL; }
long mxGetNumberOfDimensions(const mxArray* a) {
  (void)a; not_available("mxGetNumberOfDimensions"); return 0;
}
long* mxGetDimensions(const mxArray* a) { (void)a; not_available("mxGetDimensions"); return NULL; }
size_t mxGetM(const mxArray* a) { (void)a; not_available("mxGetM"); return 0; }
size_t mxGetN(const mxArray* a) { (void)a; not_available("mxGetN"); return 0; }
mxArray* mxCreateDoubleMatrix(size_t m, size_t n, mxComplexity c) {
  (void)m; (void)n; (void)c; not_available("mxCreateDoubleMatrix"); return NULL;
}
mxArray* mxCreateNumericArray(long nd, const long* dims, mxClassID id, mxComplexity c) {
  (void)nd; (void)dims; (void)id; (void)c; not_available("mxCreateNumericArray"); return NULL;
}
