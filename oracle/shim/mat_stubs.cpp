// Abort-only definitions for the MATLAB API declared in mat.h.
//
// TEST INFRASTRUCTURE (oracle build only). The oracle harness calls the reference's fusion and
// regularisation routines directly and never its .mat reader/writer, so none of these runs; if
// one ever did, the oracle must stop loudly instead of returning made-up data.
#include <cstdio>
#include <cstdlib>

#include "mat.h"

[[noreturn]] static void pct_shim_unavailable(const char *fn) {
  std::fprintf(stderr, "oracle: MATLAB API %s called, but libmat is not available\n", fn);
  std::abort();
}

extern "C" {
MATFile *matOpen(const char *, const char *) { pct_shim_unavailable("matOpen"); }
int matClose(MATFile *) { pct_shim_unavailable("matClose"); }
char **matGetDir(MATFile *, int *) { pct_shim_unavailable("matGetDir"); }
mxArray *matGetNextVariable(MATFile *, const char **) { pct_shim_unavailable("matGetNextVariable"); }
mxArray *matGetNextVariableInfo(MATFile *, const char **) {
  pct_shim_unavailable("matGetNextVariableInfo");
}
int matPutVariable(MATFile *, const char *, const mxArray *) { pct_shim_unavailable("matPutVariable"); }
void *mxGetData(const mxArray *) { pct_shim_unavailable("mxGetData"); }
double *mxGetPr(const mxArray *) { pct_shim_unavailable("mxGetPr"); }
size_t mxGetNumberOfElements(const mxArray *) { pct_shim_unavailable("mxGetNumberOfElements"); }
mwSize mxGetNumberOfDimensions(const mxArray *) { pct_shim_unavailable("mxGetNumberOfDimensions"); }
const mwSize *mxGetDimensions(const mxArray *) { pct_shim_unavailable("mxGetDimensions"); }
mxArray *mxGetField(const mxArray *, mwIndex, const char *) { pct_shim_unavailable("mxGetField"); }
mxClassID mxGetClassID(const mxArray *) { pct_shim_unavailable("mxGetClassID"); }
bool mxIsComplex(const mxArray *) { pct_shim_unavailable("mxIsComplex"); }
bool mxIsStruct(const mxArray *) { pct_shim_unavailable("mxIsStruct"); }
int mxGetNumberOfFields(const mxArray *) { pct_shim_unavailable("mxGetNumberOfFields"); }
const char *mxGetFieldNameByNumber(const mxArray *, int) {
  pct_shim_unavailable("mxGetFieldNameByNumber");
}
mxArray *mxCreateNumericArray(mwSize, const mwSize *, mxClassID, mxComplexity) {
  pct_shim_unavailable("mxCreateNumericArray");
}
void mxDestroyArray(mxArray *) { pct_shim_unavailable("mxDestroyArray"); }
void mxFree(void *) { pct_shim_unavailable("mxFree"); }
}
