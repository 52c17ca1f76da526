/*
 * Declaration-only stand-in for MATLAB's <mat.h>.
 *
 * TEST INFRASTRUCTURE (oracle build only). MATLAB's libmat/libmx are not installed, but the
 * reference CPU source (src/CPU/NewPatchedBrainPureC.cpp) only compiles with -DMATLAB (its
 * non-MATLAB branch calls MatrixIO::store/read_ and FindDimension(char*), which do not exist:
 * NewPatchedBrainPureC.cpp:976-989,1519,1747). This header declares the handful of types and
 * functions that file names so it compiles; mat_stubs.cpp defines each one to abort(). The
 * oracle harness never reaches the .mat reader or writer: it sets the reference's globals and
 * calls the fusion routines directly.
 */
#ifndef PCT_ORACLE_MAT_SHIM_H
#define PCT_ORACLE_MAT_SHIM_H

#include <stddef.h>

typedef size_t mwSize;
typedef size_t mwIndex;

typedef struct pct_shim_mxArray mxArray;
typedef struct pct_shim_MATFile MATFile;

typedef enum {
  mxUNKNOWN_CLASS = 0,
  mxCELL_CLASS,
  mxSTRUCT_CLASS,
  mxLOGICAL_CLASS,
  mxCHAR_CLASS,
  mxVOID_CLASS,
  mxDOUBLE_CLASS,
  mxSINGLE_CLASS
} mxClassID;

typedef enum { mxREAL = 0, mxCOMPLEX = 1 } mxComplexity;

#ifdef __cplusplus
extern "C" {
#endif

MATFile *matOpen(const char *filename, const char *mode);
int matClose(MATFile *mfp);
char **matGetDir(MATFile *mfp, int *num);
mxArray *matGetNextVariable(MATFile *mfp, const char **name);
mxArray *matGetNextVariableInfo(MATFile *mfp, const char **name);
int matPutVariable(MATFile *mfp, const char *name, const mxArray *pm);

void *mxGetData(const mxArray *pa);
double *mxGetPr(const mxArray *pa);
size_t mxGetNumberOfElements(const mxArray *pa);
mwSize mxGetNumberOfDimensions(const mxArray *pa);
const mwSize *mxGetDimensions(const mxArray *pa);
mxArray *mxGetField(const mxArray *pa, mwIndex i, const char *fieldname);
mxClassID mxGetClassID(const mxArray *pa);
bool mxIsComplex(const mxArray *pa);
bool mxIsStruct(const mxArray *pa);
int mxGetNumberOfFields(const mxArray *pa);
const char *mxGetFieldNameByNumber(const mxArray *pa, int n);
mxArray *mxCreateNumericArray(mwSize ndim, const mwSize *dims, mxClassID classid,
                              mxComplexity flag);
void mxDestroyArray(mxArray *pa);
void mxFree(void *ptr);

#ifdef __cplusplus
}
#endif

#endif /* PCT_ORACLE_MAT_SHIM_H */
