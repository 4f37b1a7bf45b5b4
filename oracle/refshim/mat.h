/* In-memory stand-in for the MATLAB MAT-file C API, declaring only the
 * symbols that the reference solver (CODE/C++/VS2010/simLB/simLB/cpuLBM.cpp)
 * calls.  Test infrastructure: it lets the unmodified reference compile and
 * run as the parity oracle.  Variables are read from and written to the
 * simple container format implemented in matshim.cpp ("LBMV1"), not from
 * real .mat files. */
#ifndef REFSHIM_MAT_H_
#define REFSHIM_MAT_H_
#include <stddef.h>

typedef size_t mwSize;
typedef struct shim_mxArray mxArray;
typedef struct shim_MATFile MATFile;
typedef enum { mxDOUBLE_CLASS = 6 } mxClassID;
typedef enum { mxREAL = 0, mxCOMPLEX = 1 } mxComplexity;

MATFile *matOpen(const char *filename, const char *mode);
int matClose(MATFile *pmat);
char **matGetDir(MATFile *pmat, int *num);
mxArray *matGetNextVariable(MATFile *pmat, const char **name);
int matPutVariable(MATFile *pmat, const char *name, const mxArray *pa);
mwSize mxGetNumberOfDimensions(const mxArray *pa);
const mwSize *mxGetDimensions(const mxArray *pa);
double *mxGetPr(const mxArray *pa);
mxArray *mxCreateNumericArray(mwSize ndim, const mwSize *dims, mxClassID classid, mxComplexity flag);
void mxDestroyArray(mxArray *pa);
void mxFree(void *ptr);

#endif
