/* Declarations of the MEX/mx API calls topx_mex.c makes, for a compile-only check where no
   MATLAB or Octave mex.h exists.  Not a MEX implementation. */
#ifndef TOPX_TEST_MEX_STUB_H_
#define TOPX_TEST_MEX_STUB_H_
#include <stddef.h>
typedef struct mxArray_tag mxArray;
typedef size_t mwSize;
typedef unsigned char mxLogical;
typedef enum { mxINT32_CLASS, mxDOUBLE_CLASS } mxClassID;
typedef enum { mxREAL } mxComplexity;
void mexErrMsgIdAndTxt(const char* id, const char* fmt, ...);
int mexAtExit(void (*fn)(void));
int mxIsNumeric(const mxArray* a);
size_t mxGetNumberOfElements(const mxArray* a);
double mxGetScalar(const mxArray* a);
int mxGetString(const mxArray* a, char* buf, mwSize n);
int mxIsEmpty(const mxArray* a);
int mxIsChar(const mxArray* a);
char* mxArrayToString(const mxArray* a);
void mxFree(void* p);
int mxIsLogical(const mxArray* a);
int mxIsDouble(const mxArray* a);
mwSize mxGetNumberOfDimensions(const mxArray* a);
const mwSize* mxGetDimensions(const mxArray* a);
mxLogical* mxGetLogicals(const mxArray* a);
void* mxCalloc(size_t n, size_t size);
mxArray* mxCreateStructMatrix(mwSize m, mwSize n, int nfields, const char** names);
mxArray* mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity c);
double* mxGetPr(const mxArray* a);
void mxSetField(mxArray* s, mwSize i, const char* name, mxArray* v);
mxArray* mxCreateDoubleScalar(double v);
mxArray* mxCreateNumericMatrix(mwSize m, mwSize n, mxClassID c, mxComplexity x);
void* mxGetData(const mxArray* a);
#endif
