/*
 * topx_mex.c -- MEX gateway from MATLAB / GNU Octave into libtopx.so.
 *
 * Built where mex.h exists:
 *   mex -I../../include topx_mex.c -L.. -ltopx            (MATLAB)
 *   mkoctfile --mex -I../../include topx_mex.c -L.. -ltopx (Octave)
 *
 *   [hist, xPhys, grid] = topx_mex(inputModel, consType, V0, nLoop, rMin, rHat, precision, ...
 *                                  typeVcycle, specifyPassiveRegions)
 *   topx_mex('write_design', vol, prefix)
 *
 * inputModel: logical (nely, nelx, nelz) array (built-in cuboid BCs) or a .TopVoxel path;
 * consType 'GLOBAL' | 'LOCAL'; rHat may be [] for GLOBAL; precision 'fp64' (default) | 'mixed';
 * typeVcycle 'Adapted' (default) | 'Standard'; specifyPassiveRegions a 3-vector of layer counts
 * (boundary, near loads, near fixations), default [0 0 0].  Arguments 6 to 9 are optional.
 * hist: struct with fields cSolid, c, vol, sharp, cons, change, its, tAssemble, tCG, tOpti, tFilter, tTotal.
 * xPhys: densityLayout_ (numElements x 1, eleMapBack order).
 * grid: struct with resX, resY, resZ, eleMapBack (for the padded volume of IO_ExportDesignInVolume_nii).
 *
 * The device context lives in a static handle and is released by mexAtExit.
 * Every library status is turned into mexErrMsgIdAndTxt; no C++ exception crosses this file.
 */
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include "mex.h"
#include "topx.h"

static topx_ctx* g_ctx = NULL;

static void topx_mex_cleanup(void) {
  if (g_ctx) {
    topx_destroy(g_ctx);
    g_ctx = NULL;
  }
}

static void check(topx_status s, const char* what) {
  if (s == TOPX_OK || s == TOPX_STOP) return;
  mexErrMsgIdAndTxt("topx:error", "%s failed (%d): %s", what, s, topx_last_error(g_ctx));
}

static double scalar_arg(const mxArray* a, const char* name) {
  if (!mxIsNumeric(a) || mxGetNumberOfElements(a) != 1) mexErrMsgIdAndTxt("topx:arg", "%s must be a scalar", name);
  return mxGetScalar(a);
}

/* topx_mex('write_design', V, outPath): DesignVolume.nii and DesignVolume.stl of the padded density
   volume V (ny x nx x nz double), TOP3D_XL.m:206-222 and 564-577 */
static void write_design(const mxArray* V, const mxArray* dir) {
  char path[4096], base[4000];
  const mwSize* d;
  if (!mxIsDouble(V) || mxGetNumberOfDimensions(V) != 3) mexErrMsgIdAndTxt("topx:arg", "V must be a 3-D double array");
  if (mxGetString(dir, base, sizeof(base))) mexErrMsgIdAndTxt("topx:arg", "outPath must be a string");
  d = mxGetDimensions(V);
  snprintf(path, sizeof(path), "%sDesignVolume.nii", base);
  if (topx_write_design_nii(mxGetPr(V), (int)d[0], (int)d[1], (int)d[2], path) != TOPX_OK)
    mexErrMsgIdAndTxt("topx:error", "cannot write %s", path);
  snprintf(path, sizeof(path), "%sDesignVolume.stl", base);
  if (topx_write_design_stl(mxGetPr(V), (int)d[0], (int)d[1], (int)d[2], 0.5, path, NULL) != TOPX_OK)
    mexErrMsgIdAndTxt("topx:error", "cannot write %s", path);
}

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  char cons[16], prec[16], vcyc[16];
  if (nrhs == 3 && mxIsChar(prhs[0])) {
    char cmd[16];
    mxGetString(prhs[0], cmd, sizeof(cmd));
    if (strcmp(cmd, "write_design") != 0) mexErrMsgIdAndTxt("topx:arg", "Wrong Input!");
    write_design(prhs[1], prhs[2]);
    return;
  }
  topx_params p;
  topx_info info;
  topx_iter* hist = NULL;
  int loops = 0, consType, nLoop, k;
  double V0, rMin, rHat = 0.0, cSolid = 0.0;
  if (nrhs < 5) mexErrMsgIdAndTxt("topx:arg", "Wrong Input!");
  if (mxGetString(prhs[1], cons, sizeof(cons))) mexErrMsgIdAndTxt("topx:arg", "consType must be a string");
  consType = strcmp(cons, "LOCAL") == 0 ? TOPX_LOCAL : TOPX_GLOBAL;
  if (consType == TOPX_LOCAL && nrhs < 6) mexErrMsgIdAndTxt("topx:arg", "Wrong Input!");
  V0 = scalar_arg(prhs[2], "V0");
  nLoop = (int)scalar_arg(prhs[3], "nLoop");
  rMin = scalar_arg(prhs[4], "rMin");
  if (nrhs >= 6 && !mxIsEmpty(prhs[5])) rHat = scalar_arg(prhs[5], "rHat");
  strcpy(prec, "fp64");
  if (nrhs >= 7) mxGetString(prhs[6], prec, sizeof(prec));
  strcpy(vcyc, "Adapted");
  if (nrhs >= 8) mxGetString(prhs[7], vcyc, sizeof(vcyc));
  if (strcmp(vcyc, "Adapted") != 0 && strcmp(vcyc, "Standard") != 0)
    mexErrMsgIdAndTxt("topx:arg", "typeVcycle must be 'Adapted' or 'Standard'");

  topx_default_params(&p);
  p.precision = strcmp(prec, "mixed") == 0 ? TOPX_MIXED : TOPX_FP64;
  p.typeVcycle = strcmp(vcyc, "Standard") == 0 ? TOPX_VCYCLE_STANDARD : TOPX_VCYCLE_ADAPTED;
  if (nrhs >= 9) {
    if (!mxIsNumeric(prhs[8]) || mxGetNumberOfElements(prhs[8]) != 3)
      mexErrMsgIdAndTxt("topx:arg", "specifyPassiveRegions must have 3 entries");
    for (k = 0; k < 3; ++k) p.specifyPassiveRegions[k] = (int)(mxGetPr(prhs[8])[k] + (mxGetPr(prhs[8])[k] >= 0 ? 0.5 : -0.5));
  }
  topx_mex_cleanup();
  check(topx_create(&g_ctx, &p), "topx_create");
  mexAtExit(topx_mex_cleanup);

  if (mxIsChar(prhs[0])) {
    char* path = mxArrayToString(prhs[0]);
    topx_status s = topx_load_topvoxel(g_ctx, path);
    mxFree(path);
    check(s, "topx_load_topvoxel");
  } else if (mxIsLogical(prhs[0]) && mxGetNumberOfDimensions(prhs[0]) == 3) {
    const mwSize* d = mxGetDimensions(prhs[0]);
    const mxLogical* v = mxGetLogicals(prhs[0]);
    check(topx_load_voxels(g_ctx, (const uint8_t*)v, (int)d[0], (int)d[1], (int)d[2]), "topx_load_voxels");
  } else {
    mexErrMsgIdAndTxt("topx:arg", "Inappropriate Input Model!");
  }
  check(topx_get_info(g_ctx, &info), "topx_get_info");
  hist = (topx_iter*)mxCalloc((size_t)(nLoop > 0 ? nLoop : 1), sizeof(topx_iter));
  check(topx_run(g_ctx, consType, V0, nLoop, rMin, rHat, hist, &loops, &cSolid), "topx_run");

  if (nlhs > 0) {
    const char* f[] = {"cSolid", "c", "vol", "sharp", "cons", "change", "its",
                       "tAssemble", "tCG", "tOpti", "tFilter", "tTotal"};
    mxArray* h = mxCreateStructMatrix(1, 1, 12, f);
    mxArray* a[11];
    for (k = 0; k < 11; ++k) a[k] = mxCreateDoubleMatrix((mwSize)loops, k == 5 ? (mwSize)info.numLoadCases : 1, mxREAL);
    for (k = 0; k < loops; ++k) {
      int lc;
      mxGetPr(a[0])[k] = hist[k].c;
      mxGetPr(a[1])[k] = hist[k].vol;
      mxGetPr(a[2])[k] = hist[k].sharp;
      mxGetPr(a[3])[k] = hist[k].cons;
      mxGetPr(a[4])[k] = hist[k].change;
      for (lc = 0; lc < info.numLoadCases && lc < 8; ++lc) mxGetPr(a[5])[k + (size_t)loops * lc] = hist[k].its[lc];
      mxGetPr(a[6])[k] = hist[k].t_assemble;
      mxGetPr(a[7])[k] = hist[k].t_cg;
      mxGetPr(a[8])[k] = hist[k].t_opt;
      mxGetPr(a[9])[k] = hist[k].t_filter;
      mxGetPr(a[10])[k] = hist[k].t_total;
    }
    mxSetField(h, 0, "cSolid", mxCreateDoubleScalar(cSolid));
    for (k = 0; k < 11; ++k) mxSetField(h, 0, f[k + 1], a[k]);
    plhs[0] = h;
  }
  if (nlhs > 1) {
    plhs[1] = mxCreateDoubleMatrix((mwSize)info.numElements, 1, mxREAL);
    check(topx_get_density(g_ctx, mxGetPr(plhs[1]), (size_t)info.numElements), "topx_get_density");
  }
  if (nlhs > 2) {
    const char* f[] = {"resX", "resY", "resZ", "eleMapBack"};
    mxArray* g = mxCreateStructMatrix(1, 1, 4, f);
    mxArray* emb = mxCreateNumericMatrix((mwSize)info.numElements, 1, mxINT32_CLASS, mxREAL);
    size_t need = 0;
    check(topx_get_index_array(g_ctx, 1, TOPX_ARR_ELEMAPBACK, (int32_t*)mxGetData(emb), (size_t)info.numElements, &need),
          "topx_get_index_array");
    mxSetField(g, 0, "resX", mxCreateDoubleScalar(info.resX[0]));
    mxSetField(g, 0, "resY", mxCreateDoubleScalar(info.resY[0]));
    mxSetField(g, 0, "resZ", mxCreateDoubleScalar(info.resZ[0]));
    mxSetField(g, 0, "eleMapBack", emb);
    plhs[2] = g;
  }
  mxFree(hist);
}
