// Launch wrappers of the optimiser-side kernels (filter, objective, OC, MMA).
#pragma once

#include "topx_kernels.cuh"

namespace topx {

struct ObjState {
  double cObj;  // E . ceNorm
  double xsum;  // sum(xPhys)
};

struct OcState {
  double l1, l2, lmid, fval;
  double change, sharpsum;
  int converged;
  int steps;
};

enum EwOp { EW_COPY = 0, EW_MUL = 1, EW_DIV_MAXX = 2 };

// --- PDE filter ------------------------------------------------------------
// 8x8 element matrix of the Helmholtz filter (TOP3D_XL.m:845-853), passed by value to kernels
template <typename T>
struct FilterKe {
  T v[64];
};
template <typename T>
FilterKe<T> filter_ke(const double* KF64);
template <typename T>
void launch_filter_e2n(cudaStream_t st, Grid g, const T* srcE, T* node, const uint32_t* act = nullptr);
template <typename T>
void launch_filter_diag(cudaStream_t st, Grid g, const uint8_t* solid, const FilterKe<double>& kf, T* dp);
template <typename T>
void launch_filter_ku(cudaStream_t st, KuMode mode, Grid g, const FilterKe<T>& kf, const T* in, const T* z, T* pout,
                      T* out, const uint8_t* solid, PcgScalars* sc, RedScratch rs, KuTiles tiles = KuTiles{});
// tiles of the filter's K*u launch that own a node of the domain (a null list launches them all)
std::vector<uint32_t> filter_active_tiles(Grid g, const std::vector<uint8_t>& present);
template <typename T>
void launch_filter_residual_init(cudaStream_t st, Grid g, const T* b, const T* dp, T* r, T* z, T* y, PcgScalars* sc,
                                 RedScratch rs, double tol, int maxIT, const uint32_t* act = nullptr);
template <typename T>
void launch_filter_update(cudaStream_t st, Grid g, T* y, T* p, T* r, const T* q, const T* dp, T* z, PcgScalars* sc,
                          RedScratch rs, const uint32_t* act = nullptr);
template <typename T>
void launch_filter_n2e(cudaStream_t st, Grid g, const T* node, const int32_t* eleMapBack0, int64_t Ne, double* out);
template <typename T>
void launch_scatter_elems_t(cudaStream_t st, const double* src, const int32_t* eleMapBack0, int64_t Ne, T* dstE);

// --- objective / OC --------------------------------------------------------
void launch_objective(cudaStream_t st, int64_t Ne, const double* ce, const double* xPhys, double cSolid, double Emin,
                      double E0, double penal, double* dc, ObjState* os, RedScratch rs);
void launch_sum(cudaStream_t st, int64_t n, const double* a, const double* b, double* out, RedScratch rs);
void launch_ewise(cudaStream_t st, int op, int64_t n, const double* a, const double* b, double* out, double s);
// OC bisection (TOP3D_XL.m:145-156): w = x sqrt(-dc) once, then bisection steps on lmid,
// kOcStepsPerLaunch of them per launch of launch_oc_bisect
constexpr int kOcStepsPerLaunch = 3;
void launch_oc_prep(cudaStream_t st, int64_t Ne, const double* x, const double* dc, double* w);
void launch_oc_bisect(cudaStream_t st, int64_t Ne, const double* x, const double* w, const uint8_t* passive,
                      OcState* os, RedScratch rs, double move);
void launch_oc_final(cudaStream_t st, int64_t Ne, double* x, const double* w, const uint8_t* passive, double* xPhys,
                     OcState* os, RedScratch rs, RedScratch rs2, double move);

// --- MMA (m = 1) -------------------------------------------------------------
struct MmaState {
  double lam, mu, epsi, err, tol;
  double b;  // constraint constant of the subproblem
  double grad, hess;
  double change;  // max |xnew - xval|
  int inner;      // Newton steps at the current epsilon
  int total;      // Newton steps overall
  int finished;
};
void launch_mma_gensub(cudaStream_t st, int64_t n, int iter, double move, const double* xval, const uint8_t* passive,
                       double* xold1, double* xold2, double* low, double* upp, const double* dfdx, const double* dgdx,
                       double gx, int64_t nact, double* alpha, double* beta, double* p0, double* q0, double* pij,
                       double* qij, MmaState* ms, RedScratch rs);
void launch_mma_newton(cudaStream_t st, int64_t n, const uint8_t* passive, const double* low, const double* upp,
                       const double* alpha, const double* beta, const double* p0, const double* q0, const double* pij,
                       const double* qij, MmaState* ms, RedScratch rs);
void launch_mma_residual(cudaStream_t st, int64_t n, const uint8_t* passive, const double* low, const double* upp,
                         const double* alpha, const double* beta, const double* p0, const double* q0,
                         const double* pij, const double* qij, double* x, MmaState* ms, RedScratch rs);
void launch_mma_finish(cudaStream_t st, int64_t n, const uint8_t* passive, const double* xmma, const double* xold1,
                       double* x, MmaState* ms, RedScratch rs);
// LOCAL driver elementwise chain (TOP3D_XL.m:333-382)
void launch_pnorm_terms(cudaStream_t st, int64_t Ne, const double* xhat, double Ve0, int pPIO, double* out_sum,
                        RedScratch rs);
void launch_local_sens(cudaStream_t st, int64_t Ne, const double* xhat, const double* xTilde, const double* dc,
                       double Ve0, int pPIO, double pn, double betaPIO, double etaPIO, double* dfdx_pde, double* dx,
                       double* dcdx);
void launch_heaviside(cudaStream_t st, int64_t Ne, const double* xTilde, const uint8_t* passive, double betaPIO,
                      double etaPIO, double* xPhys, double* sharpsum, RedScratch rs);

}  // namespace topx
