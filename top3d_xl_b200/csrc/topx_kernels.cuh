// Launch wrappers of the TOP3D_XL sm_100a kernels (all asynchronous on `st`).
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>

#include "topx_device.cuh"

namespace topx {

struct CudaError : std::runtime_error {
  cudaError_t code;
  CudaError(cudaError_t e, const char* expr, const char* file, int line)
      : std::runtime_error(std::string(cudaGetErrorString(e)) + " at " + file + ":" + std::to_string(line) +
                           " (" + expr + ")"),
        code(e) {}
};
// A bounded device wait gave up (its poll limit ran out); the engine has cleared the error word
// and stays usable.
struct DeviceWaitError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

// Dense padded grid of one multigrid level: ny, nx, nz elements; node fields
// are SoA with plane stride `stride` (>= (ny+1)(nx+1)(nz+1)).
struct Grid {
  int ny = 0, nx = 0, nz = 0;
  int64_t stride = 0;
  __host__ __device__ int nny() const { return ny + 1; }
  __host__ __device__ int nnx() const { return nx + 1; }
  __host__ __device__ int nnz() const { return nz + 1; }
  __host__ __device__ int64_t nnodes() const { return int64_t(ny + 1) * (nx + 1) * (nz + 1); }
  __host__ __device__ int64_t nelems() const { return int64_t(ny) * nx * nz; }
};

// KU_PLAIN: out = K in.  KU_P_UPDATE: p = z (first PCG step) or z + beta*p_in,
// out = K p, p'q reduced into sc->pq, and p stored into pout when given (a buffer other than in).
enum KuMode { KU_PLAIN = 0, KU_P_UPDATE = 2 };

// element matrices in constant memory
void upload_ke(const double* Ke576);

// --- level-1 elasticity --------------------------------------------------
template <typename T>
void launch_ku(cudaStream_t st, KuMode mode, Grid g, const T* in, const T* z, T* pout, T* out, const T* E,
               const uint8_t* fixbits, const T* cfix, PcgScalars* sc, RedScratch rs);
template <typename TE, typename T = TE>
void launch_diag_l1(cudaStream_t st, Grid g, const TE* E, const uint8_t* fixbits, const TE* cfix,
                    const uint8_t* present, T* d);
// p = z (+ beta p); y += lambda p; r -= lambda q; ||r|| stop test into sc.  z null: p already holds
// the new direction (K*u in PCG mode wrote it through pout) and is only read
template <typename T, typename TY>
void launch_pcg_update(cudaStream_t st, Grid g, TY* y, const T* z, T* p, T* r, const T* q, PcgScalars* sc,
                       RedScratch rs);
template <typename T>
void launch_residual_init(cudaStream_t st, Grid g, const T* b, const T* Ay, T* r, PcgScalars* sc, RedScratch rs,
                          double tol, int maxIT);
// --- transfers -----------------------------------------------------------
template <typename TI, typename T>
void launch_restrict(cudaStream_t st, int span, const TI* in, Grid gf, T* tmp1, T* tmp2, T* out, Grid gc);
// x = omega*(r/d) + P(xc) + (omega*r)/d on present fine nodes; with dot: z.r
// into sc (init: x1 = z.r; else beta = z.r/x1, x1 = z.r)
template <typename TX, typename T, typename TD>
void launch_prolong_smooth(cudaStream_t st, int span, const TX* xc, Grid gc, const T* r, const TD* d,
                           const uint8_t* present, T* x, Grid gf, double omega, bool dot, bool init,
                           PcgScalars* sc, RedScratch rs);
// 'Standard' V-cycle (TX:758-763, 772-777): x = omega*(r/d) + P(xc) without the smoothing term;
// x = omega*(r/d); q = r - q; x += omega*(r - q)/d (with dot: z.r into sc as above); coarse-level
// K*u with the stored Galerkin matrices Ks (dense elements x 576).  All skip once sc->done.
template <typename TX, typename T, typename TD>
void launch_prolong_add(cudaStream_t st, int span, const TX* xc, Grid gc, const T* r, const TD* d,
                        const uint8_t* present, T* x, Grid gf, double omega, PcgScalars* sc);
template <typename TR, typename T, typename TD>
void launch_jacobi_pre(cudaStream_t st, Grid g, const TR* r, const TD* d, const uint8_t* present, T* x, double omega,
                       const PcgScalars* sc);
template <typename TR, typename T>
void launch_residual_inplace(cudaStream_t st, Grid g, const TR* r, T* q, const PcgScalars* sc);
template <typename TR, typename T, typename TD>
void launch_jacobi_correct(cudaStream_t st, Grid g, const TR* r, const T* q, const TD* d, const uint8_t* present,
                           T* x, double omega, bool dot, bool init, PcgScalars* sc, RedScratch rs);
void launch_ku_coarse(cudaStream_t st, Grid g, const double* Ks, const uint8_t* epresent, const uint8_t* present,
                      const double* u, double* y, const PcgScalars* sc);
// --- conversions -----------------------------------------------------------
template <typename TA, typename TB>
void launch_convert(cudaStream_t st, const TA* a, TB* b, int64_t n);
template <typename T>
void launch_compact_to_grid_nodes(cudaStream_t st, const double* src, T* dst, Grid g, const int32_t* nodMapBack0,
                                  int64_t numNodes);
template <typename T>
void launch_grid_to_compact_nodes(cudaStream_t st, const T* src, double* dst, Grid g, const int32_t* nodMapBack0,
                                  int64_t numNodes);
void launch_simp_scatter(cudaStream_t st, const double* xPhys, const int32_t* eleMapBack0, int64_t Ne, double Emin,
                         double E0, double penal, double* Ed, float* Ef);
void launch_fill_scatter(cudaStream_t st, const int32_t* eleMapBack0, int64_t Ne, double val, double* Ed, float* Ef);
// ce_e = u_e^T Ke u_e (load-case weighted, accumulated into ce when accumulate)
void launch_unit_compliance(cudaStream_t st, Grid g, const double* U, const int32_t* eleMapBack0, int64_t Ne,
                            double weight, bool accumulate, double* ce);

// --- coarse levels -----------------------------------------------------------
void launch_galerkin_l2(cudaStream_t st, Grid gc, const double* Efine, const double* Tm, double* Ks);
void launch_galerkin_l2_flagged(cudaStream_t st, Grid gc, const double* Efine, int nflag, const int32_t* fl_elem,
                                const int32_t* fl_tsel, const double* fl_F, const double* Tall, double* Ks);
void launch_galerkin_span2(cudaStream_t st, Grid gc, const double* Ksf, const uint8_t* cpresent, const double* P8,
                           double* Ks);
template <typename T>
void launch_diag_coarse(cudaStream_t st, Grid g, const double* Ks, const uint8_t* present, T* d);

// Slab block-LDL^T of the coarsest level (node grid split into slabs along `axis`)
struct SlabInfo {
  int axis = 0;        // 0:y 1:x 2:z
  int ns = 0;          // number of slabs
  int nu = 0, nv = 0;  // in-slab node dims (u varies fastest)
  int m = 0;           // DOFs per slab = 3*nu*nv
};
void launch_slab_assemble(cudaStream_t st, Grid g, SlabInfo si, const double* Ks, const uint8_t* present, double* A,
                          double* Bup);
// one-time per-device kernel attributes of the coarse factorisation (call outside stream capture)
void prepare_coarse_kernels();
// caches the SM count used to shape the K*u launch (call once per device, outside capture)
void prepare_fem_kernels();
// Dataflow Gauss-Jordan inverse (topx_gjflow.cu): ticket-ordered task tables for one and two
// matrices (gf_plan), ring scratch (gf_scratch_doubles) and control words (gf_ctrl_words; word
// 0 is the error flag, set when a wait gave up, read and cleared by the host).
struct GJFlow {
  const uint32_t* tasks[2];
  unsigned ntasks[2];
  double* scratch;
  unsigned* ctrl;
  int nctas;
  double* ytmp;  // 2 m x m: the coupling terms of the Schur complements, by rows, before transposition
};
// one-time per-device kernel attributes (call outside stream capture)
void prepare_gj_flow();
// CTAs of one inverse launch of order m: every SM for an engine alone on the GPU, else a few
int gj_flow_ctas(bool whole_gpu, int m);
// in-place inverse of the SPD m x m matrices A0 (and A1 when nset == 2)
void launch_gj_flow(cudaStream_t st, int m, int nset, double* A0, double* A1, const uint32_t* tasks,
                    unsigned ntasks, double* scratch, unsigned* ctrl, int nctas);
// twisted block factorisation of the slab-tridiagonal coarsest matrix: Inv (ns m x m inverses of the
// Schur complements), X (ns-1 coupling blocks L_s / U_s) and XT (their transposes)
void launch_slab_factor(cudaStream_t st, const GJFlow& gf, SlabInfo si, const double* A, const double* Bup,
                        double* Inv, double* X, double* XT);
// x = K_coarsest^{-1} b; bs, W, V, xs are ns*m FP64 scratch vectors in slab order
template <typename T, typename TM>
void launch_slab_solve(cudaStream_t st, Grid g, SlabInfo si, const TM* Inv, const TM* X, const TM* XT, const T* b,
                       double* bs, double* W, double* V, double* xs, T* x, const PcgScalars* sc);

// State of the grid-wide barrier of the cooperative coarse solve (zeroed before first use;
// err != 0 after a CTA gave up waiting, and then count must be zeroed again).
struct CoopBarrier {
  unsigned count;
  unsigned gen;
  int err;  // 0, or the kind of wait that gave up first (kCoopErrBarrier, kCoopErrVector)
  int pad;
};
constexpr int kCoopErrBarrier = 1;  // a grid barrier wait gave up
constexpr int kCoopErrVector = 2;   // a wait for an entry of a solve vector gave up
// Self-test of the coarse solve's bounded waits (which: 0 grid barrier, 1 single entry, 2 vector
// of entries) against words that nothing writes; `absent` holds 65 doubles of scratch.
void launch_coop_wait_selftest(cudaStream_t st, int which, CoopBarrier* bar, double* absent);
// Self-test of the Gauss-Jordan inverse's bounded dependency wait: waits for *word >= 1 where
// nothing writes `word` (zeroed here); gives up and sets ctrl[0].
void launch_gf_wait_selftest(cudaStream_t st, unsigned* ctrl, unsigned* word);
// CTAs of launch_slab_solve_coop on the current device (one per SM), or 0 when cooperative
// launch is unavailable; sets the kernels' shared-memory limit (call outside stream capture).
int slab_solve_coop_ctas(int m);
// the coarse solve above as one cooperative launch (same factors; rows summed in another order)
template <typename T, typename TM>
void launch_slab_solve_coop(cudaStream_t st, int nctas, Grid g, SlabInfo si, const TM* Inv, const TM* X, const TM* XT,
                            const T* b, double* bs, double* W, double* V, double* xs, T* x, const PcgScalars* sc,
                            CoopBarrier* bar);

}  // namespace topx
