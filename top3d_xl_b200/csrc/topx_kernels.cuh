// Launch wrappers of the TOP3D_XL sm_100a kernels (all asynchronous on `st`).
#pragma once

#include <cstdint>
#include <vector>
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
// out = K p, p'q reduced into sc->pq, and p stored into pout when given (a buffer other than in);
// with yacc given (PCG mode only), also the previous step's y += sc->lam * p_in (not on the first step).
enum KuMode { KU_PLAIN = 0, KU_P_UPDATE = 2 };

// element matrices in constant memory
void upload_ke(const double* Ke576);

// --- level-1 elasticity --------------------------------------------------
// Tiles of the level-1 K*u launch that own a node of the domain (ku_active_tiles); a null list
// launches the whole grid
struct KuTiles {
  const uint32_t* list = nullptr;
  int n = 0;
  // the last-row kernel's (x, z) tiles that hold a present node of the row y = ny (x | z << 16);
  // used when list is given (non-null with nrows = 0: no last-row launch)
  const uint32_t* rows = nullptr;
  int nrows = 0;
  // per listed tile, the planes [lo, hi) of its z-chunk that hold a present node (lo | hi << 16);
  // the tile kernel marches only those (null: the whole chunk)
  const uint32_t* zr = nullptr;
};
// zranges (optional): the z-range entry of each listed tile
std::vector<uint32_t> ku_active_tiles(Grid g, const std::vector<uint8_t>& present,
                                      std::vector<uint32_t>* zranges = nullptr);
std::vector<uint32_t> ku_active_row_tiles(Grid g, const std::vector<uint8_t>& present);
template <typename T>
void launch_ku(cudaStream_t st, KuMode mode, Grid g, const T* in, const T* z, T* pout, T* out, const T* E,
               const uint8_t* fixbits, const T* cfix, PcgScalars* sc, RedScratch rs, KuTiles tiles = KuTiles{},
               double* yacc = nullptr);
template <typename TE, typename T = TE>
void launch_diag_l1(cudaStream_t st, Grid g, const TE* E, const uint8_t* fixbits, const TE* cfix,
                    const uint8_t* present, T* d);
// p = z (+ beta p); y += lambda p; r -= lambda q; ||r|| stop test into sc.  z null: p already holds
// the new direction (K*u in PCG mode wrote it through pout) and is only read, and y is not touched:
// lambda goes to sc->lam, for the next K*u (yacc) or launch_pcg_flush to apply
template <typename T, typename TY>
void launch_pcg_update(cudaStream_t st, Grid g, TY* y, const T* z, T* p, T* r, const T* q, PcgScalars* sc,
                       RedScratch rs, const uint32_t* act = nullptr);
// y += sc->lam * p: the solution step of the last PCG iteration
void launch_pcg_flush(cudaStream_t st, Grid g, double* y, const double* p, const PcgScalars* sc,
                      const uint32_t* act = nullptr);
template <typename T>
void launch_residual_init(cudaStream_t st, Grid g, const T* b, const T* Ay, T* r, PcgScalars* sc, RedScratch rs,
                          double tol, int maxIT);
// --- transfers -----------------------------------------------------------
template <typename TI, typename T>
// cols: bit q set when the fine grid's (x, z) column q = x + nnx z holds a present node (null: all)
void launch_restrict(cudaStream_t st, int span, const TI* in, Grid gf, T* tmp1, T* tmp2, T* out, Grid gc,
                     const uint32_t* cols = nullptr);
// x = omega*(r/d) + P(xc) + (omega*r)/d on present fine nodes; with dot: z.r
// into sc (init: x1 = z.r; else beta = z.r/x1, x1 = z.r)
template <typename TX, typename T, typename TD>
// act: the fine grid's chunk mask (chunk_active), or null
void launch_prolong_smooth(cudaStream_t st, int span, const TX* xc, Grid gc, const T* r, const TD* d,
                           const uint8_t* present, T* x, Grid gf, double omega, bool dot, bool init,
                           PcgScalars* sc, RedScratch rs, const uint32_t* act = nullptr);
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
// W8: the child prolongation weights W_c[a'][b] (child c, child node a', coarse node b) at c * 64 + 8 a' + b
void launch_galerkin_span2(cudaStream_t st, Grid gc, const double* Ksf, const uint8_t* cpresent, const double* W8,
                           double* Ks);
template <typename T>
void launch_diag_coarse(cudaStream_t st, Grid g, const double* Ks, const uint8_t* present, T* d);

// caches the SM count used to shape the K*u launch (call once per device, outside capture)
void prepare_fem_kernels();

// Control words of the persistent coarse solve (zeroed before first use; err != 0 after a CTA
// gave up waiting, and then the words, and the solve's counters, must be zeroed again).
struct CoopControl {
  unsigned idle;   // a counter that nothing raises (the wait self-test); zero
  unsigned exits;  // CTAs that left the launch (the last one re-arms the counters); zero between launches
  int err;         // 0, or kCoopErrWait once a wait gave up
  int pad;
};
constexpr int kCoopErrWait = 1;  // a wait for another CTA's tasks (dataflow solve) gave up
// Self-test of the dataflow solve's bounded dependency wait: one CTA waits for a counter that
// nothing raises, gives up within about a second and sets ctl->err to kCoopErrWait.
void launch_coop_wait_selftest(cudaStream_t st, CoopControl* ctl);

}  // namespace topx
