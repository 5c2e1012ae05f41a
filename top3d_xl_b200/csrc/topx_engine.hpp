// Device engine of the TOP3D_XL B200 path: owns all HBM-resident state of one
// design job (moduli, displacements, multigrid hierarchy, coarse factor, filter
// and optimiser state) and runs the optimisation loop of TOP3D_XL.m
// (GLOBAL: TOP3D_XL.m:40-183, LOCAL: TOP3D_XL.m:225-401) on one GPU.
#pragma once

#include <cuda_runtime.h>

#include <array>
#include <functional>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "topx_kernels.cuh"
#include "topx_mesh.hpp"
#include "topx_nd_dev.hpp"
#include "topx_opt.cuh"

namespace topx {

// Device bytes held by the DevBufs this thread allocated (a job's footprint, measured by the
// thread that builds its engine).
inline int64_t& devbuf_bytes() {
  thread_local int64_t b = 0;
  return b;
}

template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n) {
    o.p = nullptr;
    o.n = 0;
  }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) {
      release();
      p = o.p;
      n = o.n;
      o.p = nullptr;
      o.n = 0;
    }
    return *this;
  }
  ~DevBuf() { release(); }
  void alloc(size_t count, bool zero = true) {
    release();
    if (count) {
      TOPX_CUDA_OK(cudaMalloc(&p, sizeof(T) * count));
      n = count;
      devbuf_bytes() += int64_t(sizeof(T) * count);
      // the default stream's work does not order the engine's non-blocking stream: the zeroing
      // (asynchronous to the host) must be complete before any engine kernel may touch the buffer
      if (zero) {
        TOPX_CUDA_OK(cudaMemsetAsync(p, 0, sizeof(T) * count, 0));
        TOPX_CUDA_OK(cudaStreamSynchronize(0));
      }
    }
  }
  void upload(const T* h, size_t count) {
    alloc(count, false);
    if (count) {  // a copy from pageable memory may still be in flight when cudaMemcpy returns
      TOPX_CUDA_OK(cudaMemcpyAsync(p, h, sizeof(T) * count, cudaMemcpyHostToDevice, 0));
      TOPX_CUDA_OK(cudaStreamSynchronize(0));
    }
  }
  void release() {
    if (p) {
      cudaFree(p);
      devbuf_bytes() -= int64_t(sizeof(T) * n);
    }
    p = nullptr;
    n = 0;
  }
  size_t bytes() const { return sizeof(T) * n; }
};

// PREC_FP64: everything in FP64.  PREC_MIXED: FP32 multigrid preconditioner inside the FP64 Krylov
// iteration, FP64 PDE filter.  PREC_MIXED_F32_FILTER: the PDE filter's CG in FP32 as well.
enum Precision { PREC_FP64 = 0, PREC_MIXED = 1, PREC_MIXED_F32_FILTER = 2 };

struct IterRecord {
  int loop = 0;
  double c = 0, vol = 0, sharp = 0, cons = 0, change = 0;
  std::vector<int> its;  // per load case
  double t_assemble = 0, t_cg = 0, t_opt = 0, t_filter = 0, t_lvf = 0, t_total = 0;
  int filter_its = 0;
};

// Level-1 Krylov vectors of the PCG (always FP64: operator, residual, dots).
struct KrylovWork {
  DevBuf<double> r, z, p, q;
  DevBuf<double> p2;  // the direction alternates between p and p2 (K*u reads one, writes the other)
};

// Multigrid preconditioner workspace in its storage precision TC (double for
// the plain FP64 path, float for the mixed path): Jacobi diagonals and the
// residual/correction fields of every level.
template <typename TC>
struct VWork {
  DevBuf<TC> d1;
  std::vector<DevBuf<TC>> rl, xl, dl;  // per level (index = level-1; level 1 uses the Krylov vectors)
  DevBuf<TC> tmp1, tmp2;                // separable restriction passes
};

// PDE-filter workspace (scalar node fields) in precision TF.
template <typename TF>
struct FWork {
  DevBuf<TF> fr, fz, fp, fq, fy, fb, fsrc;
  std::array<DevBuf<TF>, 2> fdp;
};

class Engine {
 public:
  Engine(Model& model, int precision, int device, bool coarse_coop = true);
  ~Engine();

  // ---- design state -----------------------------------------------------
  void set_xphys(const double* h_xPhys);  // host, compact order
  void get_xphys(double* h_xPhys) const;
  void get_U(int lc, double* h_U) const;  // interleaved compact DOFs
  void set_U(int lc, const double* h_U);

  // ---- building blocks (device-resident) -----------------------------------
  void update_moduli(const double* d_xPhys, bool solid);  // SIMP -> E (dense)
  void assemble();                                        // diagonals, Galerkin, coarse factor
  int solve(int lc);                                      // PCG for load case lc (warm start U)
  void compliance(double* d_ce);                          // load-weighted unit compliance
  int filter(int slot, const double* d_src, double* d_out);
  void setup_filter(int slot, double rmin);

  // host-buffer entry points of the C ABI
  void set_moduli_host(const double* h_E);
  int pcg_host(int lc, double* h_u);
  int filter_host(double rmin, const double* h_src, double* h_out);
  void compliance_host(const double* h_U, double* h_ce);
  // for tests: y = K u (FP64), z = M r (V-cycle in the engine precision)
  void apply_K(const double* h_u, double* h_y);
  // y = K u on device vectors (compact DOF order) with caller-provided grid scratch; topx_noalloc.cu
  void apply_K_device(const double* d_u, double* d_y, double* grid_u, double* grid_y);
  void apply_vcycle(const double* h_r, double* h_z);
  // runs one bounded device wait into its poll limit (test of the give-up path)
  void selftest_wait(int which);
  void get_diag(int level, double* h_d) const;

  // ---- optimisation drivers ------------------------------------------------
  void begin(int consType, double V0, int nLoop, double rMin, double rHat);
  bool step(IterRecord& rec);  // false when the loop condition ends the run
  double cSolid() const { return cSolid_; }
  int loop() const { return loop_; }
  const std::string& info() const { return info_; }

  // ---- measurement ----------------------------------------------------------
  // device timer on the engine stream; per-launch timing of the level-1 K*u
  // kernel inside PCG solves (events around each launch, read after each chunk)
  void timer_start();
  double timer_stop_ms();
  void set_profiling(bool on);
  // per-section device time (ms) and launch-group counts since profiling was switched on
  enum Section { SEC_KU = 0, SEC_UPDATE, SEC_RESTRICT, SEC_COARSE_SOLVE, SEC_PROLONG, SEC_DIAG, SEC_GALERKIN2,
                 SEC_GALERKIN3, SEC_SLAB_ASSEMBLE, SEC_SCHUR, SEC_INVERSE, SEC_FILTER, SEC_OC, SEC_COMPLIANCE,
                 SEC_COUNT };
  static const char* section_name(int s);
  double sec_ms[SEC_COUNT] = {};
  int64_t sec_n[SEC_COUNT] = {};
  double prof_ku_ms = 0.0;
  int64_t prof_ku_launches = 0;
  int64_t prof_pcg_its = 0;

  Model& M;
  int prec;
  bool pre32() const { return prec != PREC_FP64; }              // FP32 multigrid preconditioner
  bool flt32() const { return prec == PREC_MIXED_F32_FILTER; }  // FP32 PDE-filter CG
  cudaStream_t st = nullptr;
  int nl = 0;
  std::vector<Grid> G;  // per level
  int64_t Ne = 0, Nn = 0;

 private:
  template <typename TC>
  void alloc_vwork(VWork<TC>& v);
  template <typename TF>
  void alloc_fwork(FWork<TF>& f);
  template <typename TC>
  void vcycle_t(VWork<TC>& v, bool init, PcgScalars* sc);
  void vcycle_standard(bool init, PcgScalars* sc);
  void vcycle(bool init, PcgScalars* sc);
  int pcg(const double* b, double* y, bool warm, double tol, int maxIT);
  template <typename TF>
  int filter_t(FWork<TF>& f, int slot, const double* d_src, double* d_out);
  template <typename TF>
  const FilterKe<TF>& filter_ke_of(int slot) const;
  void step_local(IterRecord& rec, const ObjState& os);
  void factor_coarsest();
  void assemble_launches();
  void read_scalars(PcgScalars& h, const PcgScalars* d) const;

  // level-1 static data
  DevBuf<uint8_t> fixbits, solid1;
  std::vector<DevBuf<uint8_t>> present, epresent;  // per level
  DevBuf<int32_t> eleMapBack0, nodMapBack0;
  DevBuf<double> E64, cfix64;        // dense moduli (elements) and fixed-DOF diagonal (nodes)
  std::vector<DevBuf<double>> F, U;  // per load case, dense SoA FP64
  // coarse operators
  std::vector<DevBuf<double>> Ks;  // per level (index = level-1), dense elements x 576
  DevBuf<double> Tall, W8;
  DevBuf<int32_t> fl_elem, fl_tsel;
  DevBuf<double> fl_F;
  int nflag = 0;
  DevBuf<uint32_t> kuTiles;  // level-1 K*u tiles that own a node of the domain
  DevBuf<uint32_t> kuRows;   // and the last-row kernel's tiles that hold one of the row y = ny
  DevBuf<uint32_t> kuZr;     // per listed tile, its planes that hold a present node
  KuTiles kut;               // their list (null: the whole grid)
  DevBuf<uint32_t> filterTiles;  // the same for the filter's K*u (its own z-chunks)
  KuTiles fut;
  DevBuf<uint32_t> act1Mask;     // level-1 chunk mask (chunk_active) of an irregular domain
  const uint32_t* act1 = nullptr;  // null: every chunk holds a present node
  DevBuf<uint32_t> cols1Mask;      // level-1 (x, z) columns that hold a present node
  const uint32_t* cols1 = nullptr;
  // coarsest level: nested-dissection plan, its device copy and the factor tiles
  NDPlan nd;
  NDDevice ndd;
  DevBuf<NDFront> ndFronts;
  DevBuf<NDTask> ndTasks;
  DevBuf<NDAsm> ndAsm;
  DevBuf<int64_t> ndPad;
  DevBuf<int32_t> ndMap, ndSep, ndUpd, ndSrc0, ndSrc1;
  DevBuf<double> ndPool, ndScr, ndW, ndPart;
  DevBuf<unsigned> ndCnt;
  DevBuf<NDTask> ndFlow;   // the solve tasks in dependency order (persistent dataflow solve)
  DevBuf<unsigned> ndDone; // its per-front counters
  DevBuf<float> ndPool32;  // FP32 copy applied by the mixed-precision V-cycle
  DevBuf<CoopControl> coopCtl;  // control words of the persistent coarse solve
  int coopCtas = 0;             // its CTA count; 0: one launch per tree level and direction
  void check_coop_waits();      // waits for the stream; throws if a wait gave up (re-arming the words)
  void check_device_waits() const;  // after a stream sync: throws if a bounded device wait gave up
  // a copy between host and device ordered on the engine's stream, complete when it returns
  void copy_sync(void* dst, const void* src, size_t bytes, cudaMemcpyKind kind) const;
  // workspaces
  KrylovWork kw;
  VWork<double> v64;
  std::vector<DevBuf<double>> vq;  // 'Standard' V-cycle: K x per coarse smoothing level (index = level-1)
  VWork<float> v32;
  FWork<double> f64;
  FWork<float> f32;
  // scalars & reductions
  DevBuf<double> red1, red2;
  DevBuf<unsigned> tickets;
  RedScratch rs1{}, rs2{};
  DevBuf<PcgScalars> scE, scF;
  DevBuf<ObjState> objS;
  DevBuf<OcState> ocS;
  DevBuf<MmaState> mmaS;
  DevBuf<double> dscal;
  PcgScalars* h_sc = nullptr;  // pinned
  CoopControl* h_ctl = nullptr;  // pinned
  // optimiser state (compact, FP64)
  DevBuf<double> x, xPhys, dc, ce, tmpA, tmpB, xTilde, xhat, dfdx, dxv, volMax;
  DevBuf<double> xold1, xold2, low, upp, alpha, beta, p0, q0, pij, qij, xmma, xmin, xmax;
  DevBuf<uint8_t> passive;
  std::array<double, 2> filterR{{0, 0}};
  std::array<FilterKe<double>, 2> filterKe64{};  // filter element matrix per slot
  std::array<FilterKe<float>, 2> filterKe32{};
  // run state
  int consType_ = 0, nLoop_ = 0, loop_ = 0, loopbeta_ = 0;
  int64_t nActive_ = 0;
  double V0_ = 0, rMin_ = 0, rHat_ = 0, cSolid_ = 0, change_ = 1, sharp_ = 1, betaPIO_ = 1;
  std::string info_;
  std::vector<cudaEvent_t> ev;
  bool prof_ = false;
  std::vector<cudaEvent_t> pev;  // pairs around K*u launches of one chunk
  // section profiler: event pairs recorded on the stream, harvested at sync points
  std::vector<cudaEvent_t> sev;
  std::vector<int> sec_of;
  int sev_used = 0;
  void sec_begin(int sec);
  void sec_end();
  void sec_harvest();
  // CUDA graphs of fixed launch sequences, keyed by name; captured on first use and replayed
  // (direct launches while profiling, so the section events stay on the stream)
  struct GraphExec {
    cudaGraphExec_t exec;
    long long kernels;  // kernel launches recorded into it
  };
  std::map<std::string, GraphExec> graphs_;
  void run_graph(const std::string& key, const std::function<void()>& body);
 public:
  bool use_graphs = true;
  cudaEvent_t tev[2] = {nullptr, nullptr};
  cudaEvent_t ev_legacy = nullptr;  // orders device-pointer calls after the legacy default stream
};

// Fixed device scratch of the allocation-free operator call (topx_noalloc.cu): its size in
// bytes, and its device address on `device`, which must be current (looked up once per device).
size_t noalloc_scratch_bytes();
double* noalloc_scratch(int device);

}  // namespace topx
