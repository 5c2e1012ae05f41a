// Device buffers of the nested-dissection factorisation of the coarsest level (topx_nd.hpp) and
// its launches (topx_nd.cu).
#pragma once

#include <cuda_runtime.h>

#include "topx_kernels.cuh"
#include "topx_nd.hpp"

namespace topx {

struct NDDevice {
  const NDFront* fronts = nullptr;
  const NDTask* tasks = nullptr;
  const NDAsm* asmb = nullptr;
  const int64_t* pad = nullptr;
  const int32_t* upd_map = nullptr;
  const int32_t* sep_dof = nullptr;
  const int32_t* upd_dof = nullptr;
  const int32_t* src0 = nullptr;
  const int32_t* src1 = nullptr;
  double* pool = nullptr;   // tiles (FP64)
  double* scr = nullptr;    // P^-1 and R_j tiles of the level being swept
  double* wvec = nullptr;   // per position: F11^-1 f1 and the update vectors
  double* part = nullptr;   // per solve task: partial sums of its chunk (64)
  unsigned* cnt = nullptr;  // per output tile: chunks done (zero between launches)
  // coop_ctas > 0: the solve runs as one persistent dataflow launch of this many CTAs, over the
  // tasks in dependency order (NDPlan::flow) with 2 x fronts counters and the control words
  int coop_ctas = 0;
  const NDTask* flow = nullptr;
  unsigned* flow_done = nullptr;
  CoopControl* ctl = nullptr;
  // assembly, extend-add and the sweep of every front: pool <- the factor of the coarsest
  // matrix whose element operators (576 per dense element of grid g) are Ks
  void factor(cudaStream_t st, const NDPlan& P, Grid g, const double* Ks) const;
  // x = K^-1 b on the coarsest grid's SoA DOF vectors; tiles: pool or an FP32 copy of it.  With
  // sc given, every launch returns at once once sc->done is set (a converged PCG).
  template <typename T, typename TM>
  void solve(cudaStream_t st, const NDPlan& P, const TM* tiles, const T* b, T* x, const PcgScalars* sc) const;
};

// kernel attributes (once per device; outside stream capture)
void prepare_nd_kernels();
// CTAs of the persistent solve on the current device (all resident), or 0 when the device has
// no cooperative launch
int nd_solve_coop_ctas();

}  // namespace topx
