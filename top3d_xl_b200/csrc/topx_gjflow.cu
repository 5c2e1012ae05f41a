// Dataflow Gauss-Jordan inverse of the coarsest level's Schur complements (in place, FP64,
// up to two matrices at once): one persistent launch whose CTAs claim tile tasks in the
// ticket order of gf_plan (topx_gjflow.hpp) and wait, with bounded polling, for the tile
// versions each task reads.  The critical path (pivot, the panel and column tiles of the
// next pivot block, its diagonal update) runs as soon as its inputs exist while the bulk
// updates of earlier steps fill the other SMs, with no launch boundaries in between.
// Replaces the sparse Cholesky factorisation of the coarsest matrix (chol(K,'lower'),
// TOP3D_XL.m:1065) together with launch_slab_factor's Schur-complement chain.
#include <mutex>

#include "topx_gjflow.hpp"
#include "topx_kernels.cuh"

namespace topx {

namespace {

constexpr int GF_THREADS = 256;
constexpr int GF_LD = GF_T + 8;   // row stride of B operands [t][c] in shared memory (doubles)
constexpr int GF_LDA = GF_T + 4;  // row stride of A operands [r][t] (row-major)
// both strides make a warp's fragment load exactly two shared-memory wavefronts
constexpr int GF_BUF = GF_T * GF_LD;  // doubles per staging buffer
constexpr size_t GF_SMEM = size_t(5) * GF_BUF * sizeof(double);  // five buffers; one holds GFPivotSmem
// polls of the version words before a CTA gives up (each poll sleeps ~100 ns: well under a second)
constexpr unsigned GF_SPIN_LIMIT = 1u << 21;
constexpr int GF_ERR = 0, GF_TICKET = 1;  // control words

struct GFArgs {
  double* A[2];
  const uint32_t* tasks;
  unsigned ntasks;
  int m, nt;
  double* scr;
  unsigned* ctrl;
};

__device__ __forceinline__ unsigned gf_ld_relaxed(const unsigned* p) {
  unsigned v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void gf_st_release(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void gf_red_release_add(unsigned* p, unsigned v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ int gf_ld_volatile(const int* p) { return *reinterpret_cast<const volatile int*>(p); }

// Waits until *p0 >= n0, *p1 >= n1 and *p2 >= n2 (null pointers count as met); the three
// words are polled together.  Returns false, with the error word set, after the poll limit
// or once another CTA has set it.
__device__ bool gf_wait(const unsigned* p0, unsigned n0, const unsigned* p1, unsigned n1, const unsigned* p2,
                        unsigned n2, int* err) {
  for (unsigned it = 0;; ++it) {
    const unsigned v0 = gf_ld_relaxed(p0);
    const unsigned v1 = p1 ? gf_ld_relaxed(p1) : n1;
    const unsigned v2 = p2 ? gf_ld_relaxed(p2) : n2;
    if (v0 >= n0 && v1 >= n1 && v2 >= n2) {
      asm volatile("fence.acq_rel.gpu;" ::: "memory");
      return true;
    }
    if (gf_ld_volatile(err)) return false;
    if (it >= GF_SPIN_LIMIT) {
      atomicExch(err, 1);
      return false;
    }
    __nanosleep(64);
  }
}

__device__ __forceinline__ void gf_cp16(double* s, const double* g) {
  const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(s));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(g) : "memory");
}
__device__ __forceinline__ void gf_cp8(double* s, const double* g) {
  const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(s));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(sa), "l"(g) : "memory");
}
__device__ __forceinline__ void gf_cp_wait() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;" ::: "memory");
}

// s[t][x] (row stride ld) = a contiguous 64 x 64 ring tile g[t * 64 + x] (L2 only: the ring is
// written by other CTAs during the launch)
__device__ __forceinline__ void gf_stage_ring(double* s, const double* g, int ld) {
#pragma unroll
  for (int e = threadIdx.x; e < GF_T * GF_T / 2; e += GF_THREADS) {
    const int t = e >> 5, x = (e & 31) * 2;
    gf_cp16(s + t * ld + x, g + t * GF_T + x);
  }
}
// s[t][x] (row stride ld) = M[r0 + t][c0 + x] for t < nr, x < nc, else 0 (M row-major with row
// stride m, which may be odd: 8-byte asynchronous copies).  The copies are weak loads issued
// after the task's acquire (thread 0's fence, then the CTA barrier), so they observe the
// released tile versions.
__device__ __forceinline__ void gf_stage_rows(double* s, const double* M, int m, int r0, int nr, int c0, int nc,
                                              int ld) {
#pragma unroll 4
  for (int e = threadIdx.x; e < GF_T * GF_T; e += GF_THREADS) {
    const int t = e >> 6, x = e & 63;
    if (t < nr && x < nc)
      gf_cp8(s + t * ld + x, M + int64_t(r0 + t) * m + c0 + x);
    else
      s[t * ld + x] = 0.0;
  }
}
// g[r * 64 + x] = s[r][x] (row stride ld): a staged tile copied into the ring
__device__ __forceinline__ void gf_copy_to_ring(double* g, const double* s, int ld) {
#pragma unroll 4
  for (int e = threadIdx.x; e < GF_T * GF_T / 2; e += GF_THREADS) {
    const int r = e >> 5, x = (e & 31) * 2;
    *reinterpret_cast<double2*>(g + r * GF_T + x) = *reinterpret_cast<const double2*>(s + r * ld + x);
  }
}

// FP64 tensor-core product step D += A B on an 8x8x4 fragment (mma.sync m8n8k4): lane l holds
// A[l/4][l%4], B[l%4][l/4] and D[l/4][2(l%4) + h].
__device__ __forceinline__ void gf_dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// acc[r][c] += sum_t sA[r][t] sB[t][c] over the 64 x 64 tile (sA row stride GF_LDA, sB GF_LD).
// Warp w takes rows 32 (w / 4) .. + 31 and columns 16 (w % 4) .. + 15; this thread's outputs
// are (rb + 8 fr + g, cb + 8 fc + 2 q + h).
__device__ __forceinline__ void gf_product(const double* sA, const double* sB, double (&acc)[4][2][2]) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
  const int rb = (warp >> 2) * 32, cb = (warp & 3) * 16;
#pragma unroll 4
  for (int k4 = 0; k4 < GF_T / 4; ++k4) {
    const int kk = 4 * k4 + q;
    double a[4], b[2];
#pragma unroll
    for (int fr = 0; fr < 4; ++fr) a[fr] = sA[(rb + 8 * fr + g) * GF_LDA + kk];
#pragma unroll
    for (int fc = 0; fc < 2; ++fc) b[fc] = sB[kk * GF_LD + cb + 8 * fc + g];
#pragma unroll
    for (int fr = 0; fr < 4; ++fr)
#pragma unroll
      for (int fc = 0; fc < 2; ++fc) gf_dmma(acc[fr][fc][0], acc[fr][fc][1], a[fr], b[fc]);
  }
}

// Applies f(r, c, value) to this thread's product outputs.
template <typename F>
__device__ __forceinline__ void gf_for_outputs(double (&acc)[4][2][2], F&& f) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
  const int rb = (warp >> 2) * 32, cb = (warp & 3) * 16;
#pragma unroll
  for (int fr = 0; fr < 4; ++fr)
#pragma unroll
    for (int fc = 0; fc < 2; ++fc)
#pragma unroll
      for (int h = 0; h < 2; ++h) f(rb + 8 * fr + g, cb + 8 * fc + 2 * q + h, acc[fr][fc][h]);
}

// PIV works in the last staging buffer of the CTA's dynamic shared memory
struct GFPivotSmem {
  double rowS[2][8][72];   // pivot row block (old values), double-buffered by step
  double colT[2][8][72];   // pivot column block, transposed: colT[t][row]
  double rowR[2][8][72];   // R = -Pinv rowS per warp row (wr)
  double pinv[8][8];
};
static_assert(sizeof(GFPivotSmem) <= GF_BUF * sizeof(double), "pivot workspace exceeds a staging buffer");

// 1/v: hardware reciprocal approximation refined by two Newton-Raphson steps
// x <- x + x (1 - v x) (each doubles the correct bits), off the long IEEE division.
__device__ __forceinline__ double gf_recip(double v) {
  double x;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(x) : "d"(v));
  double e = fma(-v, x, 1.0);
  x = fma(x, e, x);
  e = fma(-v, x, 1.0);
  return fma(x, e, x);
}
// PIV: the 64 x 64 diagonal tile (identity beyond kb) inverted by blocked Gauss-Jordan exchange
// on 8-wide pivot blocks, held in registers in the FP64 tensor-core accumulator layout of
// gf_product (warp (wr, wc) = rows 32 wr.., columns 16 wc..).  Per block S:
//   the owners publish row block A[S, :] and column block A[:, S] to shared memory;
//   warp 0 inverts P = A[S, S] (one pivot per step, operands by shuffles);
//   every warp forms R = -P^-1 A[S, cols] for its columns and then, on the tensor cores,
//   A[i, j] += A[i, S] R_j,  A[i, S] = A[i, S] P^-1,  A[S, j] = R_j,  A[S, S] = P^-1.
// acc: the tile (identity beyond kb) on entry, P^-1 on return.
__device__ __forceinline__ void gf_pivot(double (&acc)[4][2][2], double* __restrict__ M, int m, int k0, int kb,
                                         double* __restrict__ Pinv, GFPivotSmem& sm) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
  const int wr = warp >> 2, wc = warp & 3, rb = wr * 32, cb = wc * 16;
  const int nsteps = (kb + 7) >> 3;
  for (int s = 0; s < nsteps; ++s) {
    const int buf = s & 1;
    const int sfr = s & 3, swr = s >> 2, sfc = s & 1, swc = s >> 1;
    // publish the pivot row block (warps of row half swr, fragment row sfr) and column block
    if (wr == swr) {
#pragma unroll
      for (int fr = 0; fr < 4; ++fr)
        if (fr == sfr)
#pragma unroll
          for (int fc = 0; fc < 2; ++fc)
            *reinterpret_cast<double2*>(&sm.rowS[buf][g][cb + 8 * fc + 2 * q]) = make_double2(acc[fr][fc][0], acc[fr][fc][1]);
    }
    if (wc == swc) {
#pragma unroll
      for (int fc = 0; fc < 2; ++fc)
        if (fc == sfc)
#pragma unroll
          for (int fr = 0; fr < 4; ++fr) {
            sm.colT[buf][2 * q][rb + 8 * fr + g] = acc[fr][fc][0];
            sm.colT[buf][2 * q + 1][rb + 8 * fr + g] = acc[fr][fc][1];
          }
    }
    __syncthreads();
    if (warp == 0) {  // 8 x 8 pivot block inverse, one pivot per step: lane holds P[g][2q], P[g][2q+1]
      double p0 = sm.rowS[buf][g][8 * s + 2 * q], p1 = sm.rowS[buf][g][8 * s + 2 * q + 1];
#pragma unroll
      for (int t = 0; t < 8; ++t) {
        // pivot value in lane 4t + t/2, pivot row at my columns in lane 4t + q, my row's pivot
        // column in lane 4g + t/2
        const double pt = __shfl_sync(0xffffffffu, (t & 1) ? p1 : p0, 4 * t + (t >> 1));
        const double rt0 = __shfl_sync(0xffffffffu, p0, 4 * t + q);
        const double rt1 = __shfl_sync(0xffffffffu, p1, 4 * t + q);
        const double ct = __shfl_sync(0xffffffffu, (t & 1) ? p1 : p0, 4 * g + (t >> 1));
        const double d = gf_recip(pt);
        const double cd = ct * d;
        if (g == t) {
          p0 = (2 * q == t) ? d : -d * rt0;
          p1 = (2 * q + 1 == t) ? d : -d * rt1;
        } else {
          p0 = (2 * q == t) ? cd : fma(-cd, rt0, p0);
          p1 = (2 * q + 1 == t) ? cd : fma(-cd, rt1, p1);
        }
      }
      *reinterpret_cast<double2*>(&sm.pinv[g][2 * q]) = make_double2(p0, p1);
    }
    __syncthreads();
    // R = -Pinv rowS for this warp's 16 columns (D layout: R[g][cb + 8 fc + 2q + h])
    double R[2][2];
#pragma unroll
    for (int fc = 0; fc < 2; ++fc) {
      R[fc][0] = R[fc][1] = 0.0;
#pragma unroll
      for (int k4 = 0; k4 < 2; ++k4)
        gf_dmma(R[fc][0], R[fc][1], sm.pinv[g][4 * k4 + q], sm.rowS[buf][4 * k4 + q][cb + 8 * fc + g]);
      R[fc][0] = -R[fc][0];
      R[fc][1] = -R[fc][1];
      *reinterpret_cast<double2*>(&sm.rowR[wr][g][cb + 8 * fc + 2 * q]) = make_double2(R[fc][0], R[fc][1]);
    }
    __syncwarp();
    // one tensor-core product for every fragment (no branches, so the products interleave):
    // column block S takes C P^-1 (B = P^-1, from zero), all others A + C R; the pivot row
    // block then takes R and the pivot block P^-1
#pragma unroll
    for (int fr = 0; fr < 4; ++fr) {
      double ca[2];  // C operand: C[rb + 8 fr + g][4 k4 + q]
#pragma unroll
      for (int k4 = 0; k4 < 2; ++k4) ca[k4] = sm.colT[buf][4 * k4 + q][rb + 8 * fr + g];
#pragma unroll
      for (int fc = 0; fc < 2; ++fc) {
        const bool inCol = (wc == swc && fc == sfc);
        const double* bsrc = inCol ? &sm.pinv[q][g] : &sm.rowR[wr][q][cb + 8 * fc + g];
        const int bstep = inCol ? 4 * 8 : 4 * 72;  // 4 rows down in pinv or rowR
        acc[fr][fc][0] = inCol ? 0.0 : acc[fr][fc][0];
        acc[fr][fc][1] = inCol ? 0.0 : acc[fr][fc][1];
#pragma unroll
        for (int k4 = 0; k4 < 2; ++k4) gf_dmma(acc[fr][fc][0], acc[fr][fc][1], ca[k4], bsrc[k4 * bstep]);
      }
    }
    if (wr == swr) {
#pragma unroll
      for (int fr = 0; fr < 4; ++fr)
        if (fr == sfr)
#pragma unroll
          for (int fc = 0; fc < 2; ++fc) {
            const bool inCol = (wc == swc && fc == sfc);
            acc[fr][fc][0] = inCol ? sm.pinv[g][2 * q] : R[fc][0];
            acc[fr][fc][1] = inCol ? sm.pinv[g][2 * q + 1] : R[fc][1];
          }
    }
  }
  // outputs: Pinv into the ring and the tile of M
#pragma unroll
  for (int fr = 0; fr < 4; ++fr)
#pragma unroll
    for (int fc = 0; fc < 2; ++fc) {
      const int r = rb + 8 * fr + g, c = cb + 8 * fc + 2 * q;
      *reinterpret_cast<double2*>(Pinv + r * 64 + c) = make_double2(acc[fr][fc][0], acc[fr][fc][1]);
#pragma unroll
      for (int h = 0; h < 2; ++h)
        if (r < kb && c + h < kb) M[int64_t(k0 + r) * m + k0 + c + h] = acc[fr][fc][h];
    }
}
__global__ void __launch_bounds__(GF_THREADS, 1) k_gj_flow(GFArgs f) {
  extern __shared__ __align__(16) double gf_smem[];
  __shared__ unsigned s_task;
  __shared__ int s_ok;
  double* const buf0 = gf_smem;
  double* const buf1 = gf_smem + GF_BUF;
  double* const buf2 = gf_smem + 2 * GF_BUF;
  double* const buf3 = gf_smem + 3 * GF_BUF;
  double* const buf4 = gf_smem + 4 * GF_BUF;
  int* err = reinterpret_cast<int*>(f.ctrl + GF_ERR);
  unsigned* ticket = f.ctrl + GF_TICKET;
  const int tid = threadIdx.x, m = f.m, nt = f.nt;
  const size_t slot_doubles = gf_slot_doubles(m);

  if (tid == 0) s_task = gf_ld_volatile(err) ? f.ntasks : atomicAdd(ticket, 1u);
  __syncthreads();
  for (;;) {
    const unsigned tk = s_task;
    if (tk >= f.ntasks) return;
    unsigned nxt = 0;
    if (tid == 0) nxt = atomicAdd(ticket, 1u);  // the next task, claimed ahead (used after this one)
    int type, mat, k, i, j;
    gf_decode(__ldg(f.tasks + tk), type, mat, k, i, j);
    double* __restrict__ M = mat ? f.A[1] : f.A[0];
    unsigned* ver = f.ctrl + GF_CTRL_HEAD + size_t(mat) * (nt * nt + 2 * nt);
    unsigned* done = ver + nt * nt;
    unsigned* cready = done + nt;  // C of row block k (step k-1) in the ring, set by PIV(k)
    if (tid == 0) {
      bool ok;
      const unsigned* vkk = ver + k * nt + k;
      if (type == GF_PIV)  // the previous pivot and step k-1's three critical tiles, then the ring slot
        ok = (k == 0 || gf_wait(ver + (k - 1) * nt + (k - 1), k, ver + k * nt + (k - 1), k - 1, ver + (k - 1) * nt + k,
                                k - 1, err)) &&
             gf_wait(vkk, k > 0 ? k - 1 : 0, (k >= GF_RING && nt > 1) ? done + (k - GF_RING) : nullptr,
                     unsigned((nt - 1) * (nt - 1)), nullptr, 0, err);
      else if (type == GF_PAN)
        ok = gf_wait(vkk, k + 1, ver + k * nt + j, k, nullptr, 0, err);
      else if (type == GF_COL)
        ok = gf_wait(vkk, k + 1, ver + i * nt + k, k, nullptr, 0, err);
      else  // the tile, R_j, and C_i (whose ring copy PIV(k+1) publishes early for i = k+1)
        ok = gf_wait(ver + i * nt + j, k, ver + k * nt + j, k + 1,
                     i == k + 1 ? cready + i : ver + i * nt + k, i == k + 1 ? 1u : unsigned(k + 1), err);
      s_ok = ok;
    }
    __syncthreads();
    if (!s_ok) return;

    // ring slot of step k: P^-1 (row-major), R_j tiles [t][c], C_i tiles [r][t]
    double* slot = f.scr + (size_t(mat) * GF_RING + size_t(k % GF_RING)) * slot_doubles;
    double* Pinv = slot;
    const int k0 = k * GF_T, kb = min(GF_T, m - k0);
    double acc[4][2][2];
    gf_for_outputs(acc, [&](int, int, double& v) { v = 0.0; });
    if (type == GF_PIV) {
      if (k == 0) {
        gf_for_outputs(acc, [&](int r, int c, double& v) {
          v = (r < kb && c < kb) ? __ldcg(M + int64_t(k0 + r) * m + k0 + c) : (r == c ? 1.0 : 0.0);
        });
      } else {
        // step k-1's critical tiles first (its pivot block is full: only the last block is partial)
        double* pslot = f.scr + (size_t(mat) * GF_RING + size_t((k - 1) % GF_RING)) * slot_doubles;
        const int kp0 = k0 - GF_T;
        gf_stage_ring(buf3, pslot, GF_LDA);              // P_{k-1}^-1 as an A operand
        gf_stage_ring(buf1, pslot, GF_LD);               // ... and as a B operand
        gf_stage_rows(buf0, M, m, k0, kb, kp0, GF_T, GF_LDA);  // C = A[k, k-1]
        gf_stage_rows(buf2, M, m, kp0, GF_T, k0, kb, GF_LD);   // T = A[k-1, k]
        gf_stage_rows(buf4, M, m, k0, kb, k0, kb, GF_LD);      // A[k, k]
        gf_cp_wait();
        __syncthreads();
        double dg[4][2][2];
        gf_for_outputs(dg, [&](int r, int c, double& v) { v = buf4[r * GF_LD + c]; });
        // C into the ring: step k-1's updates of row block k may start
        gf_copy_to_ring(pslot + size_t(1 + nt + k) * GF_T * GF_T, buf0, GF_LDA);
        __syncthreads();
        if (tid == 0) gf_st_release(cready + k, 1u);
        // PAN(k-1, k): R = -P^-1 T into A[k-1, k] and the ring
        gf_product(buf3, buf2, acc);
        __syncthreads();  // every product read of T is done: R takes its buffer
        gf_for_outputs(acc, [&](int r, int c, double v) {
          buf2[r * GF_LD + c] = -v;
          if (c < kb) M[int64_t(kp0 + r) * m + k0 + c] = -v;
        });
        __syncthreads();
        gf_copy_to_ring(pslot + size_t(1 + k) * GF_T * GF_T, buf2, GF_LD);
        __syncthreads();
        if (tid == 0) gf_st_release(ver + (k - 1) * nt + k, unsigned(k));
        // UPD(k-1, k, k): the diagonal tile plus C R, identity beyond kb
        gf_product(buf0, buf2, dg);
#pragma unroll
        for (int fr = 0; fr < 4; ++fr)
#pragma unroll
          for (int fc = 0; fc < 2; ++fc)
#pragma unroll
            for (int h = 0; h < 2; ++h) acc[fr][fc][h] = dg[fr][fc][h];
        gf_for_outputs(acc, [&](int r, int c, double& v) {
          if (r >= kb || c >= kb) v = (r == c) ? 1.0 : 0.0;
        });
      }
      gf_pivot(acc, M, m, k0, kb, Pinv, *reinterpret_cast<GFPivotSmem*>(buf3));
      if (k > 0) {
        // the pivot is out; then COL(k-1, k): A[k, k-1] = C P_{k-1}^-1 (C and P^-1 are still staged)
        __syncthreads();
        if (tid == 0) {
          gf_st_release(ver + k * nt + k, unsigned(k + 1));
          gf_red_release_add(done + (k - 1), 1u);  // the fused UPD(k-1, k, k)
        }
        const int kp0 = k0 - GF_T;
        gf_for_outputs(acc, [&](int, int, double& v) { v = 0.0; });
        gf_product(buf0, buf1, acc);
        gf_for_outputs(acc, [&](int r, int c, double v) {
          if (r < kb) M[int64_t(k0 + r) * m + kp0 + c] = v;
        });
      }
    } else if (type == GF_PAN) {  // R_j = -P^-1 A[K, j] into the ring and A[K, j]
      const int j0 = j * GF_T, cw = min(GF_T, m - j0);
      double* R = slot + size_t(1 + j) * GF_T * GF_T;
      gf_stage_ring(buf0, Pinv, GF_LDA);
      gf_stage_rows(buf1, M, m, k0, kb, j0, cw, GF_LD);
      gf_cp_wait();
      __syncthreads();
      gf_product(buf0, buf1, acc);
      gf_for_outputs(acc, [&](int r, int c, double v) {
        R[r * GF_T + c] = -v;
        if (r < kb && c < cw) M[int64_t(k0 + r) * m + j0 + c] = -v;
      });
    } else if (type == GF_COL) {  // C_i = A[i, K] kept in the ring, A[i, K] = C_i P^-1
      const int i0 = i * GF_T, rh = min(GF_T, m - i0);
      gf_stage_ring(buf1, Pinv, GF_LD);
      gf_stage_rows(buf0, M, m, i0, rh, k0, kb, GF_LDA);
      gf_cp_wait();
      __syncthreads();
      gf_copy_to_ring(slot + size_t(1 + nt + i) * GF_T * GF_T, buf0, GF_LDA);
      gf_product(buf0, buf1, acc);
      gf_for_outputs(acc, [&](int r, int c, double v) {
        if (r < rh && c < kb) M[int64_t(i0 + r) * m + k0 + c] = v;
      });
    } else {  // A[i, j] += C_i R_j
      const int i0 = i * GF_T, rh = min(GF_T, m - i0), j0 = j * GF_T, cw = min(GF_T, m - j0);
      gf_stage_ring(buf0, slot + size_t(1 + nt + i) * GF_T * GF_T, GF_LDA);
      gf_stage_ring(buf1, slot + size_t(1 + j) * GF_T * GF_T, GF_LD);
      gf_stage_rows(buf2, M, m, i0, rh, j0, cw, GF_LD);
      gf_cp_wait();
      __syncthreads();
      gf_for_outputs(acc, [&](int r, int c, double& v) { v = buf2[r * GF_LD + c]; });
      gf_product(buf0, buf1, acc);
      gf_for_outputs(acc, [&](int r, int c, double v) { buf2[r * GF_LD + c] = v; });
      __syncthreads();
#pragma unroll 4
      for (int e = tid; e < GF_T * GF_T; e += GF_THREADS) {  // whole rows: coalesced stores
        const int r = e >> 6, c = e & 63;
        if (r < rh && c < cw) M[int64_t(i0 + r) * m + j0 + c] = buf2[r * GF_LD + c];
      }
    }
    // publish: the barrier orders every thread's stores before one thread's release store of the
    // tile's version (a release is cumulative), as in the usual CTA-semaphore pattern.  A lane of
    // warp 1 releases, so warp 0 can go on to claim and poll the next task meanwhile.
    if (tid == 0) s_task = gf_ld_volatile(err) ? f.ntasks : nxt;
    __syncthreads();
    if (tid == 32) {
      if (type == GF_PIV) {
        if (k == 0)
          gf_st_release(ver, 1u);
        else
          gf_st_release(ver + k * nt + (k - 1), unsigned(k));  // COL(k-1, k)
      } else if (type == GF_PAN) {
        gf_st_release(ver + k * nt + j, unsigned(k + 1));
      } else if (type == GF_COL) {
        gf_st_release(ver + i * nt + k, unsigned(k + 1));
      } else {
        gf_st_release(ver + i * nt + j, unsigned(k + 1));
        gf_red_release_add(done + k, 1u);
      }
    }
  }
}

}  // namespace

void prepare_gj_flow() {
  static std::mutex mu;
  static bool done[64] = {};
  int dev = 0;
  TOPX_CUDA_OK(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  if (dev >= 0 && dev < 64 && done[dev]) return;
  TOPX_CUDA_OK(cudaFuncSetAttribute(k_gj_flow, cudaFuncAttributeMaxDynamicSharedMemorySize, int(GF_SMEM)));
  if (dev >= 0 && dev < 64) done[dev] = true;
}

int gj_flow_ctas(bool whole_gpu, int m) {
  int dev = 0, nsm = 0, per = 0;
  TOPX_CUDA_OK(cudaGetDevice(&dev));
  TOPX_CUDA_OK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  TOPX_CUDA_OK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_gj_flow, GF_THREADS, GF_SMEM));
  per = std::max(1, std::min(per, 2));
  if (whole_gpu) return nsm * per;
  // an engine sharing the GPU: one CTA per tile row, at most an eighth of the SMs (each CTA holds
  // its SM's shared memory while it waits for its next task, which the other jobs' kernels need)
  const int nt = gf_tiles(m);
  return std::max(2, std::min(nsm / 8, nt));
}

// One thread waits, through the inverse's own wait primitive, for a version word that nothing
// writes: it gives up after GF_SPIN_LIMIT polls and sets the error word.
__global__ void k_gf_wait_selftest(unsigned* ctrl, const unsigned* word) {
  if (threadIdx.x == 0) gf_wait(word, 1u, nullptr, 0, nullptr, 0, reinterpret_cast<int*>(ctrl + GF_ERR));
}

void launch_gf_wait_selftest(cudaStream_t st, unsigned* ctrl, unsigned* word) {
  TOPX_CUDA_OK(cudaMemsetAsync(word, 0, sizeof(unsigned), st));
  (k_gf_wait_selftest<<<1, 32, 0, st>>>(ctrl, word), topx::count_launch());
  TOPX_CUDA_OK(cudaGetLastError());
}

void launch_gj_flow(cudaStream_t st, int m, int nset, double* A0, double* A1, const uint32_t* tasks,
                    unsigned ntasks, double* scratch, unsigned* ctrl, int nctas) {
  // the error word (ctrl[0]) is left alone: the host reads and clears it after the factorisation
  TOPX_CUDA_OK(cudaMemsetAsync(ctrl + GF_TICKET, 0, (gf_ctrl_words(m) - GF_TICKET) * sizeof(unsigned), st));
  GFArgs a;
  a.A[0] = A0;
  a.A[1] = nset > 1 ? A1 : A0;
  a.tasks = tasks;
  a.ntasks = ntasks;
  a.m = m;
  a.nt = gf_tiles(m);
  a.scr = scratch;
  a.ctrl = ctrl;
  const unsigned grid = std::max(1u, std::min(unsigned(nctas), ntasks));
  (k_gj_flow<<<grid, GF_THREADS, GF_SMEM, st>>>(a), topx::count_launch());
  TOPX_CUDA_OK(cudaGetLastError());
}

}  // namespace topx
