// 64 x 64 FP64 tile primitives on the tensor cores (mma.sync m8n8k4) shared by the coarsest-
// level factorisations: asynchronous tile staging, the tile product and the register-blocked
// Gauss-Jordan inversion of a 64 x 64 pivot tile.  One CTA of GF_THREADS threads works on a tile.
#pragma once

#include <cstdint>

namespace topx {

constexpr int GF_T = 64;  // tile width

constexpr int GF_THREADS = 256;
constexpr int GF_LD = GF_T + 8;   // row stride of B operands [t][c] in shared memory (doubles)
constexpr int GF_LDA = GF_T + 4;  // row stride of A operands [r][t] (row-major)
// both strides make a warp's fragment load exactly two shared-memory wavefronts
constexpr int GF_BUF = GF_T * GF_LD;  // doubles per staging buffer

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

// This thread's accumulators from / to a contiguous 64 x 64 tile in global memory (16-byte
// accesses; loads through L2 only, since earlier launches wrote the tile)
__device__ __forceinline__ void gf_load_acc(double (&acc)[4][2][2], const double* __restrict__ g) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, gi = lane >> 2, q = lane & 3;
  const int rb = (warp >> 2) * 32, cb = (warp & 3) * 16;
#pragma unroll
  for (int fr = 0; fr < 4; ++fr)
#pragma unroll
    for (int fc = 0; fc < 2; ++fc) {
      const double2 v = __ldcg(reinterpret_cast<const double2*>(g + (rb + 8 * fr + gi) * GF_T + cb + 8 * fc + 2 * q));
      acc[fr][fc][0] = v.x;
      acc[fr][fc][1] = v.y;
    }
}
__device__ __forceinline__ void gf_store_acc(double* __restrict__ g, const double (&acc)[4][2][2]) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, gi = lane >> 2, q = lane & 3;
  const int rb = (warp >> 2) * 32, cb = (warp & 3) * 16;
#pragma unroll
  for (int fr = 0; fr < 4; ++fr)
#pragma unroll
    for (int fc = 0; fc < 2; ++fc)
      *reinterpret_cast<double2*>(g + (rb + 8 * fr + gi) * GF_T + cb + 8 * fc + 2 * q) =
          make_double2(acc[fr][fc][0], acc[fr][fc][1]);
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
// acc: the tile (identity beyond kb) on entry, P^-1 on return (also stored to Pinv, and to the
// tile's place in M unless M is null).
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
        if (M && r < kb && c + h < kb) M[int64_t(k0 + r) * m + k0 + c + h] = acc[fr][fc][h];
    }
}

}  // namespace topx
