// Device side of the nested-dissection multifrontal factorisation and solve of the coarsest-
// level matrix (plan and storage in topx_nd.hpp).  Replaces the reference's sparse Cholesky
// with fill-reducing permutation (chol(K,'lower'), TOP3D_XL.m:1052-1065) and its triangular
// solves in the V-cycle (TOP3D_XL.m:767): the same exact solve, another elimination order.
//
// Factorisation, per tree level from the leaves up: extend-add of the children's Schur
// complements, then for k = 0 .. T1-1 three launches over all fronts of the level:
//   pivot   P^-1 of tile (k, k) (register-blocked Gauss-Jordan on the tensor cores), with the
//           write-back of the previous step's row and column;
//   panel   R_j = -P^-1 A[k][j] for every tile column j != k (into scratch);
//   update  A[i][j] += A[i][k] R_j for every stored tile (i >= j), i, j != k;
// and at the end of a step the new row k is R and the new column k is -R^T.  Only the lower
// triangle of tiles is stored: an upper tile is the transpose of its mirror, negated when
// exactly one of its two tile indices has already been swept.
// Solve, per level: up the tree f = b + children's updates, w1 = F11^-1 f1, u = f2 - X f1;
// down the tree x1 = w1 - X^T x2.  No kernel waits on another: launches order the steps.
#include <algorithm>
#include <mutex>

#include "topx_coop.cuh"
#include "topx_kernels.cuh"
#include "topx_nd.hpp"
#include "topx_nd_dev.hpp"
#include "topx_tile64.cuh"

namespace topx {

namespace {

constexpr int ND_TILE = ND_T * ND_T;
constexpr int ND_THREADS = GF_THREADS;  // 256
// two staging buffers per sweep CTA (three CTAs per SM)
constexpr size_t ND_SMEM_SWEEP = size_t(2) * GF_BUF * sizeof(double);
static_assert(ND_T == GF_T, "tile widths");

__device__ __forceinline__ int64_t nd_tri(int64_t i) { return i * (i + 1) / 2; }
__device__ __forceinline__ double* nd_tile(double* pool, const NDFront& d, int i, int j) {
  return pool + (d.tile0 + nd_tri(i) + j) * ND_TILE;
}
template <typename TM>
__device__ __forceinline__ const TM* nd_tile_c(const TM* pool, const NDFront& d, int i, int j) {
  return pool + (d.tile0 + nd_tri(i) + j) * ND_TILE;
}
// the stored element of the symmetric entry (p1, p2) of front d; also its mirror inside a
// diagonal tile (-1 when there is none)
__device__ __forceinline__ void nd_entry(const NDFront& d, int p1, int p2, int64_t& at, int64_t& mirror) {
  const int hi = max(p1, p2), lo = min(p1, p2);
  const int ti = hi / ND_T, tj = lo / ND_T;
  const int64_t base = (d.tile0 + nd_tri(ti) + tj) * ND_TILE;
  at = base + (hi % ND_T) * ND_T + lo % ND_T;
  mirror = (ti == tj && hi != lo) ? base + (lo % ND_T) * ND_T + hi % ND_T : -1;
}

// s[t][c] (row stride ld) = sgn * g[c][t] for a contiguous 64 x 64 tile g
__device__ __forceinline__ void nd_stage_transposed(double* s, const double* g, int ld, double sgn) {
#pragma unroll 4
  for (int e = threadIdx.x; e < ND_TILE; e += ND_THREADS) {
    const int c = e >> 6, t = e & 63;
    s[t * ld + c] = sgn * __ldcg(g + e);
  }
}

// ---------------------------------------------------------------------------
// assembly of the original matrix into the fronts (writes), and the padding identity
// ---------------------------------------------------------------------------
__global__ void k_nd_assemble(Grid g, const NDFront* __restrict__ fronts, const NDAsm* __restrict__ asmb, int64_t n,
                              const double* __restrict__ Ks, double* __restrict__ pool) {
  const int nny = g.ny + 1, nnx = g.nx + 1;
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < n; t += int64_t(gridDim.x) * blockDim.x) {
    const NDAsm e = asmb[t];
    const NDFront d = fronts[e.f];
    const int ay = e.a % nny, ax = (e.a / nny) % nnx, az = e.a / (nny * nnx);
    const int by = e.b % nny, bx = (e.b / nny) % nnx, bz = e.b / (nny * nnx);
    double blk[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int la = 0; la < 8; ++la) {  // the hexes around node a that also hold node b
      const int ey = ay - hex_ly(la), ex = ax - hex_lx(la), ez = az - hex_lz(la);
      if (ey < 0 || ey >= g.ny || ex < 0 || ex >= g.nx || ez < 0 || ez >= g.nz) continue;
      const int ly = by - ey, lx = bx - ex, lz = bz - ez;
      if (ly < 0 || ly > 1 || lx < 0 || lx > 1 || lz < 0 || lz > 1) continue;
      const int lb = hex_local(ly, lx, lz);
      const double* K = Ks + (ey + int64_t(g.ny) * (ex + int64_t(g.nx) * ez)) * 576;
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) blk[i * 3 + j] += K[(3 * la + i) * 24 + 3 * lb + j];
    }
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        int64_t at, mir;
        nd_entry(d, e.pa + i, e.pb + j, at, mir);
        pool[at] = blk[i * 3 + j];
        if (mir >= 0) pool[mir] = blk[i * 3 + j];
      }
  }
}

__global__ void k_nd_pad(const int64_t* __restrict__ at, int64_t n, double* __restrict__ pool) {
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < n; t += int64_t(gridDim.x) * blockDim.x)
    pool[at[t]] = 1.0;
}

// ---------------------------------------------------------------------------
// extend-add: child tile (i, j) of its update block into the parent front (adds; the map is
// one to one, so no two threads of a launch touch one entry)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(ND_THREADS) k_nd_extend(const NDFront* __restrict__ fronts,
                                                          const NDTask* __restrict__ tasks,
                                                          const int32_t* __restrict__ upd_map,
                                                          double* __restrict__ pool) {
  const NDTask tk = tasks[blockIdx.x];
  const NDFront c = fronts[tk.f];
  const NDFront d = fronts[c.parent];
  const double* src = nd_tile(pool, c, tk.i, tk.j);
  const int P1 = ND_T * c.T1;
  for (int e = threadIdx.x; e < ND_TILE; e += ND_THREADS) {
    const int r = e >> 6, cc = e & 63;
    const int k1 = ND_T * tk.i + r - P1, k2 = ND_T * tk.j + cc - P1;
    if (k1 >= c.n2 || k2 >= c.n2 || (tk.i == tk.j && r < cc)) continue;
    const double v = src[e];
    int64_t at, mir;
    nd_entry(d, upd_map[c.map0 + k1], upd_map[c.map0 + k2], at, mir);
    pool[at] += v;
    if (mir >= 0) pool[mir] += v;
  }
}

// ---------------------------------------------------------------------------
// sweep step k
// ---------------------------------------------------------------------------
// scratch slot of R_j of step k (R tiles alternate between two sets by the parity of k)
__device__ __forceinline__ double* nd_rslot(double* scr, const NDFront& d, int k, int j) {
  return scr + int64_t(d.scr0 + 1 + (k & 1) * d.N + j) * ND_TILE;
}

// write-back of step i for tile column j: row i takes R_j (j < i), column i takes -R_j^T (j > i)
__device__ __forceinline__ void nd_finalize_task(const NDFront& d, NDTask tk, double* pool, double* scr, double* s) {
  const double* R = nd_rslot(scr, d, tk.i, tk.j);
  if (tk.j < tk.i) {
    double* D = nd_tile(pool, d, tk.i, tk.j);
    for (int e = threadIdx.x; e < ND_TILE; e += ND_THREADS) D[e] = __ldcg(R + e);
  } else {
    double* D = nd_tile(pool, d, tk.j, tk.i);
    for (int e = threadIdx.x; e < ND_TILE; e += ND_THREADS) s[(e >> 6) * 65 + (e & 63)] = __ldcg(R + e);  // [64][65]
    __syncthreads();
    for (int e = threadIdx.x; e < ND_TILE; e += ND_THREADS) D[e] = -s[(e & 63) * 65 + (e >> 6)];
  }
}

// the inverse of the (symmetric positive definite) tile in acc, into scratch slot 0 and tile A
__device__ __forceinline__ void nd_pivot_acc(double (&acc)[4][2][2], double* A, double* scr, const NDFront& d,
                                             double* smem) {
  double* Pinv = scr + int64_t(d.scr0) * ND_TILE;
  gf_pivot(acc, nullptr, 0, 0, ND_T, Pinv, *reinterpret_cast<GFPivotSmem*>(smem));
  gf_for_outputs(acc, [&](int r, int c, double v) { A[r * ND_T + c] = v; });
}

// Blocks [0, npiv): pivot of step 0 of front f (tile (0, 0) <- its inverse, also into scratch
// slot 0).  Blocks [npiv, gridDim.x): write-back tasks (the last step of a level).
__global__ void __launch_bounds__(ND_THREADS) k_nd_pivot(const NDFront* __restrict__ fronts,
                                                         const NDTask* __restrict__ tasks, int npiv,
                                                         double* __restrict__ pool, double* __restrict__ scr) {
  extern __shared__ __align__(16) double nd_smem[];
  const NDTask tk = tasks[blockIdx.x];
  const NDFront d = fronts[tk.f];
  if (int(blockIdx.x) < npiv) {
    double* A = nd_tile(pool, d, tk.i, tk.i);
    double acc[4][2][2];
    gf_for_outputs(acc, [&](int r, int c, double& v) { v = __ldcg(A + r * ND_T + c); });
    nd_pivot_acc(acc, A, scr, d, nd_smem);
    return;
  }
  nd_finalize_task(d, tk, pool, scr, nd_smem);
}

// Blocks [0, npan): R_j = -P^-1 A[k][j] of step k into its scratch slot; A[k][k-1] is the column
// k-1 that step k-1's write-back (blocks [npan, gridDim.x) of the same launch) is storing, so it
// is taken from step k-1's R_k instead: -R_k^T.
__global__ void __launch_bounds__(ND_THREADS) k_nd_panel(const NDFront* __restrict__ fronts,
                                                         const NDTask* __restrict__ tasks, int npan, int k,
                                                         double* __restrict__ pool, double* __restrict__ scr) {
  extern __shared__ __align__(16) double nd_smem[];
  const NDTask tk = tasks[blockIdx.x];
  const NDFront d = fronts[tk.f];
  if (int(blockIdx.x) >= npan) {
    nd_finalize_task(d, tk, pool, scr, nd_smem);
    return;
  }
  double* bufA = nd_smem;
  double* bufB = nd_smem + GF_BUF;
  const double* Pinv = scr + int64_t(d.scr0) * ND_TILE;
  gf_stage_ring(bufA, Pinv, GF_LDA);
  if (tk.j == k - 1)
    nd_stage_transposed(bufB, nd_rslot(scr, d, k - 1, k), GF_LD, -1.0);
  else if (tk.j < k)
    gf_stage_ring(bufB, nd_tile_c(pool, d, k, tk.j), GF_LD);
  else
    nd_stage_transposed(bufB, nd_tile_c(pool, d, tk.j, k), GF_LD, 1.0);
  gf_cp_wait();
  __syncthreads();
  double acc[4][2][2];
  gf_for_outputs(acc, [&](int, int, double& v) { v = 0.0; });
  gf_product(bufA, bufB, acc);
  double* R = nd_rslot(scr, d, k, tk.j);
  gf_for_outputs(acc, [&](int r, int c, double v) { R[r * ND_T + c] = -v; });
}

// A[i][j] += A[i][k] R_j for a stored tile (i >= j); the CTA of tile (k+1, k+1) then inverts it,
// the pivot of step k+1
__global__ void __launch_bounds__(ND_THREADS) k_nd_update(const NDFront* __restrict__ fronts,
                                                          const NDTask* __restrict__ tasks, int k,
                                                          double* __restrict__ pool, double* __restrict__ scr) {
  extern __shared__ __align__(16) double nd_smem[];
  double* bufA = nd_smem;
  double* bufB = nd_smem + GF_BUF;
  const NDTask tk = tasks[blockIdx.x];
  const NDFront d = fronts[tk.f];
  if (tk.i > k)
    gf_stage_ring(bufA, nd_tile_c(pool, d, tk.i, k), GF_LDA);
  else  // tile column i is swept, k is not: A[i][k] = -A[k][i]^T
    nd_stage_transposed(bufA, nd_tile_c(pool, d, k, tk.i), GF_LDA, -1.0);
  gf_stage_ring(bufB, nd_rslot(scr, d, k, tk.j), GF_LD);
  double* D = nd_tile(pool, d, tk.i, tk.j);
  double acc[4][2][2];
  gf_load_acc(acc, D);  // the tile goes straight into the accumulators while the operands land
  gf_cp_wait();
  __syncthreads();
  gf_product(bufA, bufB, acc);
  if (tk.i == k + 1 && tk.j == k + 1 && k + 1 < d.T1) {
    __syncthreads();  // bufA becomes the pivot's workspace
    nd_pivot_acc(acc, D, scr, d, bufA);
    return;
  }
  gf_store_acc(D, acc);
}

// ---------------------------------------------------------------------------
// solve: GEMVs over whole tiles.  A warp streams a tile with coalesced 16-byte loads: lane
// (h, c) = (lane / 16, lane % 16) reads columns 4c .. 4c + 3 of rows 2 k + h.  Row sums
// (y = A x) are kept per row and reduced across the 16 lanes of a half by recursive halving,
// which leaves lane (h, c) the rows 4c + h and 4c + 2 + h; column sums (y = A^T x) are kept
// per column and the two halves added.  Either way a lane ends with outputs 4c + h, 4c + 2 + h.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void nd_load4(const double* p, double (&v)[4]) {
  const double2 a = __ldg(reinterpret_cast<const double2*>(p));
  const double2 b = __ldg(reinterpret_cast<const double2*>(p) + 1);
  v[0] = a.x;
  v[1] = a.y;
  v[2] = b.x;
  v[3] = b.y;
}
__device__ __forceinline__ void nd_load4(const float* p, double (&v)[4]) {
  const float4 a = __ldg(reinterpret_cast<const float4*>(p));
  v[0] = a.x;
  v[1] = a.y;
  v[2] = a.z;
  v[3] = a.w;
}

// acc[k] += tile row (2k + h) (of the 32 rows at t), columns 4c .. 4c + 3, times x[4c ..]
template <typename TM>
__device__ __forceinline__ void nd_rows(const TM* t, const double* x, int h, int c, double (&acc)[16]) {
  const double x0 = x[4 * c], x1 = x[4 * c + 1], x2 = x[4 * c + 2], x3 = x[4 * c + 3];
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    double v[4];
    nd_load4(t + (2 * k + h) * ND_T + 4 * c, v);
    acc[k] = fma(v[0], x0, fma(v[1], x1, fma(v[2], x2, fma(v[3], x3, acc[k]))));
  }
}
// col[e] += sum over the rows (2k + h) of the 32 rows at t of t[row][4c + e] x[row]
template <typename TM>
__device__ __forceinline__ void nd_cols(const TM* t, const double* x, int h, int c, double (&col)[4]) {
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    const int row = 2 * k + h;
    double v[4];
    nd_load4(t + row * ND_T + 4 * c, v);
    const double xr = x[row];
#pragma unroll
    for (int e = 0; e < 4; ++e) col[e] = fma(v[e], xr, col[e]);
  }
}
// recursive halving of 16 row sums over the 16 lanes of a half: lane c ends with the sum of
// local row k = c, i.e. row 2c + h of the 32 rows
__device__ __forceinline__ double nd_reduce_rows(double (&acc)[16], int c) {
#pragma unroll
  for (int o = 8, n = 16; o >= 1; o >>= 1, n >>= 1) {
    const bool up = (c & o) != 0;
#pragma unroll
    for (int t = 0; t < n / 2; ++t) {
      const double send = up ? acc[t] : acc[t + n / 2];
      const double keep = up ? acc[t + n / 2] : acc[t];
      acc[t] = keep + __shfl_xor_sync(0xffffffffu, send, o);
    }
  }
  return acc[0];
}

// One chunk (up to ND_CHUNK input tiles) of output tile i: warp w takes rows 32 (w & 1) .. + 31
// of input tile w >> 1 and leaves its part of the 64 outputs in red[w][].  Row sums (y = A x)
// give each lane the row 2c + h of its 32; column sums (y = A^T x) the columns 4c + h, 4c + 2 + h.
template <typename TM>
__device__ __forceinline__ void nd_chunk_rows(const TM* t, const double* x, double* redw, int rh, int h, int c) {
  double acc[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) acc[k] = 0.0;
  nd_rows(t + 32 * rh * ND_T, x, h, c, acc);
  redw[32 * rh + 2 * c + h] = nd_reduce_rows(acc, c);
}
template <typename TM>
__device__ __forceinline__ void nd_chunk_cols(const TM* t, const double* x, double* redw, int rh, int h, int c) {
  double col[4] = {0.0, 0.0, 0.0, 0.0};
  nd_cols(t + 32 * rh * ND_T, x + 32 * rh, h, c, col);
#pragma unroll
  for (int e = 0; e < 4; ++e) col[e] += __shfl_xor_sync(0xffffffffu, col[e], 16);
  redw[4 * c + h] = h ? col[1] : col[0];
  redw[4 * c + 2 + h] = h ? col[3] : col[2];
}

// The 64 sums of a chunk (threads < 64 hold them in s) complete output tile `id`: with one
// chunk the caller writes at once; else the chunk's partial goes to part[ti] (ti: the task's
// index in its launch or phase), and the last CTA of the output tile to finish (atomic ticket,
// no waiting) adds the chunks in order.  Returns true (with s the total) in the threads < 64 of
// the CTA that writes the output.
__device__ __forceinline__ unsigned nd_ticket(unsigned* p) {
  // release: the CTA's partial sums (ordered before by the barrier) are visible to whoever
  // acquires the count; acquire: so are the other chunks' partials to the last CTA
  unsigned v;
  asm volatile("atom.add.acq_rel.gpu.global.u32 %0, [%1], 1;" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ bool nd_finish(double& s, int64_t ti, int ch, int nch, unsigned* cnt, int64_t id,
                                          double* part, bool* last) {
  if (nch == 1) return threadIdx.x < ND_T;
  if (threadIdx.x < ND_T) part[ti * ND_T + threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x == 0) *last = nd_ticket(cnt + id) == unsigned(nch - 1);
  __syncthreads();
  if (!*last) return false;
  if (threadIdx.x == 0) cnt[id] = 0u;  // ready for the next launch
  if (threadIdx.x < ND_T) {
    double t = 0.0;
    for (int q = 0; q < nch; ++q) t += __ldcg(part + (ti - ch + q) * ND_T + threadIdx.x);
    s = t;
  }
  return threadIdx.x < ND_T;
}

__device__ __forceinline__ void nd_prefetch_l2(const char* p) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

static_assert(ND_CHUNK * ND_T <= ND_THREADS, "a solve task gathers one input entry per thread");
struct NDSolveSmem {
  double vec[ND_CHUNK * ND_T];  // the chunk's input entries
  double red[8][ND_T];
  bool last;
  int ok;  // dataflow launch: the task's inputs are complete (0: a wait gave up)
};

// Dataflow launch: per front, output tiles completed by its children on the way up, and output
// tiles of its own solution (zero between launches)
struct NDFlow {
  unsigned* fwd_done;
  unsigned* bwd_done;
  CoopControl* ctl;  // error word and exit count
};

template <typename T, typename TM>
struct NDSolveArgs {
  const NDFront* fronts;
  const NDTask* tasks;
  const TM* pool;
  const T* b;
  T* x;
  const int32_t *sep_dof, *upd_dof, *src0, *src1;
  double* w;
  double* part;
  unsigned* cnt;
};

// Forward task: one chunk of the eliminated tiles for output tile i of a front, per level up the
// tree.  i < T1: w = F11^-1 f1; i >= T1: w = f2 - X f1, where f1 is the eliminated part of the
// front's right-hand side (b at its DOFs plus what its children's updates put there) and f2
// what the children's updates put on the update DOFs.
template <typename T, typename TM, bool FLOW>
__device__ __forceinline__ bool nd_forward_task(const NDSolveArgs<T, TM>& a, const NDTask tk, int64_t ti,
                                                NDSolveSmem& sm, const NDFlow* fl) {
  const NDFront d = a.fronts[tk.f];
  const int i = tk.i, ch = tk.j;
  const int nch = max(1, (d.T1 + ND_CHUNK - 1) / ND_CHUNK);
  const int j0 = ch * ND_CHUNK, nj = min(ND_CHUNK, d.T1 - j0);
  // the chunk's tiles start on their way to L2 while the right-hand side is gathered
  for (int e = threadIdx.x; e < nj * (ND_TILE * int(sizeof(TM)) / 128); e += ND_THREADS) {
    const int t = e / (ND_TILE * int(sizeof(TM)) / 128), off = e % (ND_TILE * int(sizeof(TM)) / 128);
    const int j = j0 + t;
    const TM* tile = (i >= d.T1 || j <= i) ? nd_tile_c(a.pool, d, i, j) : nd_tile_c(a.pool, d, j, i);
    nd_prefetch_l2(reinterpret_cast<const char*>(tile) + 128 * off);
  }
  // Right-hand side at position p: b at its grid DOF (eliminated DOFs) plus the children's
  // update entries that land there.  The indices and b come before the wait, the children's
  // entries (written by other CTAs of the launch: loads bypass L1) after it.  Thread k gathers
  // input entry k of the chunk; threads < 64 also the entry at their output position.
  const bool has_in = threadIdx.x < nj * ND_T;
  const int64_t pin = d.pos0 + int64_t(ND_T) * j0 + threadIdx.x;
  const int64_t pout = d.pos0 + int64_t(ND_T) * i + threadIdx.x;
  int32_t s0 = -1, s1 = -1, o0 = -1, o1 = -1, og = -1;
  double v = 0.0, ov = 0.0;
  if (has_in) {
    const int32_t g = a.sep_dof[pin];
    s0 = a.src0[pin];
    s1 = a.src1[pin];
    if (g >= 0) v = double(a.b[g]);
  }
  if (threadIdx.x < ND_T) {
    og = a.sep_dof[pout];
    if (i >= d.T1) {  // an update position: no grid DOF of this front, so no b
      o0 = a.src0[pout];
      o1 = a.src1[pout];
    }
  }
  // dataflow: the children's update vectors (all their output tiles) are complete
  if (FLOW && threadIdx.x == 0)
    sm.ok = d.fwd_need == 0 || coop_wait_count(fl->fwd_done + tk.f, unsigned(d.fwd_need), fl->ctl);
  __syncthreads();  // the previous task's readers of sm are done
  if (FLOW && !sm.ok) return false;
  if (has_in) {
    if (s0 >= 0) v += __ldcg(a.w + s0);
    if (s1 >= 0) v += __ldcg(a.w + s1);
    sm.vec[threadIdx.x] = v;
  }
  if (o0 >= 0) ov += __ldcg(a.w + o0);
  if (o1 >= 0) ov += __ldcg(a.w + o1);
  for (int e = threadIdx.x; e < 8 * ND_T; e += ND_THREADS) sm.red[e >> 6][e & 63] = 0.0;
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, h = lane >> 4, c = lane & 15;
  const int ts = warp >> 1, rh = warp & 1;
  if (ts < nj) {
    const int j = j0 + ts;
    if (i >= d.T1 || j <= i)
      nd_chunk_rows(nd_tile_c(a.pool, d, i, j), sm.vec + ND_T * ts, sm.red[warp], rh, h, c);
    else  // F11^-1 (i, j) = (stored tile (j, i))^T
      nd_chunk_cols(nd_tile_c(a.pool, d, j, i), sm.vec + ND_T * ts, sm.red[warp], rh, h, c);
  }
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x < ND_T)
#pragma unroll
    for (int q = 0; q < 8; ++q) s += sm.red[q][threadIdx.x];
  if (nd_finish(s, ti, ch, nch, a.cnt, d.pos0 / ND_T + i, a.part, &sm.last)) {
    if (i >= d.T1)
      a.w[pout] = ov - s;
    else if (d.n2 > 0)
      a.w[pout] = s;
    else if (og >= 0)  // no update DOFs: x1 = F11^-1 f1 is the solution (no phase on the way down)
      a.x[og] = T(s);
  }
  if (FLOW && (nch == 1 || sm.last)) {  // this CTA wrote output tile i: count it (release)
    __syncthreads();
    if (threadIdx.x == 0) {
      if (d.parent >= 0) red_release_add(fl->fwd_done + d.parent, 1u);
      if (d.n2 == 0) red_release_add(fl->bwd_done + tk.f, 1u);
    }
  }
  return true;
}

// Backward task: one chunk of the update tiles for output tile i < T1 of a front, per level
// down the tree: x1 = w1 - X^T x2, with x2 gathered from the solution at the update DOFs
// (written by the ancestors' phases); x1 goes to the separator DOFs.
template <typename T, typename TM, bool FLOW>
__device__ __forceinline__ bool nd_backward_task(const NDSolveArgs<T, TM>& a, const NDTask tk, int64_t ti,
                                                 NDSolveSmem& sm, const NDFlow* fl) {
  const NDFront d = a.fronts[tk.f];
  const int i = tk.i, ch = tk.j, P1 = ND_T * d.T1;
  const int nch = max(1, (d.N - d.T1 + ND_CHUNK - 1) / ND_CHUNK);
  const int j0 = d.T1 + ch * ND_CHUNK, nj = min(ND_CHUNK, d.N - j0);
  for (int e = threadIdx.x; e < nj * (ND_TILE * int(sizeof(TM)) / 128); e += ND_THREADS) {
    const int t = e / (ND_TILE * int(sizeof(TM)) / 128), off = e % (ND_TILE * int(sizeof(TM)) / 128);
    nd_prefetch_l2(reinterpret_cast<const char*>(nd_tile_c(a.pool, d, j0 + t, i)) + 128 * off);
  }
  // thread k gathers the solution at update DOF k of the chunk (index before the wait, value
  // after it); threads < 64 also w1 at their output position, after the wait
  const int u = ND_T * (j0 - d.T1) + int(threadIdx.x);
  const bool has_in = threadIdx.x < nj * ND_T;
  const int64_t pout = d.pos0 + int64_t(ND_T) * i + threadIdx.x;
  const int32_t gi = has_in && u < d.n2 ? a.upd_dof[d.pos0 + P1 + u] : -1;
  const int32_t og = threadIdx.x < ND_T ? a.sep_dof[pout] : -1;
  // dataflow: the nearest eliminating ancestor's solution is complete (and with it every ancestor's)
  if (FLOW && threadIdx.x == 0)
    sm.ok = d.bwd_need == 0 || coop_wait_count(fl->bwd_done + d.bwd_front, unsigned(d.bwd_need), fl->ctl);
  __syncthreads();
  if (FLOW && !sm.ok) return false;
  if (has_in) sm.vec[threadIdx.x] = gi >= 0 ? double(__ldcg(a.x + gi)) : 0.0;
  const double wv = og >= 0 ? __ldcg(a.w + pout) : 0.0;
  for (int e = threadIdx.x; e < 8 * ND_T; e += ND_THREADS) sm.red[e >> 6][e & 63] = 0.0;
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, h = lane >> 4, c = lane & 15;
  const int ts = warp >> 1, rh = warp & 1;
  if (ts < nj) nd_chunk_cols(nd_tile_c(a.pool, d, j0 + ts, i), sm.vec + ND_T * ts, sm.red[warp], rh, h, c);
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x < ND_T)
#pragma unroll
    for (int q = 0; q < 8; ++q) s += sm.red[q][threadIdx.x];
  if (nd_finish(s, ti, ch, nch, a.cnt, d.pos0 / ND_T + i, a.part, &sm.last)) {
    if (og >= 0) a.x[og] = T(wv - s);
  }
  if (FLOW && (nch == 1 || sm.last)) {
    __syncthreads();
    if (threadIdx.x == 0) red_release_add(fl->bwd_done + tk.f, 1u);
  }
  return true;
}

// one launch per tree level and direction
template <typename T, typename TM, bool FWD>
__global__ void __launch_bounds__(ND_THREADS) k_nd_solve_level(NDSolveArgs<T, TM> a, const PcgScalars* sc) {
  if (sc && sc->done) return;
  __shared__ NDSolveSmem sm;
  if (FWD)
    nd_forward_task<T, TM, false>(a, a.tasks[blockIdx.x], blockIdx.x, sm, nullptr);
  else
    nd_backward_task<T, TM, false>(a, a.tasks[blockIdx.x], blockIdx.x, sm, nullptr);
}

// The whole solve as one dataflow launch (all CTAs resident): the tasks in dependency order
// (a.tasks: the forward tasks from the leaves up, the first nfwd, then the backward tasks from the
// root down), CTA b taking tasks b, b + grid, ...  A task waits only for the fronts it reads:
// a forward task for its children's update vectors, a backward task for its parent's solution.
// Every dependency points to an earlier task, and each CTA takes its tasks in order, so the
// earliest unfinished task always has its inputs and its CTA is running it: the launch cannot
// deadlock, and every wait is bounded all the same.
template <typename T, typename TM>
__global__ void __launch_bounds__(ND_THREADS) k_nd_solve_flow(NDSolveArgs<T, TM> a, int64_t nfwd, int64_t ntot,
                                                              NDFlow fl, int nfronts, const PcgScalars* sc) {
  if (sc && sc->done) return;  // the same for every CTA
  __shared__ NDSolveSmem sm;
  for (int64_t t = blockIdx.x; t < ntot; t += gridDim.x) {
    const bool ok = t < nfwd ? nd_forward_task<T, TM, true>(a, a.tasks[t], t, sm, &fl)
                             : nd_backward_task<T, TM, true>(a, a.tasks[t], t, sm, &fl);
    if (!ok) break;  // a wait gave up (ctl->err is set): the CTAs after it give up too
  }
  // the last CTA out zeroes the counters for the next launch (every other CTA is past its tasks)
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    sm.last = atomicAdd(&fl.ctl->exits, 1u) == gridDim.x - 1;
    __threadfence();
  }
  __syncthreads();
  if (sm.last) {
    for (int f = threadIdx.x; f < nfronts; f += ND_THREADS) {
      fl.fwd_done[f] = 0u;
      fl.bwd_done[f] = 0u;
    }
    if (threadIdx.x == 0) fl.ctl->exits = 0u;
  }
}

// one CTA waits for a counter that nothing raises
__global__ void k_coop_wait_selftest(CoopControl* ctl) {
  if (threadIdx.x == 0) coop_wait_count(&ctl->idle, 1u, ctl);
}

inline unsigned nd_grid(int64_t n, int threads) {
  return unsigned(std::max<int64_t>(1, std::min<int64_t>((n + threads - 1) / threads, 148 * 16)));
}

}  // namespace

void prepare_nd_kernels() {
  static std::mutex mu;
  static bool done[64] = {};
  int dev = 0;
  TOPX_CUDA_OK(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  if (dev >= 0 && dev < 64 && done[dev]) return;
  TOPX_CUDA_OK(cudaFuncSetAttribute(k_nd_pivot, cudaFuncAttributeMaxDynamicSharedMemorySize, int(ND_SMEM_SWEEP)));
  TOPX_CUDA_OK(cudaFuncSetAttribute(k_nd_panel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(ND_SMEM_SWEEP)));
  TOPX_CUDA_OK(cudaFuncSetAttribute(k_nd_update, cudaFuncAttributeMaxDynamicSharedMemorySize, int(ND_SMEM_SWEEP)));
  if (dev >= 0 && dev < 64) done[dev] = true;
}

void NDDevice::factor(cudaStream_t st, const NDPlan& P, Grid g, const double* Ks) const {
  TOPX_CUDA_OK(cudaMemsetAsync(pool, 0, sizeof(double) * size_t(P.ntiles) * ND_TILE, st));
  const int64_t na = int64_t(P.asmb.size()), np = int64_t(P.pad_diag.size());
  (k_nd_assemble<<<nd_grid(na, 256), 256, 0, st>>>(g, fronts, asmb, na, Ks, pool), topx::count_launch());
  if (np) (k_nd_pad<<<nd_grid(np, 256), 256, 0, st>>>(pad, np, pool), topx::count_launch());
  for (int l = int(P.levels.size()) - 1; l >= 0; --l) {
    const NDLevel& L = P.levels[size_t(l)];
    for (int s = 0; s < 2; ++s) {
      const int64_t n = L.ext[s + 1] - L.ext[s];
      if (n) (k_nd_extend<<<unsigned(n), ND_THREADS, 0, st>>>(fronts, tasks + L.ext[s], upd_map, pool), topx::count_launch());
    }
    const int64_t npiv0 = L.piv0[1] - L.piv0[0];
    if (npiv0)
      (k_nd_pivot<<<unsigned(npiv0), ND_THREADS, ND_SMEM_SWEEP, st>>>(fronts, tasks + L.piv0[0], int(npiv0), pool, scr),
       topx::count_launch());
    for (int k = 0; k < L.maxT1; ++k) {
      const int64_t* s = &L.step[size_t(4) * k];
      const int64_t npan = s[1] - s[0], nfin = s[2] - s[1], nupd = s[3] - s[2];
      if (npan + nfin)
        (k_nd_panel<<<unsigned(npan + nfin), ND_THREADS, ND_SMEM_SWEEP, st>>>(fronts, tasks + s[0], int(npan), k, pool,
                                                                             scr),
         topx::count_launch());
      if (nupd)
        (k_nd_update<<<unsigned(nupd), ND_THREADS, ND_SMEM_SWEEP, st>>>(fronts, tasks + s[2], k, pool, scr),
         topx::count_launch());
    }
    const int64_t nfin = L.fin_last[1] - L.fin_last[0];
    if (nfin)
      (k_nd_pivot<<<unsigned(nfin), ND_THREADS, ND_SMEM_SWEEP, st>>>(fronts, tasks + L.fin_last[0], 0, pool, scr),
       topx::count_launch());
  }
  TOPX_CUDA_OK(cudaGetLastError());
}

template <typename T, typename TM>
void NDDevice::solve(cudaStream_t st, const NDPlan& P, const TM* tiles, const T* b, T* x, const PcgScalars* sc) const {
  NDSolveArgs<T, TM> a{fronts, tasks, tiles, b, x, sep_dof, upd_dof, src0, src1, wvec, part, cnt};
  const int nlev = int(P.levels.size());
  if (coop_ctas > 0 && nlev > 0) {
    int64_t most = 1;
    for (const NDLevel& L : P.levels) most = std::max(most, std::max(L.fwd[1] - L.fwd[0], L.bwd[1] - L.bwd[0]));
    NDSolveArgs<T, TM> af = a;
    af.tasks = flow;
    NDFlow fl{flow_done, flow_done + P.fronts.size(), ctl};
    const int64_t ntot = int64_t(P.flow.size());
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(unsigned(std::min<int64_t>(coop_ctas, most)));
    cfg.blockDim = dim3(ND_THREADS);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    TOPX_CUDA_OK(cudaLaunchKernelEx(&cfg, k_nd_solve_flow<T, TM>, af, P.flow_fwd, ntot, fl, int(P.fronts.size()), sc));
    topx::count_launch();
    return;
  }
  for (int l = nlev - 1; l >= 0; --l) {
    const NDLevel& L = P.levels[size_t(l)];
    a.tasks = tasks + L.fwd[0];
    (k_nd_solve_level<T, TM, true><<<unsigned(L.fwd[1] - L.fwd[0]), ND_THREADS, 0, st>>>(a, sc), topx::count_launch());
  }
  for (int l = 0; l < nlev; ++l) {
    const NDLevel& L = P.levels[size_t(l)];
    a.tasks = tasks + L.bwd[0];
    if (L.bwd[1] > L.bwd[0])
      (k_nd_solve_level<T, TM, false><<<unsigned(L.bwd[1] - L.bwd[0]), ND_THREADS, 0, st>>>(a, sc), topx::count_launch());
  }
  TOPX_CUDA_OK(cudaGetLastError());
}

int nd_solve_coop_ctas() {
  int dev = 0, coop = 0, nsm = 0, per = 0, per32 = 0;
  TOPX_CUDA_OK(cudaGetDevice(&dev));
  TOPX_CUDA_OK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
  TOPX_CUDA_OK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  if (!coop) return 0;
  TOPX_CUDA_OK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_nd_solve_flow<double, double>, ND_THREADS, 0));
  TOPX_CUDA_OK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per32, k_nd_solve_flow<float, float>, ND_THREADS, 0));
  per = std::min(std::min(per, per32), 4);
  return per >= 1 ? nsm * per : 0;
}

void launch_coop_wait_selftest(cudaStream_t st, CoopControl* ctl) {
  (k_coop_wait_selftest<<<1, 32, 0, st>>>(ctl), topx::count_launch());
  TOPX_CUDA_OK(cudaGetLastError());
}

template void NDDevice::solve<double, double>(cudaStream_t, const NDPlan&, const double*, const double*, double*,
                                             const PcgScalars*) const;
template void NDDevice::solve<float, float>(cudaStream_t, const NDPlan&, const float*, const float*, float*,
                                           const PcgScalars*) const;

}  // namespace topx
