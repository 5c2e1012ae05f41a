// Coarse-level kernels of the TOP3D_XL B200 path (Solving_AssembleFEAstencil,
// TOP3D_XL.m:919-1066): Galerkin element operators per level, their Jacobi
// diagonals, and the FP64 coarsest-level direct solver.
//
// Coarsest solver: the coarsest node grid is split into slabs (one node layer
// each) along its longest axis, which makes K block tridiagonal; it is
// factorised from both ends toward the middle slab with explicit FP64 inverses
// of the diagonal Schur complements (see launch_slab_factor), so a coarse solve
// is ~ns dense GEMVs spread over all SMs.  This replaces the reference's sparse
// Cholesky with fill-reducing permutation (chol(K,'lower') with P,
// TOP3D_XL.m:1065): same exact solve, different rounding.
#include <algorithm>
#include <mutex>

#include "topx_kernels.cuh"

namespace topx {

static inline unsigned grid1d(int64_t n, int threads, int cap = 148 * 16) {
  int64_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > cap) b = cap;
  return unsigned(b);
}

// ---------------------------------------------------------------------------
// Level-2 Galerkin operators (TOP3D_XL.m:946-978): Ks2_j = sum_c E_c T_c over the
// 64 children of every dense level-2 element (void children have E = 0).
// ---------------------------------------------------------------------------
constexpr int GL2_ELEMS = 16, GL2_THREADS = 192;

__global__ void __launch_bounds__(GL2_THREADS) k_galerkin_l2(Grid gc, const double* __restrict__ Ef,
                                                             const double* __restrict__ Tm, double* __restrict__ Ks) {
  __shared__ double sE[GL2_ELEMS][64];
  const int64_t nce = gc.nelems();
  const int64_t j0 = int64_t(blockIdx.x) * GL2_ELEMS;
  const int fny = 4 * gc.ny, fnx = 4 * gc.nx;
  for (int i = threadIdx.x; i < GL2_ELEMS * 64; i += GL2_THREADS) {
    const int jj = i / 64, c = i % 64;
    const int64_t j = j0 + jj;
    double v = 0.0;
    if (j < nce) {
      const int gy = int(j % gc.ny), gx = int((j / gc.ny) % gc.nx), gz = int(j / (int64_t(gc.ny) * gc.nx));
      const int cy = c & 3, cx = (c >> 2) & 3, cz = c >> 4;
      v = Ef[(4 * gy + cy) + int64_t(fny) * ((4 * gx + cx) + int64_t(fnx) * (4 * gz + cz))];
    }
    sE[jj][c] = v;
  }
  __syncthreads();
  double acc[GL2_ELEMS][3];
#pragma unroll
  for (int jj = 0; jj < GL2_ELEMS; ++jj) acc[jj][0] = acc[jj][1] = acc[jj][2] = 0.0;
  const int k0 = threadIdx.x;
  for (int c = 0; c < 64; ++c) {
    const double t0 = __ldg(&Tm[c * 576 + k0]);
    const double t1 = __ldg(&Tm[c * 576 + k0 + GL2_THREADS]);
    const double t2 = __ldg(&Tm[c * 576 + k0 + 2 * GL2_THREADS]);
#pragma unroll
    for (int jj = 0; jj < GL2_ELEMS; ++jj) {
      const double e = sE[jj][c];
      acc[jj][0] = fma(e, t0, acc[jj][0]);
      acc[jj][1] = fma(e, t1, acc[jj][1]);
      acc[jj][2] = fma(e, t2, acc[jj][2]);
    }
  }
#pragma unroll
  for (int jj = 0; jj < GL2_ELEMS; ++jj) {
    const int64_t j = j0 + jj;
    if (j < nce) {
      Ks[j * 576 + k0] = acc[jj][0];
      Ks[j * 576 + k0 + GL2_THREADS] = acc[jj][1];
      Ks[j * 576 + k0 + 2 * GL2_THREADS] = acc[jj][2];
    }
  }
}

void launch_galerkin_l2(cudaStream_t st, Grid gc, const double* Efine, const double* Tm, double* Ks) {
  const int64_t nb = (gc.nelems() + GL2_ELEMS - 1) / GL2_ELEMS;
  (k_galerkin_l2<<<unsigned(nb), GL2_THREADS, 0, st>>>(gc, Efine, Tm, Ks), topx::count_launch());
  TOPX_CUDA_OK(cudaGetLastError());
}

// Level-2 elements holding children with fixed DOFs (TOP3D_XL.m:961-971):
// Ks2_j = sum_c E_c T_sel(j,c) + F_j, where T_sel is the child's template or the
// template of its BC-modified Ke (uniqueKesFree_), and F_j collects the
// E-independent uniqueKesFixed_ parts.
__global__ void __launch_bounds__(GL2_THREADS) k_galerkin_l2_flagged(Grid gc, const double* __restrict__ Ef,
                                                                     const int32_t* __restrict__ fl_elem,
                                                                     const int32_t* __restrict__ fl_tsel,
                                                                     const double* __restrict__ fl_F,
                                                                     const double* __restrict__ Tall,
                                                                     double* __restrict__ Ks) {
  __shared__ double sE[64];
  __shared__ int sT[64];
  const int f = blockIdx.x;
  const int64_t j = fl_elem[f];
  const int fny = 4 * gc.ny, fnx = 4 * gc.nx;
  const int gy = int(j % gc.ny), gx = int((j / gc.ny) % gc.nx), gz = int(j / (int64_t(gc.ny) * gc.nx));
  for (int c = threadIdx.x; c < 64; c += GL2_THREADS) {
    const int cy = c & 3, cx = (c >> 2) & 3, cz = c >> 4;
    sE[c] = Ef[(4 * gy + cy) + int64_t(fny) * ((4 * gx + cx) + int64_t(fnx) * (4 * gz + cz))];
    sT[c] = fl_tsel[f * 64 + c];
  }
  __syncthreads();
  for (int k = threadIdx.x; k < 576; k += GL2_THREADS) {
    double a = 0.0;
    for (int c = 0; c < 64; ++c) a = fma(sE[c], Tall[int64_t(sT[c]) * 576 + k], a);
    Ks[j * 576 + k] = a + fl_F[int64_t(f) * 576 + k];
  }
}

void launch_galerkin_l2_flagged(cudaStream_t st, Grid gc, const double* Efine, int nflag, const int32_t* fl_elem,
                                const int32_t* fl_tsel, const double* fl_F, const double* Tall, double* Ks) {
  if (nflag <= 0) return;
  (k_galerkin_l2_flagged<<<nflag, GL2_THREADS, 0, st>>>(gc, Efine, fl_elem, fl_tsel, fl_F, Tall, Ks), topx::count_launch());
  TOPX_CUDA_OK(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// Span-2 Galerkin operators of levels >= 3 (TOP3D_XL.m:979-995):
// Ks_J = sum_{c<8} P_c^T Ks_child(c) P_c.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_galerkin_span2(Grid gc, const double* __restrict__ Ksf,
                                                        const uint8_t* __restrict__ cpresent,
                                                        const double* __restrict__ P8, double* __restrict__ Ks) {
  __shared__ double sK[576], sP[576], sT[576];
  const int64_t J = blockIdx.x;
  const int tid = threadIdx.x;
  double acc[3] = {0.0, 0.0, 0.0};
  if (cpresent[J]) {
    const int gy = int(J % gc.ny), gx = int((J / gc.ny) % gc.nx), gz = int(J / (int64_t(gc.ny) * gc.nx));
    const int fny = 2 * gc.ny, fnx = 2 * gc.nx;
    for (int c = 0; c < 8; ++c) {
      const int cy = c & 1, cx = (c >> 1) & 1, cz = c >> 2;
      const int64_t f = (2 * gy + cy) + int64_t(fny) * ((2 * gx + cx) + int64_t(fnx) * (2 * gz + cz));
      for (int k = tid; k < 576; k += 256) {
        sK[k] = Ksf[f * 576 + k];
        sP[k] = P8[c * 576 + k];
      }
      __syncthreads();
      for (int k = tid; k < 576; k += 256) {
        const int i = k / 24, jj = k % 24;
        double s = 0.0;
        for (int q = 0; q < 24; ++q) s = fma(sK[i * 24 + q], sP[q * 24 + jj], s);
        sT[k] = s;
      }
      __syncthreads();
      int m = 0;
      for (int k = tid; k < 576; k += 256, ++m) {
        const int i = k / 24, jj = k % 24;
        double s = acc[m];
        for (int q = 0; q < 24; ++q) s = fma(sP[q * 24 + i], sT[q * 24 + jj], s);
        acc[m] = s;
      }
      __syncthreads();
    }
  }
  int m = 0;
  for (int k = tid; k < 576; k += 256, ++m) Ks[J * 576 + k] = acc[m];
}

void launch_galerkin_span2(cudaStream_t st, Grid gc, const double* Ksf, const uint8_t* cpresent, const double* P8,
                           double* Ks) {
  (k_galerkin_span2<<<unsigned(gc.nelems()), 256, 0, st>>>(gc, Ksf, cpresent, P8, Ks), topx::count_launch());
  TOPX_CUDA_OK(cudaGetLastError());
}

// Jacobi diagonal of a coarse level from its element operators (TOP3D_XL.m:1000-1018),
// stored as its reciprocal (0 on absent nodes) so the smoother multiplies
template <typename T>
__global__ void k_diag_coarse(Grid g, const double* __restrict__ Ks, const uint8_t* __restrict__ present,
                              T* __restrict__ d) {
  const int64_t N = g.nnodes();
  const int nny = g.ny + 1, nnx = g.nx + 1;
  for (int64_t n = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; n < N; n += int64_t(gridDim.x) * blockDim.x) {
    double s[3] = {0.0, 0.0, 0.0};
    if (present[n]) {
      const int gy = int(n % nny), gx = int((n / nny) % nnx), gz = int(n / (int64_t(nny) * nnx));
      for (int a = 0; a < 8; ++a) {
        const int ey = gy - hex_ly(a), ex = gx - hex_lx(a), ez = gz - hex_lz(a);
        if (ey < 0 || ey >= g.ny || ex < 0 || ex >= g.nx || ez < 0 || ez >= g.nz) continue;
        const int64_t e = ey + int64_t(g.ny) * (ex + int64_t(g.nx) * ez);
        for (int c = 0; c < 3; ++c) s[c] += Ks[e * 576 + (3 * a + c) * 25];
      }
      for (int c = 0; c < 3; ++c) s[c] = 1.0 / s[c];
    }
    for (int c = 0; c < 3; ++c) d[n + c * g.stride] = T(s[c]);
  }
}

template <typename T>
void launch_diag_coarse(cudaStream_t st, Grid g, const double* Ks, const uint8_t* present, T* d) {
  (k_diag_coarse<T><<<grid1d(g.nnodes(), 256), 256, 0, st>>>(g, Ks, present, d), topx::count_launch());
  TOPX_CUDA_OK(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// coarsest level: slab block-tridiagonal assembly
// ---------------------------------------------------------------------------
__host__ __device__ inline void slab_node(const Grid& g, const SlabInfo& si, int s, int u, int v, int& gy, int& gx,
                                          int& gz) {
  if (si.axis == 0) {
    gy = s;
    gx = u;
    gz = v;
  } else if (si.axis == 1) {
    gx = s;
    gy = u;
    gz = v;
  } else {
    gz = s;
    gy = u;
    gx = v;
  }
}

// one thread per (slab s, node a of the slab, neighbour (ds in {0,1}, du, dv))
__global__ void k_slab_assemble(Grid g, SlabInfo si, const double* __restrict__ Ks, const uint8_t* __restrict__ present,
                                double* __restrict__ A, double* __restrict__ Bup) {
  const int64_t per = int64_t(si.nu) * si.nv * 18;
  const int64_t N = per * si.ns;
  const int nny = g.ny + 1, nnx = g.nx + 1;
  const int64_t m = si.m;
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < N; t += int64_t(gridDim.x) * blockDim.x) {
    const int s = int(t / per);
    int64_t r = t % per;
    const int nbk = int(r % 18);
    const int a = int(r / 18);
    const int ua = a % si.nu, va = a / si.nu;
    const int ds = nbk / 9, du = (nbk % 9) % 3 - 1, dv = (nbk % 9) / 3 - 1;
    const int ub = ua + du, vb = va + dv, sb = s + ds;
    if (ub < 0 || ub >= si.nu || vb < 0 || vb >= si.nv || sb >= si.ns) continue;
    int ay, ax, az, by, bx, bz;
    slab_node(g, si, s, ua, va, ay, ax, az);
    slab_node(g, si, sb, ub, vb, by, bx, bz);
    double blk[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    const int64_t na = ay + int64_t(nny) * (ax + int64_t(nnx) * az);
    if (present[na]) {
      for (int la = 0; la < 8; ++la) {
        const int ey = ay - hex_ly(la), ex = ax - hex_lx(la), ez = az - hex_lz(la);
        if (ey < 0 || ey >= g.ny || ex < 0 || ex >= g.nx || ez < 0 || ez >= g.nz) continue;
        const int ly = by - ey, lx = bx - ex, lz = bz - ez;
        if (ly < 0 || ly > 1 || lx < 0 || lx > 1 || lz < 0 || lz > 1) continue;
        const int lb = hex_local(ly, lx, lz);
        const double* K = Ks + (ey + int64_t(g.ny) * (ex + int64_t(g.nx) * ez)) * 576;
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) blk[i * 3 + j] += K[(3 * la + i) * 24 + 3 * lb + j];
      }
    } else if (ds == 0 && du == 0 && dv == 0) {
      blk[0] = blk[4] = blk[8] = 1.0;  // absent node: identity row, zero right-hand side
    }
    if (ds == 0) {
      const int64_t ia = 3 * int64_t(a), ib = 3 * int64_t(ub + si.nu * vb);
      double* As = A + int64_t(s) * m * m;
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) As[(ia + i) * m + ib + j] = blk[i * 3 + j];
    } else {
      const int nbi = (du + 1) + 3 * (dv + 1);
      double* Bs = Bup + (int64_t(s) * si.nu * si.nv + a) * 81 + nbi * 9;
      for (int k = 0; k < 9; ++k) Bs[k] = blk[k];
    }
  }
}

void launch_slab_assemble(cudaStream_t st, Grid g, SlabInfo si, const double* Ks, const uint8_t* present, double* A,
                          double* Bup) {
  TOPX_CUDA_OK(cudaMemsetAsync(A, 0, sizeof(double) * size_t(si.m) * si.m * si.ns, st));
  const int64_t N = int64_t(si.nu) * si.nv * 18 * si.ns;
  (k_slab_assemble<<<grid1d(N, 256), 256, 0, st>>>(g, si, Ks, present, A, Bup), topx::count_launch());
  TOPX_CUDA_OK(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// Twisted ("from both ends") block LDL^T of the slab-tridiagonal coarsest matrix.
// Slabs 0..mid-1 are eliminated from the top, slabs ns-1..mid+1 from the bottom,
// and the middle slab last, so both chains run side by side in the same
// launches (grid dimension selects the chain) and the sequential depth halves.
//   top:    S_s = A_s - L_{s-1} B_{s-1},        L_s = B_s^T S_s^{-1}   (s < mid)
//   bottom: T_s = A_s - U_s B_s^T,              U_{s-1} = B_{s-1} T_s^{-1} (s > mid)
//   middle: M   = A_mid - L_{mid-1} B_{mid-1} - U_mid B_mid^T
// B_s couples slab s (rows) to slab s+1 (cols) and is kept as a 27-point
// stencil Bup[node of slab s][9 neighbours][3][3].  Every diagonal inverse is
// formed explicitly (blocked Gauss-Jordan exchange, FP64), so a solve is a
// short chain of dense GEMVs on all SMs.
// ---------------------------------------------------------------------------
// Y[r][:] = sum_t coef_t(r) src[idx_t(r)][:] over the 27-point coupling stencil B of the slab
// pair, for the rows r of one CTA: the rows' (coefficient, source row) lists are built once in
// shared memory and the columns are swept with coalesced loads.  Two stencil kinds:
//   kind 0: r = DOF (c, k) of the upper slab, terms a in the lower slab around c:
//           coef = B[a][(du+1) + 3 (dv+1)][i][k], source row 3a + i   ((du, dv) = c - a)
//   kind 1: r = DOF (c, k) of the lower slab, terms n in the upper slab around c:
//           coef = B[c][(du+1) + 3 (dv+1)][k][q], source row 3n + q   ((du, dv) = n - c)
// An op takes up to two terms (the middle slab's Schur complement), summed in one FMA chain in
// the order (dv, du, i) of each term, first term first.
struct RowCombOp {
  const double* src[2];  // m x m row-major sources (src[1] optional)
  const double* B[2];    // their stencils
  int kind[2];
  double* Y;
};
constexpr int RC_ROWS = 4, RC_THREADS = 256, RC_TERMS = 54;

__device__ int rc_terms(const SlabInfo& si, int kind, const double* B, const double* src, int r, double* coef,
                        const double** row) {
  const int m = si.m, c = r / 3, k = r - 3 * c, uc = c % si.nu, vc = c / si.nu;
  int n = 0;
  for (int dv = -1; dv <= 1; ++dv)
    for (int du = -1; du <= 1; ++du) {
      if (kind == 0) {
        const int ua = uc - du, va = vc - dv;
        if (ua < 0 || ua >= si.nu || va < 0 || va >= si.nv) continue;
        const int aa = ua + si.nu * va;
        const double* Bb = B + int64_t(aa) * 81 + ((du + 1) + 3 * (dv + 1)) * 9;
        for (int i = 0; i < 3; ++i) {
          coef[n] = Bb[i * 3 + k];
          row[n++] = src + (3 * int64_t(aa) + i) * m;
        }
      } else {
        const int un = uc + du, vn = vc + dv;
        if (un < 0 || un >= si.nu || vn < 0 || vn >= si.nv) continue;
        const int nn = un + si.nu * vn;
        const double* Bn = B + int64_t(c) * 81 + ((du + 1) + 3 * (dv + 1)) * 9;
        for (int q = 0; q < 3; ++q) {
          coef[n] = Bn[k * 3 + q];
          row[n++] = src + (3 * int64_t(nn) + q) * m;
        }
      }
    }
  return n;
}

__global__ void __launch_bounds__(RC_THREADS) k_rowcomb(SlabInfo si, RowCombOp op0, RowCombOp op1) {
  const RowCombOp op = blockIdx.y == 0 ? op0 : op1;
  const int m = si.m, r0 = blockIdx.x * RC_ROWS;
  __shared__ double scoef[RC_ROWS][RC_TERMS];
  __shared__ const double* srow[RC_ROWS][RC_TERMS];
  __shared__ int scnt[RC_ROWS];
  if (threadIdx.x < RC_ROWS) {
    const int r = r0 + threadIdx.x;
    int n = 0;
    if (r < m)
      for (int t = 0; t < 2; ++t)
        if (op.src[t]) n += rc_terms(si, op.kind[t], op.B[t], op.src[t], r, &scoef[threadIdx.x][n], &srow[threadIdx.x][n]);
    scnt[threadIdx.x] = n;
  }
  __syncthreads();
  for (int col = threadIdx.x; col < m; col += RC_THREADS)
    for (int rr = 0; rr < RC_ROWS; ++rr) {
      const int r = r0 + rr;
      if (r >= m) break;
      double acc = 0.0;
      const int n = scnt[rr];
      for (int t = 0; t < n; ++t) acc = fma(scoef[rr][t], srow[rr][t][col], acc);
      op.Y[int64_t(r) * m + col] = acc;
    }
}

// D[r][c] = (A ? A[r][c] : 0) - / + Y[c][r] over 32 x 32 tiles staged in shared memory
// (sub: D = A - Y^T for a Schur complement, Y null -> D = A; copy: D = Y^T)
struct TransOp {
  const double* A;
  const double* Y;
  double* D;
};
__global__ void __launch_bounds__(256) k_transpose_tiles(int m, TransOp op0, TransOp op1, int sub) {
  const TransOp op = blockIdx.z == 0 ? op0 : op1;
  __shared__ double t[32][33];
  const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  if (op.Y)
    for (int j = ty; j < 32; j += 8) {
      const int r = by + j, c = bx + tx;  // Y[r][c], r: rows of Y = columns of D
      t[j][tx] = (r < m && c < m) ? op.Y[int64_t(r) * m + c] : 0.0;
    }
  __syncthreads();
  for (int j = ty; j < 32; j += 8) {
    const int r = bx + j, c = by + tx;  // D[r][c] = ... Y[c][r] = t[tx][j]
    if (r >= m || c >= m) continue;
    const int64_t k = int64_t(r) * m + c;
    const double y = op.Y ? t[tx][j] : 0.0;
    op.D[k] = sub ? op.A[k] - y : y;
  }
}

// once per device and process: engines on several host threads share the attributes
void prepare_coarse_kernels() { prepare_gj_flow(); }

// Every Schur complement is inverted in place by the dataflow Gauss-Jordan kernel
// (topx_gjflow.cu), the top and bottom chains' matrices in the same launch.
void launch_slab_factor(cudaStream_t st, const GJFlow& gf, SlabInfo si, const double* A, const double* Bup,
                        double* Sinv, double* X, double* XT) {
  const int m = si.m, ns = si.ns, mid = ns / 2;
  const int64_t mm = int64_t(m) * m;
  const int64_t bs = int64_t(si.nu) * si.nv * 81;
  const unsigned nrc = unsigned((m + RC_ROWS - 1) / RC_ROWS), nt32 = unsigned((m + 31) / 32);
  auto invert = [&](int nset, double* A0, double* A1) {
    launch_gj_flow(st, m, nset, A0, A1, gf.tasks[nset - 1], gf.ntasks[nset - 1], gf.scratch, gf.ctrl, gf.nctas);
  };
  // S = A - Y^T with Y = (sum of the coupling terms)^T by rows (ops without a term copy A)
  auto schur = [&](int nset, const RowCombOp (&ro)[2], const TransOp (&to)[2]) {
    int nrow = 0;
    RowCombOp rc[2] = {};
    for (int i = 0; i < nset; ++i)
      if (ro[i].src[0]) rc[nrow++] = ro[i];
    if (nrow) (k_rowcomb<<<dim3(nrc, nrow), RC_THREADS, 0, st>>>(si, rc[0], rc[1]), topx::count_launch());
    (k_transpose_tiles<<<dim3(nt32, nt32, nset), 256, 0, st>>>(m, to[0], to[1], 1), topx::count_launch());
  };
  const int ntop = mid, nbot = ns - 1 - mid;
  for (int k = 0; k < std::max(ntop, nbot); ++k) {
    RowCombOp ro[2] = {}, fo[2] = {};
    TransOp to[2] = {}, ft[2] = {};
    double* inv[2] = {nullptr, nullptr};
    int nset = 0, nform = 0;
    if (k < ntop) {  // top slab k: S_k = A_k - L_{k-1} B_{k-1}
      const int s = k;
      double* Y = gf.ytmp + nset * mm;
      if (s) ro[nset] = RowCombOp{{XT + (s - 1) * mm, nullptr}, {Bup + (s - 1) * bs, nullptr}, {0, 0}, Y};
      to[nset] = TransOp{A + s * mm, s ? Y : nullptr, Sinv + s * mm};
      inv[nset++] = Sinv + s * mm;
    }
    if (k < nbot) {  // bottom slab s = ns-1-k: T_s = A_s - U_s B_s^T
      const int s = ns - 1 - k;
      double* Y = gf.ytmp + nset * mm;
      if (k) ro[nset] = RowCombOp{{XT + s * mm, nullptr}, {Bup + s * bs, nullptr}, {1, 0}, Y};
      to[nset] = TransOp{A + s * mm, k ? Y : nullptr, Sinv + s * mm};
      inv[nset++] = Sinv + s * mm;
    }
    schur(nset, ro, to);
    invert(nset, inv[0], inv[1]);
    if (k < ntop) {  // L_k = B_k^T S_k^{-1}
      fo[nform] = RowCombOp{{Sinv + k * mm, nullptr}, {Bup + k * bs, nullptr}, {0, 0}, X + k * mm};
      ft[nform++] = TransOp{nullptr, X + k * mm, XT + k * mm};
    }
    if (k < nbot) {  // U_{s-1} = B_{s-1} T_s^{-1}, s = ns-1-k
      const int s = ns - 1 - k;
      fo[nform] = RowCombOp{{Sinv + s * mm, nullptr}, {Bup + (s - 1) * bs, nullptr}, {1, 0}, X + (s - 1) * mm};
      ft[nform++] = TransOp{nullptr, X + (s - 1) * mm, XT + (s - 1) * mm};
    }
    if (nform) {
      (k_rowcomb<<<dim3(nrc, nform), RC_THREADS, 0, st>>>(si, fo[0], fo[1]), topx::count_launch());
      (k_transpose_tiles<<<dim3(nt32, nt32, nform), 256, 0, st>>>(m, ft[0], ft[1], 0), topx::count_launch());
    }
  }
  // middle slab: M = A_mid - L_{mid-1} B_{mid-1} - U_mid B_mid^T (top term first)
  {
    RowCombOp ro[2] = {};
    TransOp to[2] = {};
    const bool up = mid > 0, dn = mid < ns - 1;
    if (up || dn) {
      ro[0].Y = gf.ytmp;
      int t = 0;
      if (up) {
        ro[0].src[t] = XT + (mid - 1) * mm;
        ro[0].B[t] = Bup + (mid - 1) * bs;
        ro[0].kind[t++] = 0;
      }
      if (dn) {
        ro[0].src[t] = XT + mid * mm;
        ro[0].B[t] = Bup + mid * bs;
        ro[0].kind[t++] = 1;
      }
    }
    to[0] = TransOp{A + mid * mm, (up || dn) ? gf.ytmp : nullptr, Sinv + mid * mm};
    schur(1, ro, to);
  }
  invert(1, Sinv + mid * mm, nullptr);
  TOPX_CUDA_OK(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// coarse solve x = K^{-1} b with the twisted slab factorization (TOP3D_XL.m:767)
//   forward:  W_0 = b_0,  W_{s+1} = b_{s+1} - L_s W_s            (s+1 < mid)
//             W_{ns-1} = b_{ns-1},  W_s = b_s - U_s W_{s+1}      (s > mid)
//             W_mid = b_mid - L_{mid-1} W_{mid-1} - U_mid W_{mid+1}
//   all s:    V_s = Inv_s W_s                                     (one batched launch)
//   backward: x_mid = V_mid,  x_s = V_s - L_s^T x_{s+1} (s < mid),  x_s = V_s - U_{s-1}^T x_{s-1} (s > mid)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_slab_gather(Grid g, SlabInfo si, const T* __restrict__ b, double* __restrict__ bs,
                              const PcgScalars* sc) {
  if (sc && sc->done) return;
  const int64_t N = int64_t(si.ns) * si.m;
  const int nny = g.ny + 1, nnx = g.nx + 1;
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < N; t += int64_t(gridDim.x) * blockDim.x) {
    const int s = int(t / si.m), row = int(t % si.m);
    const int c = row / 3, k = row % 3;
    int gy, gx, gz;
    slab_node(g, si, s, c % si.nu, c / si.nu, gy, gx, gz);
    bs[t] = double(b[gy + int64_t(nny) * (gx + int64_t(nnx) * gz) + k * g.stride]);
  }
}

template <typename T>
__global__ void k_slab_scatter(Grid g, SlabInfo si, const double* __restrict__ xs, T* __restrict__ x,
                               const PcgScalars* sc) {
  if (sc && sc->done) return;
  const int64_t N = int64_t(si.ns) * si.m;
  const int nny = g.ny + 1, nnx = g.nx + 1;
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < N; t += int64_t(gridDim.x) * blockDim.x) {
    const int s = int(t / si.m), row = int(t % si.m);
    const int c = row / 3, k = row % 3;
    int gy, gx, gz;
    slab_node(g, si, s, c % si.nu, c / si.nu, gy, gx, gz);
    x[gy + int64_t(nny) * (gx + int64_t(nnx) * gz) + k * g.stride] = T(xs[t]);
  }
}

// y = a - M1 u1 - M2 u2 (M2 optional; a optional: y = M1 u1) over `nmat` stacked m x m blocks
// (u, a, y stacked alike).  Two rows per CTA, four warps per row, four independent
// accumulators per lane; grid y selects one of two independent operations.
struct GemvOp {
  const void* M1;
  const double* u1;
  const void* M2;
  const double* u2;
  const double* a;
  double* y;
  int nmat;
};

template <typename TM>
__device__ __forceinline__ double row_dot(const TM* __restrict__ Mr, const double* __restrict__ u, int j0, int j1,
                                          int lane) {
  double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
  int jj = j0 + lane;
  for (; jj + 96 < j1; jj += 128) {
    a0 = fma(double(Mr[jj]), u[jj], a0);
    a1 = fma(double(Mr[jj + 32]), u[jj + 32], a1);
    a2 = fma(double(Mr[jj + 64]), u[jj + 64], a2);
    a3 = fma(double(Mr[jj + 96]), u[jj + 96], a3);
  }
  for (; jj < j1; jj += 32) a0 = fma(double(Mr[jj]), u[jj], a0);
  return (a0 + a1) + (a2 + a3);
}

template <typename TM>
__global__ void __launch_bounds__(256) k_slab_gemv(int m, GemvOp op0, GemvOp op1, const PcgScalars* sc) {
  if (sc && sc->done) return;
  const GemvOp op = blockIdx.y == 0 ? op0 : op1;
  __shared__ double part[2][4];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int rsub = warp >> 2, q = warp & 3;
  const int64_t rows = int64_t(m) * op.nmat;
  const int chunk = (m + 3) / 4;
  const int j0 = q * chunk, j1 = min(m, (q + 1) * chunk);
  for (int64_t r0 = int64_t(blockIdx.x) * 2; r0 < rows; r0 += int64_t(gridDim.x) * 2) {
    const int64_t r = r0 + rsub;
    double acc = 0.0;
    if (r < rows) {
      const int64_t blk = r / m;
      acc = row_dot<TM>(static_cast<const TM*>(op.M1) + r * m, op.u1 + blk * m, j0, j1, lane);
      if (op.M2) acc += row_dot<TM>(static_cast<const TM*>(op.M2) + r * m, op.u2 + blk * m, j0, j1, lane);
    }
    acc = warp_sum(acc);
    if (lane == 0) part[rsub][q] = acc;
    __syncthreads();
    if (threadIdx.x < 2) {
      const int64_t rr = r0 + threadIdx.x;
      if (rr < rows) {
        const double sum =
            (part[threadIdx.x][0] + part[threadIdx.x][1]) + (part[threadIdx.x][2] + part[threadIdx.x][3]);
        op.y[rr] = op.a ? op.a[rr] - sum : sum;
      }
    }
    __syncthreads();
  }
}

template <typename T, typename TM>
void launch_slab_solve(cudaStream_t st, Grid g, SlabInfo si, const TM* Inv, const TM* X, const TM* XT,
                       const T* b, double* bs, double* W, double* V, double* xs, T* x, const PcgScalars* sc) {
  const int m = si.m, ns = si.ns, mid = ns / 2;
  const int64_t mm = int64_t(m) * m;
  const int64_t N = int64_t(ns) * m;
  const int ntop = mid, nbot = ns - 1 - mid;
  const unsigned nb1 = unsigned((m + 1) / 2);
  (k_slab_gather<T><<<grid1d(N, 256), 256, 0, st>>>(g, si, b, bs, sc), topx::count_launch());
  // chain heads
  if (ntop > 0) TOPX_CUDA_OK(cudaMemcpyAsync(W, bs, sizeof(double) * m, cudaMemcpyDeviceToDevice, st));
  if (nbot > 0)
    TOPX_CUDA_OK(cudaMemcpyAsync(W + int64_t(ns - 1) * m, bs + int64_t(ns - 1) * m, sizeof(double) * m,
                                 cudaMemcpyDeviceToDevice, st));
  // forward chains toward the middle
  for (int k = 0; k + 1 < std::max(ntop, nbot); ++k) {
    GemvOp ops[2] = {};
    int n = 0;
    if (k + 1 < ntop)
      ops[n++] = GemvOp{X + k * mm, W + int64_t(k) * m, nullptr, nullptr, bs + int64_t(k + 1) * m,
                        W + int64_t(k + 1) * m, 1};
    if (k + 1 < nbot) {
      const int s = ns - 2 - k;  // W_s = b_s - U_s W_{s+1}
      ops[n++] = GemvOp{X + s * mm, W + int64_t(s + 1) * m, nullptr, nullptr, bs + int64_t(s) * m,
                        W + int64_t(s) * m, 1};
    }
    (k_slab_gemv<TM><<<dim3(nb1, n), 256, 0, st>>>(m, ops[0], ops[1], sc), topx::count_launch());
  }
  {  // middle
    GemvOp op{nullptr, nullptr, nullptr, nullptr, bs + int64_t(mid) * m, W + int64_t(mid) * m, 1};
    if (ntop > 0) {
      op.M1 = X + (mid - 1) * mm;
      op.u1 = W + int64_t(mid - 1) * m;
    }
    if (nbot > 0) {
      if (op.M1) {
        op.M2 = X + mid * mm;
        op.u2 = W + int64_t(mid + 1) * m;
      } else {
        op.M1 = X + mid * mm;
        op.u1 = W + int64_t(mid + 1) * m;
      }
    }
    if (op.M1)
      (k_slab_gemv<TM><<<dim3(nb1, 1), 256, 0, st>>>(m, op, op, sc), topx::count_launch());
    else
      TOPX_CUDA_OK(cudaMemcpyAsync(W + int64_t(mid) * m, bs + int64_t(mid) * m, sizeof(double) * m,
                                   cudaMemcpyDeviceToDevice, st));
  }
  GemvOp ov{Inv, W, nullptr, nullptr, nullptr, V, ns};
  (k_slab_gemv<TM><<<dim3(grid1d(N / 2 + 1, 1, 148 * 32), 1), 256, 0, st>>>(m, ov, ov, sc), topx::count_launch());
  TOPX_CUDA_OK(cudaMemcpyAsync(xs + int64_t(mid) * m, V + int64_t(mid) * m, sizeof(double) * m,
                               cudaMemcpyDeviceToDevice, st));
  // backward chains outward from the middle
  for (int k = 0; k < std::max(ntop, nbot); ++k) {
    GemvOp ops[2] = {};
    int n = 0;
    if (k < ntop) {
      const int s = mid - 1 - k;  // x_s = V_s - L_s^T x_{s+1}
      ops[n++] = GemvOp{XT + s * mm, xs + int64_t(s + 1) * m, nullptr, nullptr, V + int64_t(s) * m,
                        xs + int64_t(s) * m, 1};
    }
    if (k < nbot) {
      const int s = mid + 1 + k;  // x_s = V_s - U_{s-1}^T x_{s-1}
      ops[n++] = GemvOp{XT + (s - 1) * mm, xs + int64_t(s - 1) * m, nullptr, nullptr, V + int64_t(s) * m,
                        xs + int64_t(s) * m, 1};
    }
    (k_slab_gemv<TM><<<dim3(nb1, n), 256, 0, st>>>(m, ops[0], ops[1], sc), topx::count_launch());
  }
  (k_slab_scatter<T><<<grid1d(N, 256), 256, 0, st>>>(g, si, xs, x, sc), topx::count_launch());
  TOPX_CUDA_OK(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// The same coarse solve as one cooperative launch, one CTA per SM.  After the gather there is
// one grid-wide barrier; from then on every vector of the solve (W, V and x in slab order)
// starts out "absent" (a signalling-NaN bit pattern, which no arithmetic result can equal) and
// each chain step polls the entries it reads until their producers' values replace it.  A step
// so waits only for its own inputs, at the cost of one L2 round trip, instead of a grid
// barrier followed by a reload; each warp loads its matrix row into registers before it polls.
// ---------------------------------------------------------------------------
constexpr int COOP_THREADS = 512;
constexpr int COOP_WARPS = COOP_THREADS / 32;
// polls of the barrier word, and of a solve vector (each after a ~64 ns sleep), before a CTA
// gives up (well under a second in all)
constexpr unsigned kCoopSpinLimit = 1u << 20;
constexpr unsigned kFlowSpinLimit = 1u << 20;
constexpr unsigned long long kAbsent = 0x7FF4DEADBEEF0001ull;
static_assert(kCoopErrBarrier != 0 && kCoopErrVector != 0 && kCoopErrBarrier != kCoopErrVector, "error codes");

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ int ld_volatile_int(const int* p) { return *reinterpret_cast<const volatile int*>(p); }
__device__ __forceinline__ double ld_relaxed_f64(const double* p) {
  double v;
  asm volatile("ld.relaxed.gpu.global.f64 %0, [%1];" : "=d"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_f64(double* p, double v) {
  asm volatile("st.relaxed.gpu.global.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}
__device__ __forceinline__ bool coop_has(double v) {
  return static_cast<unsigned long long>(__double_as_longlong(v)) != kAbsent;
}

// Grid-wide barrier with a bounded wait.  bar->count only grows within a launch: barrier
// number i (1, 2, ...) is passed once it reaches i * gridDim.x, so an arrival is one
// fire-and-forget release add and the wait polls that single word (no reset round trip).
// The last CTA to leave the kernel (coop_exit) zeroes the words for the next launch.
// Returns false in every thread of the CTA once any CTA has given up (bar->err set); the
// kernel then returns, so it always ends.
__device__ bool coop_barrier(CoopBarrier* bar, unsigned& epoch) {
  __shared__ int s_ok;
  __syncthreads();
  ++epoch;
  if (threadIdx.x == 0) {
    int ok = ld_volatile_int(&bar->err) == 0;
    if (ok) {
      const unsigned target = epoch * gridDim.x;
      asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(&bar->count) : "memory");
      unsigned it = 0;
      while (ld_acquire_gpu(&bar->count) < target) {
        if (++it > kCoopSpinLimit || ld_volatile_int(&bar->err)) {
          atomicCAS(&bar->err, 0, kCoopErrBarrier);
          ok = 0;
          break;
        }
      }
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// Called once by every CTA on every exit path after its first barrier: the last one out
// re-arms the barrier words (all other CTAs have left their waits by then).
__device__ void coop_exit(CoopBarrier* bar) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(&bar->gen, 1u) == gridDim.x - 1) {
      atomicExch(&bar->count, 0u);
      atomicExch(&bar->gen, 0u);
    }
  }
}

// su[j] = g0[j] (j < m) and g1[j - m] (m <= j < n), in the factors' type, once every one of them
// is present; called by the whole CTA.  False (in every thread) once this CTA or another one
// gave up.
template <typename TS>
__device__ bool coop_wait_vector(TS* su, const double* g0, const double* g1, int m, int n, CoopBarrier* bar) {
  for (unsigned it = 0;; ++it) {
    bool ok = true;
    for (int j = threadIdx.x; j < n; j += COOP_THREADS) {
      const double v = ld_relaxed_f64(j < m ? g0 + j : g1 + (j - m));
      su[j] = TS(v);
      ok = ok && coop_has(v);
    }
    if (__syncthreads_and(ok)) return true;
    const int bad = threadIdx.x == 0 && (it >= kFlowSpinLimit || ld_volatile_int(&bar->err));
    if (__syncthreads_or(bad)) {
      if (threadIdx.x == 0) atomicCAS(&bar->err, 0, kCoopErrVector);
      return false;
    }
    __nanosleep(64);
  }
}

// one entry, polled by one thread (0.0 once the wait gave up; the error word is then set)
__device__ double coop_wait_value(const double* p, CoopBarrier* bar) {
  for (unsigned it = 0;; ++it) {
    const double v = ld_relaxed_f64(p);
    if (coop_has(v)) return v;
    if (it >= kFlowSpinLimit || ld_volatile_int(&bar->err)) {
      atomicCAS(&bar->err, 0, kCoopErrVector);
      return 0.0;
    }
    __nanosleep(64);
  }
}

// Per-lane partial dot products (two accumulators).  FP64 factors accumulate in FP64.  FP32
// factors multiply and add in FP32 over runs of a few terms, each run then added in FP64: no
// per-term widening, and the FP32 rounding stays that of short sums whatever m is.
template <typename TM>
struct LaneDot;
template <>
struct LaneDot<double> {
  double a0 = 0.0, a1 = 0.0;
  __device__ __forceinline__ void add0(double v, double u) { a0 = fma(v, u, a0); }
  __device__ __forceinline__ void add1(double v, double u) { a1 = fma(v, u, a1); }
  __device__ __forceinline__ void flush() {}
  __device__ __forceinline__ double total() const { return a0 + a1; }
};
template <>
struct LaneDot<float> {
  float f0 = 0.f, f1 = 0.f;
  double a0 = 0.0, a1 = 0.0;
  __device__ __forceinline__ void add0(float v, float u) { f0 = fmaf(v, u, f0); }
  __device__ __forceinline__ void add1(float v, float u) { f1 = fmaf(v, u, f1); }
  __device__ __forceinline__ void flush() {
    a0 += double(f0);
    a1 += double(f1);
    f0 = f1 = 0.f;
  }
  __device__ __forceinline__ double total() const { return (a0 + double(f0)) + (a1 + double(f1)); }
};
constexpr int kDotRun = 4;  // FP32 terms per accumulator between FP64 flushes

// Dot of one matrix row with a shared-memory vector by one warp.  The row is read in
// pieces of 32 x 32 elements whose loads are all issued before the first use, so a row
// of up to 1024 entries costs one memory round trip.  The warp sum is FP64.
template <typename TM>
__device__ __forceinline__ double warp_row_dot(const TM* __restrict__ Mr, const TM* __restrict__ u, int m, int lane) {
  constexpr int PIECE = 32;
  LaneDot<TM> acc;
  for (int base = 0; base < m; base += 32 * PIECE) {
    TM v[PIECE];
#pragma unroll
    for (int i = 0; i < PIECE; ++i) {
      const int j = base + lane + 32 * i;
      v[i] = j < m ? __ldg(Mr + j) : TM(0);
    }
#pragma unroll
    for (int i = 0; i < PIECE; i += 2) {
      const int j = base + lane + 32 * i;
      if (j < m) acc.add0(v[i], u[j]);
      if (j + 32 < m) acc.add1(v[i + 1], u[j + 32]);
      if ((i / 2) % kDotRun == kDotRun - 1) acc.flush();
    }
  }
  return warp_sum(acc.total());
}

// One chain step: up to two independent row blocks y = a - M u (M: m x m).
struct ChainOp {
  const void* M;
  const double* u;
  const double* a;
  double* y;
};

// The warp's first row (up to 1024 entries) is loaded into registers before the step's input
// vectors are polled into su, so the two memory round trips overlap; results are stored as
// strong (relaxed) writes, which the next step's pollers observe.  a_polled: the a vector
// is itself produced during the launch (V in the backward chains).
// (op[0] / op[1] picked by value so the descriptors stay in registers)
template <typename TM>
__device__ __forceinline__ bool chain_step(const ChainOp (&op)[2], int nop, int m, TM* su, int gw, int nw,
                                           int lane, bool a_polled, CoopBarrier* bar) {
  constexpr int PIECE = 32;
  TM v[PIECE];
  const int r0 = gw;
  const bool have = r0 < nop * m;
  const int o0 = r0 >= m ? 1 : 0;
  const ChainOp c0 = o0 ? op[1] : op[0];
  const TM* M0 = static_cast<const TM*>(c0.M) + int64_t(r0 - o0 * m) * m;
#pragma unroll
  for (int i = 0; i < PIECE; ++i) {
    const int j = lane + 32 * i;
    v[i] = (have && j < m) ? __ldg(M0 + j) : TM(0);
  }
  // the first row's a entry too: it does not depend on this step's inputs
  double a_first = 0.0;
  if (have && lane == 0) {
    const double* pa = c0.a + (r0 - o0 * m);
    a_first = a_polled ? coop_wait_value(pa, bar) : __ldcg(pa);
  }
  if (!coop_wait_vector(su, op[0].u, nop > 1 ? op[1].u : op[0].u, m, nop * m, bar)) return false;
  auto finish = [&](const ChainOp& c, int rr, double d) {
    if (lane == 0) {
      const double a = a_polled ? coop_wait_value(c.a + rr, bar) : __ldcg(c.a + rr);
      st_relaxed_f64(c.y + rr, a - d);
    }
  };
  if (have) {
    const TM* u = su + o0 * m;
    LaneDot<TM> acc;
#pragma unroll
    for (int i = 0; i < PIECE; i += 2) {
      const int j = lane + 32 * i;
      if (j < m) acc.add0(v[i], u[j]);
      if (j + 32 < m) acc.add1(v[i + 1], u[j + 32]);
      if ((i / 2) % kDotRun == kDotRun - 1) acc.flush();
    }
    int run = 0;
    for (int base = 32 * PIECE; base < m; base += 32) {
      const int j = base + lane;
      if (j < m) acc.add0(__ldg(M0 + j), u[j]);
      if (++run == kDotRun) {
        acc.flush();
        run = 0;
      }
    }
    const double d = warp_sum(acc.total());
    if (lane == 0) st_relaxed_f64(c0.y + (r0 - o0 * m), a_first - d);
  }
  for (int r = gw + nw; r < nop * m; r += nw) {
    const int o = r >= m ? 1 : 0, rr = r - o * m;
    const ChainOp c = o ? op[1] : op[0];
    finish(c, rr, warp_row_dot(static_cast<const TM*>(c.M) + int64_t(rr) * m, su + o * m, m, lane));
  }
  return true;
}

// forward step k: top W_{k+1} = bs_{k+1} - L_k W_k; bottom W_s = bs_s - U_s W_{s+1}, s = ns-2-k
template <typename TM>
__device__ __forceinline__ int forward_ops(int k, const SlabInfo& si, const TM* X, const double* bs, double* W,
                                           ChainOp (&op)[2]) {
  const int m = si.m, ns = si.ns, mid = ns / 2, ntop = mid, nbot = ns - 1 - mid;
  const int64_t mm = int64_t(m) * m;
  int n = 0;
  if (k + 1 < ntop) {
    op[0] = ChainOp{X + k * mm, W + int64_t(k) * m, bs + int64_t(k + 1) * m, W + int64_t(k + 1) * m};
    n = 1;
  }
  if (k + 1 < nbot) {
    const int s = ns - 2 - k;
    const ChainOp c{X + s * mm, W + int64_t(s + 1) * m, bs + int64_t(s) * m, W + int64_t(s) * m};
    if (n)
      op[1] = c;
    else
      op[0] = c;
    ++n;
  }
  return n;
}

// backward step k: top x_s = V_s - L_s^T x_{s+1}, s = mid-1-k; bottom x_s = V_s - U_{s-1}^T x_{s-1}, s = mid+1+k
template <typename TM>
__device__ __forceinline__ int backward_ops(int k, const SlabInfo& si, const TM* XT, const double* V, double* xs,
                                            ChainOp (&op)[2]) {
  const int m = si.m, ns = si.ns, mid = ns / 2, ntop = mid, nbot = ns - 1 - mid;
  const int64_t mm = int64_t(m) * m;
  int n = 0;
  if (k < ntop) {
    const int s = mid - 1 - k;
    op[0] = ChainOp{XT + s * mm, xs + int64_t(s + 1) * m, V + int64_t(s) * m, xs + int64_t(s) * m};
    n = 1;
  }
  if (k < nbot) {
    const int s = mid + 1 + k;
    const ChainOp c{XT + (s - 1) * mm, xs + int64_t(s - 1) * m, V + int64_t(s) * m, xs + int64_t(s) * m};
    if (n)
      op[1] = c;
    else
      op[0] = c;
    ++n;
  }
  return n;
}

template <typename T, typename TM>
__global__ void __launch_bounds__(COOP_THREADS, 1)
    k_slab_solve_coop(Grid g, SlabInfo si, const TM* __restrict__ Inv, const TM* __restrict__ X,
                      const TM* __restrict__ XT, const T* __restrict__ b, double* bs, double* W, double* V,
                      double* xs, T* __restrict__ x, const PcgScalars* sc, CoopBarrier* bar) {
  if (sc && sc->done) return;
  extern __shared__ double su_dyn[];  // two buffers of 2 m entries, alternating by step
  TM* const su_all = reinterpret_cast<TM*>(su_dyn);
  const int m = si.m, ns = si.ns, mid = ns / 2, ntop = mid, nbot = ns - 1 - mid;
  const int nsteps = max(ntop, nbot);
  const int64_t mm = int64_t(m) * m, N = int64_t(ns) * m;
  const int nny = g.ny + 1, nnx = g.nx + 1;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gw = blockIdx.x * COOP_WARPS + warp, nw = gridDim.x * COOP_WARPS;
  const int64_t tid = int64_t(blockIdx.x) * COOP_THREADS + threadIdx.x, nth = int64_t(gridDim.x) * COOP_THREADS;
  const double absent = __longlong_as_double(static_cast<long long>(kAbsent));
  int sbuf = 0;
  auto next_su = [&]() {
    TM* p = su_all + sbuf * 2 * m;
    sbuf ^= 1;
    return p;
  };
  ChainOp op[2];
  unsigned epoch = 0;

  // gather into slab order (chain heads and a lone middle slab take b directly); every other
  // entry of the solve vectors starts absent
  for (int64_t t = tid; t < N; t += nth) {
    const int s = int(t / m), row = int(t - int64_t(s) * m);
    const int c = row / 3, k = row - 3 * c;
    int gy, gx, gz;
    slab_node(g, si, s, c % si.nu, c / si.nu, gy, gx, gz);
    const double v = double(b[gy + int64_t(nny) * (gx + int64_t(nnx) * gz) + k * g.stride]);
    bs[t] = v;
    const bool head = (s == 0 && ntop > 0) || (s == ns - 1 && nbot > 0) || (ntop == 0 && nbot == 0);
    W[t] = head ? v : absent;
    V[t] = absent;
    xs[t] = absent;
  }
  if (!coop_barrier(bar, epoch)) {
    coop_exit(bar);
    return;
  }

  // forward chains toward the middle
  for (int k = 0; k + 1 < nsteps; ++k) {
    const int nop = forward_ops(k, si, X, bs, W, op);
    if (!chain_step<TM>(op, nop, m, next_su(), gw, nw, lane, false, bar)) {
      coop_exit(bar);
      return;
    }
  }
  // middle slab: W_mid = b_mid - L_{mid-1} W_{mid-1} - U_mid W_{mid+1}
  if (ntop > 0 || nbot > 0) {
    const ChainOp up{X + (mid - 1) * mm, W + int64_t(mid - 1) * m, nullptr, nullptr};
    const ChainOp dn{X + mid * mm, W + int64_t(mid + 1) * m, nullptr, nullptr};
    const int nop = (ntop > 0) + (nbot > 0);
    op[0] = ntop > 0 ? up : dn;
    op[1] = dn;
    TM* su = next_su();
    if (!coop_wait_vector(su, op[0].u, op[1].u, m, nop * m, bar)) {
      coop_exit(bar);
      return;
    }
    for (int r = gw; r < m; r += nw) {
      double d = warp_row_dot(static_cast<const TM*>(op[0].M) + int64_t(r) * m, su, m, lane);
      if (nop > 1) d += warp_row_dot(static_cast<const TM*>(op[1].M) + int64_t(r) * m, su + m, m, lane);
      if (lane == 0) st_relaxed_f64(W + int64_t(mid) * m + r, __ldcg(bs + int64_t(mid) * m + r) - d);
    }
  }
  // V_s = Inv_s W_s for all slabs, each CTA over a contiguous row range; x_mid = V_mid
  {
    const int64_t r0 = N * blockIdx.x / gridDim.x, r1 = N * (blockIdx.x + 1) / gridDim.x;
    for (int64_t rs = r0; rs < r1;) {
      const int s = int(rs / m);
      const int64_t re = min(r1, int64_t(s + 1) * m);
      TM* su = next_su();
      if (!coop_wait_vector(su, W + int64_t(s) * m, W + int64_t(s) * m, m, m, bar)) {
        coop_exit(bar);
        return;
      }
      for (int64_t r = rs + warp; r < re; r += COOP_WARPS) {
        const int rr = int(r - int64_t(s) * m);
        const double d = warp_row_dot(Inv + s * mm + int64_t(rr) * m, su, m, lane);
        if (lane == 0) {
          st_relaxed_f64(V + r, d);
          if (s == mid) st_relaxed_f64(xs + r, d);
        }
      }
      rs = re;
    }
  }
  // backward chains outward from the middle
  for (int k = 0; k < nsteps; ++k) {
    const int nop = backward_ops(k, si, XT, V, xs, op);
    if (!chain_step<TM>(op, nop, m, next_su(), gw, nw, lane, true, bar)) {
      coop_exit(bar);
      return;
    }
  }
  // scatter to the grid
  for (int64_t t = tid; t < N; t += nth) {
    const int s = int(t / m), row = int(t - int64_t(s) * m);
    const int c = row / 3, k = row - 3 * c;
    int gy, gx, gz;
    slab_node(g, si, s, c % si.nu, c / si.nu, gy, gx, gz);
    x[gy + int64_t(nny) * (gx + int64_t(nnx) * gz) + k * g.stride] = T(coop_wait_value(xs + t, bar));
  }
  coop_exit(bar);
}

int slab_solve_coop_ctas(int m) {
  int dev = 0, coop = 0, nsm = 0, per = 0;
  TOPX_CUDA_OK(cudaGetDevice(&dev));
  TOPX_CUDA_OK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
  TOPX_CUDA_OK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  if (!coop) return 0;
  const size_t smem = size_t(4) * m * sizeof(double);
  if (smem > size_t(200) * 1024) return 0;
  const void* kernels[2] = {reinterpret_cast<const void*>(&k_slab_solve_coop<double, double>),
                            reinterpret_cast<const void*>(&k_slab_solve_coop<float, float>)};
  for (int i = 0; i < 2; ++i) {
    TOPX_CUDA_OK(cudaFuncSetAttribute(kernels[i], cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    int b = 0;
    TOPX_CUDA_OK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernels[i], COOP_THREADS, smem));
    per = i == 0 ? b : std::min(per, b);
  }
  return per >= 1 ? nsm : 0;
}

template <typename T, typename TM>
void launch_slab_solve_coop(cudaStream_t st, int nctas, Grid g, SlabInfo si, const TM* Inv, const TM* X,
                            const TM* XT, const T* b, double* bs, double* W, double* V, double* xs, T* x,
                            const PcgScalars* sc, CoopBarrier* bar) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(unsigned(nctas));
  cfg.blockDim = dim3(COOP_THREADS);
  cfg.dynamicSmemBytes = size_t(4) * si.m * sizeof(double);
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  TOPX_CUDA_OK(cudaLaunchKernelEx(&cfg, k_slab_solve_coop<T, TM>, g, si, Inv, X, XT, b, bs, W, V, xs, x, sc, bar));
  topx::count_launch();
}

template void launch_slab_solve_coop<double, double>(cudaStream_t, int, Grid, SlabInfo, const double*, const double*,
                                                     const double*, const double*, double*, double*, double*,
                                                     double*, double*, const PcgScalars*, CoopBarrier*);
template void launch_slab_solve_coop<float, float>(cudaStream_t, int, Grid, SlabInfo, const float*, const float*,
                                                   const float*, const float*, double*, double*, double*, double*,
                                                   float*, const PcgScalars*, CoopBarrier*);

// ---------------------------------------------------------------------------
// Self-test of the bounded waits above: each case runs one wait primitive against a word that
// nothing writes, so the wait must give up after its poll limit, set the error word and return.
//  0: grid barrier of a two-CTA grid whose second CTA leaves without arriving;
//  1: coop_wait_value on an entry left absent;
//  2: coop_wait_vector on 64 entries left absent.
// `absent` holds at least 64 doubles.  The launch ends within the poll limits (about a second).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(COOP_THREADS) k_coop_wait_selftest(int which, CoopBarrier* bar, double* absent) {
  __shared__ double su[64];
  for (int j = threadIdx.x; j < 64; j += COOP_THREADS)
    reinterpret_cast<unsigned long long*>(absent)[j] = kAbsent;  // this CTA's own stores: seen below
  __syncthreads();
  if (which == 0) {
    if (blockIdx.x != 0) return;  // never arrives
    unsigned epoch = 0;
    coop_barrier(bar, epoch);
  } else if (which == 1) {
    if (threadIdx.x == 0) absent[64] = coop_wait_value(absent, bar);
  } else {
    coop_wait_vector<double>(su, absent, absent, 64, 64, bar);
  }
}

void launch_coop_wait_selftest(cudaStream_t st, int which, CoopBarrier* bar, double* absent) {
  const unsigned grid = which == 0 ? 2u : 1u;
  (k_coop_wait_selftest<<<grid, COOP_THREADS, 0, st>>>(which, bar, absent), topx::count_launch());
  TOPX_CUDA_OK(cudaGetLastError());
}

template void launch_diag_coarse<double>(cudaStream_t, Grid, const double*, const uint8_t*, double*);
template void launch_diag_coarse<float>(cudaStream_t, Grid, const double*, const uint8_t*, float*);
template void launch_slab_solve<double, double>(cudaStream_t, Grid, SlabInfo, const double*, const double*,
                                                const double*, const double*, double*, double*, double*, double*,
                                                double*, const PcgScalars*);
template void launch_slab_solve<float, float>(cudaStream_t, Grid, SlabInfo, const float*, const float*, const float*,
                                              const float*, double*, double*, double*, double*, float*,
                                              const PcgScalars*);

}  // namespace topx
