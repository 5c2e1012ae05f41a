// Coarse-level kernels of the TOP3D_XL B200 path (Solving_AssembleFEAstencil,
// TOP3D_XL.m:919-1066): Galerkin element operators per level, their Jacobi
// diagonals, and the FP64 coarsest-level direct solver.
//
// Coarsest solver: the coarsest node grid is split into slabs (one node layer
// each) along its longest axis, which makes K block tridiagonal:
//     K = L D L^T,  D_s = S_s = A_s - B_{s-1}^T S_{s-1}^{-1} B_{s-1}
// Each S_s^{-1} is formed explicitly (blocked Gauss-Jordan exchange, FP64), so
// a coarse solve is 2*ns dense GEMVs that spread over all SMs.  This replaces
// the reference's sparse Cholesky with fill-reducing permutation (chol(K,'lower')
// with P, TOP3D_XL.m:1065): same exact solve, different rounding.
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
  k_galerkin_l2<<<unsigned(nb), GL2_THREADS, 0, st>>>(gc, Efine, Tm, Ks);
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
  k_galerkin_l2_flagged<<<nflag, GL2_THREADS, 0, st>>>(gc, Efine, fl_elem, fl_tsel, fl_F, Tall, Ks);
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
  k_galerkin_span2<<<unsigned(gc.nelems()), 256, 0, st>>>(gc, Ksf, cpresent, P8, Ks);
  TOPX_CUDA_OK(cudaGetLastError());
}

// Jacobi diagonal of a coarse level from its element operators (TOP3D_XL.m:1000-1018)
template <typename T>
__global__ void k_diag_coarse(Grid g, const double* __restrict__ Ks, const uint8_t* __restrict__ present,
                              T* __restrict__ d) {
  const int64_t N = g.nnodes();
  const int nny = g.ny + 1, nnx = g.nx + 1;
  for (int64_t n = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; n < N; n += int64_t(gridDim.x) * blockDim.x) {
    double s[3] = {1.0, 1.0, 1.0};
    if (present[n]) {
      s[0] = s[1] = s[2] = 0.0;
      const int gy = int(n % nny), gx = int((n / nny) % nnx), gz = int(n / (int64_t(nny) * nnx));
      for (int a = 0; a < 8; ++a) {
        const int ey = gy - hex_ly(a), ex = gx - hex_lx(a), ez = gz - hex_lz(a);
        if (ey < 0 || ey >= g.ny || ex < 0 || ex >= g.nx || ez < 0 || ez >= g.nz) continue;
        const int64_t e = ey + int64_t(g.ny) * (ex + int64_t(g.nx) * ez);
        for (int c = 0; c < 3; ++c) s[c] += Ks[e * 576 + (3 * a + c) * 25];
      }
    }
    for (int c = 0; c < 3; ++c) d[n + c * g.stride] = T(s[c]);
  }
}

template <typename T>
void launch_diag_coarse(cudaStream_t st, Grid g, const double* Ks, const uint8_t* present, T* d) {
  k_diag_coarse<T><<<grid1d(g.nnodes(), 256), 256, 0, st>>>(g, Ks, present, d);
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
  k_slab_assemble<<<grid1d(N, 256), 256, 0, st>>>(g, si, Ks, present, A, Bup);
  TOPX_CUDA_OK(cudaGetLastError());
}

// T = S_{s-1}^{-1} B_{s-1}   (m x m, B given as the stencil Bup[node a of slab s-1][9 nbrs][3][3])
__global__ void k_schur_T(SlabInfo si, const double* __restrict__ Sinv, const double* __restrict__ Bp,
                          double* __restrict__ T) {
  const int64_t m = si.m;
  const int64_t N = m * m;
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < N; t += int64_t(gridDim.x) * blockDim.x) {
    const int64_t row = t / m, col = t % m;
    const int b = int(col / 3), j = int(col % 3);
    const int ub = b % si.nu, vb = b / si.nu;
    double s = 0.0;
    for (int dv = -1; dv <= 1; ++dv)
      for (int du = -1; du <= 1; ++du) {
        const int ua = ub - du, va = vb - dv;  // a + (du,dv) = b
        if (ua < 0 || ua >= si.nu || va < 0 || va >= si.nv) continue;
        const int a = ua + si.nu * va;
        const double* Bb = Bp + (int64_t(a) * 81) + ((du + 1) + 3 * (dv + 1)) * 9;
        for (int i = 0; i < 3; ++i) s = fma(Sinv[row * m + 3 * a + i], Bb[i * 3 + j], s);
      }
    T[t] = s;
  }
}

// S = A_s - B^T T
__global__ void k_schur_S(SlabInfo si, const double* __restrict__ Bp, const double* __restrict__ T,
                          const double* __restrict__ As, double* __restrict__ S) {
  const int64_t m = si.m;
  const int64_t N = m * m;
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < N; t += int64_t(gridDim.x) * blockDim.x) {
    const int64_t row = t / m, col = t % m;
    const int c = int(row / 3), k = int(row % 3);
    const int uc = c % si.nu, vc = c / si.nu;
    double s = 0.0;
    for (int dv = -1; dv <= 1; ++dv)
      for (int du = -1; du <= 1; ++du) {
        const int ua = uc - du, va = vc - dv;
        if (ua < 0 || ua >= si.nu || va < 0 || va >= si.nv) continue;
        const int a = ua + si.nu * va;
        const double* Bb = Bp + (int64_t(a) * 81) + ((du + 1) + 3 * (dv + 1)) * 9;
        for (int i = 0; i < 3; ++i) s = fma(Bb[i * 3 + k], T[(3 * int64_t(a) + i) * m + col], s);
      }
    S[t] = As[t] - s;
  }
}

void launch_slab_schur(cudaStream_t st, SlabInfo si, int s, const double* Sinv_prev, const double* Bup_prev,
                       const double* A_s, double* T, double* S_out) {
  const int64_t N = int64_t(si.m) * si.m;
  if (s == 0) {
    TOPX_CUDA_OK(cudaMemcpyAsync(S_out, A_s, sizeof(double) * size_t(N), cudaMemcpyDeviceToDevice, st));
    return;
  }
  k_schur_T<<<grid1d(N, 256), 256, 0, st>>>(si, Sinv_prev, Bup_prev, T);
  k_schur_S<<<grid1d(N, 256), 256, 0, st>>>(si, Bup_prev, T, A_s, S_out);
  TOPX_CUDA_OK(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// SPD inverse in place by blocked Gauss-Jordan exchange (pivot blocks of 32).
// One exchange step on pivot block K:  [P B; C D] -> [P^-1, -P^-1 B; C P^-1, D - C P^-1 B]
// After all blocks the matrix holds its inverse.  No pivoting is needed for SPD.
// ---------------------------------------------------------------------------
constexpr int GJB = 32;

__global__ void __launch_bounds__(256) k_gj_panel(int m, int k0, int kb, double* __restrict__ A,
                                                  double* __restrict__ Pinv, double* __restrict__ R,
                                                  double* __restrict__ C) {
  __shared__ double M[GJB][GJB + 1];
  __shared__ double col[GJB], row[GJB];
  const int tid = threadIdx.x;
  for (int i = tid; i < GJB * GJB; i += 256) {
    const int r = i / GJB, c = i % GJB;
    M[r][c] = (r < kb && c < kb) ? A[int64_t(k0 + r) * m + k0 + c] : (r == c ? 1.0 : 0.0);
  }
  __syncthreads();
  for (int t = 0; t < kb; ++t) {
    const double piv = M[t][t];
    if (tid < GJB) {
      col[tid] = M[tid][t];
      row[tid] = M[t][tid];
    }
    __syncthreads();
    for (int i = tid; i < GJB * GJB; i += 256) {
      const int r = i / GJB, c = i % GJB;
      double v;
      if (r == t && c == t)
        v = 1.0 / piv;
      else if (r == t)
        v = -row[c] / piv;
      else if (c == t)
        v = col[r] / piv;
      else
        v = M[r][c] - col[r] * row[c] / piv;
      M[r][c] = v;
    }
    __syncthreads();
  }
  if (blockIdx.x == 0)
    for (int i = tid; i < GJB * GJB; i += 256) Pinv[i] = M[i / GJB][i % GJB];
  // this CTA's columns: row panel R[:, j] = -P^-1 A[K, j]; old column panel C[j, :] = A[j, K]
  const int j = blockIdx.x * 256 + tid;
  if (j < m && (j < k0 || j >= k0 + kb)) {
    double a[GJB];
#pragma unroll
    for (int t = 0; t < GJB; ++t) a[t] = t < kb ? A[int64_t(k0 + t) * m + j] : 0.0;
    for (int r = 0; r < kb; ++r) {
      double s = 0.0;
#pragma unroll
      for (int t = 0; t < GJB; ++t) s = fma(M[r][t], a[t], s);
      R[int64_t(r) * m + j] = -s;
    }
    for (int t = 0; t < kb; ++t) C[int64_t(j) * GJB + t] = A[int64_t(j) * m + k0 + t];
  }
}

__global__ void __launch_bounds__(256) k_gj_update(int m, int k0, int kb, double* __restrict__ A,
                                                   const double* __restrict__ Pinv, const double* __restrict__ R,
                                                   const double* __restrict__ C) {
  __shared__ double sC[GJB][GJB + 1];  // rows i0..i0+31 of C (or Pinv rows), GJB cols
  __shared__ double sR[GJB][GJB + 1];  // GJB rows of R for cols j0..j0+31
  const int i0 = blockIdx.y * GJB, j0 = blockIdx.x * GJB;
  const int tid = threadIdx.x;
  const bool jK = (j0 == k0);  // column tiles are aligned to the pivot blocks
  const bool iK = (i0 == k0);
  for (int q = tid; q < GJB * GJB; q += 256) {
    const int r = q / GJB, c = q % GJB;
    const int i = i0 + r, j = j0 + c;
    sC[r][c] = (i < m && c < kb) ? (iK ? 0.0 : C[int64_t(i) * GJB + c]) : 0.0;
    if (jK)
      sR[r][c] = (r < kb && c < kb) ? Pinv[r * GJB + c] : 0.0;
    else
      sR[r][c] = (r < kb && j < m) ? R[int64_t(r) * m + j] : 0.0;
  }
  __syncthreads();
  for (int q = tid; q < GJB * GJB; q += 256) {
    const int r = q / GJB, c = q % GJB;
    const int i = i0 + r, j = j0 + c;
    if (i >= m || j >= m) continue;
    double v;
    if (iK && jK) {
      v = Pinv[r * GJB + c];
    } else if (iK) {
      v = sR[r][c];
    } else {
      double s = 0.0;
#pragma unroll 8
      for (int t = 0; t < GJB; ++t) s = fma(sC[r][t], sR[t][c], s);
      v = jK ? s : A[int64_t(i) * m + j] + s;
    }
    A[int64_t(i) * m + j] = v;
  }
}

void launch_spd_inverse(cudaStream_t st, int m, double* A, double* Pinv, double* R, double* C) {
  const unsigned nt = (m + GJB - 1) / GJB;
  for (int k0 = 0; k0 < m; k0 += GJB) {
    const int kb = (m - k0) < GJB ? (m - k0) : GJB;
    k_gj_panel<<<(m + 255) / 256, 256, 0, st>>>(m, k0, kb, A, Pinv, R, C);
    k_gj_update<<<dim3(nt, nt), 256, 0, st>>>(m, k0, kb, A, Pinv, R, C);
  }
  TOPX_CUDA_OK(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// coarse solve x = K^{-1} b with the slab LDL^T (TOP3D_XL.m:767)
//   forward:  w_s = b_s - B_{s-1}^T v_{s-1},  v_s = S_s^{-1} w_s
//   backward: x_s = S_s^{-1} (w_s - B_s x_{s+1})
// One launch per slab step; each CTA forms the full right-hand side in shared
// memory and computes a block of rows (one warp per row).
// ---------------------------------------------------------------------------
constexpr int SLAB_MAXM = 4096;

template <typename T>
__global__ void __launch_bounds__(256) k_slab_step(Grid g, SlabInfo si, int s, int fwd,
                                                    const double* __restrict__ Sinv, const double* __restrict__ Bup,
                                                    const T* __restrict__ b, double* __restrict__ w,
                                                    double* __restrict__ v, double* __restrict__ xs, T* __restrict__ x,
                                                    const PcgScalars* sc) {
  if (sc && sc->done) return;
  extern __shared__ double rhs[];
  const int m = si.m;
  const int nny = g.ny + 1, nnx = g.nx + 1;
  const int tid = threadIdx.x;
  for (int row = tid; row < m; row += 256) {
    const int c = row / 3, k = row % 3;
    const int uc = c % si.nu, vc = c / si.nu;
    double val;
    if (fwd) {
      int gy, gx, gz;
      slab_node(g, si, s, uc, vc, gy, gx, gz);
      val = double(b[gy + int64_t(nny) * (gx + int64_t(nnx) * gz) + k * g.stride]);
      if (s > 0) {  // - B_{s-1}^T v_{s-1}
        const double* Bp = Bup + int64_t(s - 1) * si.nu * si.nv * 81;
        const double* vp = v + int64_t(s - 1) * m;
        for (int dv = -1; dv <= 1; ++dv)
          for (int du = -1; du <= 1; ++du) {
            const int ua = uc - du, va = vc - dv;
            if (ua < 0 || ua >= si.nu || va < 0 || va >= si.nv) continue;
            const int a = ua + si.nu * va;
            const double* Bb = Bp + int64_t(a) * 81 + ((du + 1) + 3 * (dv + 1)) * 9;
            for (int i = 0; i < 3; ++i) val -= Bb[i * 3 + k] * vp[3 * a + i];
          }
      }
      if (blockIdx.x == 0) w[int64_t(s) * m + row] = val;
    } else {
      val = w[int64_t(s) * m + row];
      if (s < si.ns - 1) {  // - B_s x_{s+1}
        const double* Bs = Bup + int64_t(s) * si.nu * si.nv * 81 + int64_t(c) * 81;
        const double* xp = xs + int64_t(s + 1) * m;
        for (int dv = -1; dv <= 1; ++dv)
          for (int du = -1; du <= 1; ++du) {
            const int ub = uc + du, vb = vc + dv;
            if (ub < 0 || ub >= si.nu || vb < 0 || vb >= si.nv) continue;
            const double* Bb = Bs + ((du + 1) + 3 * (dv + 1)) * 9;
            const int b2 = ub + si.nu * vb;
            for (int j = 0; j < 3; ++j) val -= Bb[k * 3 + j] * xp[3 * b2 + j];
          }
      }
    }
    rhs[row] = val;
  }
  __syncthreads();
  const int warp = tid >> 5, lane = tid & 31;
  const double* Sm = Sinv + int64_t(s) * m * m;
  for (int row = blockIdx.x * 8 + warp; row < m; row += gridDim.x * 8) {
    double acc = 0.0;
    for (int j = lane; j < m; j += 32) acc = fma(Sm[int64_t(row) * m + j], rhs[j], acc);
    acc = warp_sum(acc);
    if (lane == 0) {
      if (fwd) {
        v[int64_t(s) * m + row] = acc;
      } else {
        xs[int64_t(s) * m + row] = acc;
        const int c = row / 3, k = row % 3;
        int gy, gx, gz;
        slab_node(g, si, s, c % si.nu, c / si.nu, gy, gx, gz);
        x[gy + int64_t(nny) * (gx + int64_t(nnx) * gz) + k * g.stride] = T(acc);
      }
    }
  }
}

template <typename T>
void launch_slab_solve(cudaStream_t st, Grid g, SlabInfo si, const double* Sinv, const double* Bup, const T* b,
                       double* w, double* v, T* x, const PcgScalars* sc) {
  if (si.m > SLAB_MAXM) throw std::runtime_error("coarsest slab too large");
  const unsigned nb = unsigned((si.m + 7) / 8);
  const size_t sh = sizeof(double) * size_t(si.m);
  double* xs = v + int64_t(si.ns) * si.m;  // second half of the v buffer
  for (int s = 0; s < si.ns; ++s)
    k_slab_step<T><<<nb, 256, sh, st>>>(g, si, s, 1, Sinv, Bup, b, w, v, xs, x, sc);
  for (int s = si.ns - 1; s >= 0; --s)
    k_slab_step<T><<<nb, 256, sh, st>>>(g, si, s, 0, Sinv, Bup, b, w, v, xs, x, sc);
  TOPX_CUDA_OK(cudaGetLastError());
}

template void launch_diag_coarse<double>(cudaStream_t, Grid, const double*, const uint8_t*, double*);
template void launch_diag_coarse<float>(cudaStream_t, Grid, const double*, const uint8_t*, float*);
template void launch_slab_solve<double>(cudaStream_t, Grid, SlabInfo, const double*, const double*, const double*,
                                        double*, double*, double*, const PcgScalars*);
template void launch_slab_solve<float>(cudaStream_t, Grid, SlabInfo, const double*, const double*, const float*,
                                       double*, double*, float*, const PcgScalars*);

}  // namespace topx
