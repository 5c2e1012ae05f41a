// Coarse-level kernels of the TOP3D_XL B200 path (Solving_AssembleFEAstencil,
// TOP3D_XL.m:919-1018): Galerkin element operators per level and their Jacobi diagonals.
// The coarsest level's direct solver is in topx_nd.cu.
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
  // a group of coarse elements whose children are all void (E = 0) sums to zero: write it
  // without streaming the templates (irregular domains)
  bool any = false;
  for (int i = threadIdx.x; i < GL2_ELEMS * 64; i += GL2_THREADS) any = any || sE[i / 64][i % 64] != 0.0;
  if (!__syncthreads_or(any)) {
    for (int jj = 0; jj < GL2_ELEMS; ++jj) {
      const int64_t j = j0 + jj;
      if (j < nce)
        for (int k = threadIdx.x; k < 576; k += GL2_THREADS) Ks[j * 576 + k] = 0.0;
    }
    return;
  }
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
// The child prolongators are P_c = W_c (x) I_3 (DOFs interleaved, 3 a + i): W_c[a'][b] is the
// weight of coarse node b at child node a'.  So Ks_J = sum_c (W_c^T (x) I) K_c (W_c (x) I) costs
// 2 x 24 x 24 x 8 FMA per child instead of 2 x 24^3, and it sums the same nonzero products in the
// same order as the dense 24 x 24 products (the skipped terms are exact zeros).
constexpr int GS2_THREADS = 192;
constexpr int GS2_PER_THREAD = 8 * 576 / GS2_THREADS;  // 24 outputs of the first product
__global__ void __launch_bounds__(GS2_THREADS) k_galerkin_span2(Grid gc, const double* __restrict__ Ksf,
                                                                const uint8_t* __restrict__ cpresent,
                                                                const double* __restrict__ W8, double* __restrict__ Ks) {
  __shared__ double sK[8 * 576];  // the 8 children's operators, then T_c = K_c (W_c (x) I) in place
  __shared__ double sW[8 * 64];   // W_c[a'][b] at c * 64 + 8 a' + b
  const int64_t J = blockIdx.x;
  const int tid = threadIdx.x;
  if (!cpresent[J]) {  // the same for the whole CTA
    for (int k = tid; k < 576; k += GS2_THREADS) Ks[J * 576 + k] = 0.0;
    return;
  }
  const int gy = int(J % gc.ny), gx = int((J / gc.ny) % gc.nx), gz = int(J / (int64_t(gc.ny) * gc.nx));
  const int fny = 2 * gc.ny, fnx = 2 * gc.nx;
  for (int c = 0; c < 8; ++c) {
    const int cy = c & 1, cx = (c >> 1) & 1, cz = c >> 2;
    const int64_t f = (2 * gy + cy) + int64_t(fny) * ((2 * gx + cx) + int64_t(fnx) * (2 * gz + cz));
    for (int k = tid; k < 576; k += GS2_THREADS) sK[c * 576 + k] = Ksf[f * 576 + k];
  }
  for (int k = tid; k < 8 * 64; k += GS2_THREADS) sW[k] = W8[k];
  __syncthreads();
  // T_c[r][3b + j] = sum_a' K_c[r][3a' + j] W_c[a'][b]
  double t[GS2_PER_THREAD];
#pragma unroll
  for (int m = 0; m < GS2_PER_THREAD; ++m) {
    const int o = tid + m * GS2_THREADS;
    const int c = o / 576, rem = o - 576 * c, r = rem / 24, col = rem - 24 * r, b = col / 3, j = col - 3 * b;
    const double* Kr = sK + c * 576 + r * 24 + j;
    const double* Wc = sW + c * 64 + b;
    double s = 0.0;
#pragma unroll
    for (int ap = 0; ap < 8; ++ap) s = fma(Kr[3 * ap], Wc[8 * ap], s);
    t[m] = s;
  }
  __syncthreads();
#pragma unroll
  for (int m = 0; m < GS2_PER_THREAD; ++m) sK[tid + m * GS2_THREADS] = t[m];
  __syncthreads();
  // Ks_J[3a + i][col] = sum_c sum_a' W_c[a'][a] T_c[3a' + i][col]
  for (int o = tid; o < 576; o += GS2_THREADS) {
    const int row = o / 24, col = o - 24 * row, a = row / 3, i = row - 3 * a;
    double s = 0.0;
    for (int c = 0; c < 8; ++c)
#pragma unroll
      for (int ap = 0; ap < 8; ++ap) s = fma(sW[c * 64 + 8 * ap + a], sK[c * 576 + (3 * ap + i) * 24 + col], s);
    Ks[J * 576 + o] = s;
  }
}

void launch_galerkin_span2(cudaStream_t st, Grid gc, const double* Ksf, const uint8_t* cpresent, const double* W8,
                           double* Ks) {
  (k_galerkin_span2<<<unsigned(gc.nelems()), GS2_THREADS, 0, st>>>(gc, Ksf, cpresent, W8, Ks), topx::count_launch());
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


template void launch_diag_coarse<double>(cudaStream_t, Grid, const double*, const uint8_t*, double*);
template void launch_diag_coarse<float>(cudaStream_t, Grid, const double*, const uint8_t*, float*);

}  // namespace topx
