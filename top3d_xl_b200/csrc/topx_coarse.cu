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


template void launch_diag_coarse<double>(cudaStream_t, Grid, const double*, const uint8_t*, double*);
template void launch_diag_coarse<float>(cudaStream_t, Grid, const double*, const uint8_t*, float*);

}  // namespace topx
