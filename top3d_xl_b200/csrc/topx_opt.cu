// Optimiser-side kernels of the TOP3D_XL B200 path: the PDE (Helmholtz)
// density filter (TOP3D_XL.m:816-917), objective/sensitivities
// (TOP3D_XL.m:124-130), OC bisection (TOP3D_XL.m:145-163), MMA subproblem and
// dual interior-point steps (TOP3D_XL.m:1804-2049) and the Heaviside chain of
// the LOCAL driver (TOP3D_XL.m:333-382).
#include "topx_kernels.cuh"
#include "topx_opt.cuh"

#include <algorithm>

namespace topx {

static inline unsigned grid1d(int64_t n, int threads, int cap = 148 * 16) {
  int64_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > cap) b = cap;
  return unsigned(b);
}

// The filter kernel matrix travels as a launch parameter (no process-wide constant memory),
// so engines with different filter radii can run side by side.
template <typename T>
FilterKe<T> filter_ke(const double* KF64) {
  FilterKe<T> k;
  for (int i = 0; i < 64; ++i) k.v[i] = T(KF64[i]);
  return k;
}
template FilterKe<double> filter_ke<double>(const double*);
template FilterKe<float> filter_ke<float>(const double*);

// element -> node: node = sum over its hexes (local-node order) of src_e*(1/8)  (TOP3D_XL.m:880-886)
template <typename T>
__global__ void k_filter_e2n(Grid g, const T* __restrict__ srcE, T* __restrict__ node, FastDiv dny, FastDiv dnx,
                             const uint32_t* __restrict__ act) {
  const uint32_t N = uint32_t(g.nnodes());  // < 2^32 (checked at launch)
  const uint32_t nny = uint32_t(g.ny + 1), nnx = uint32_t(g.nx + 1);
  for (uint32_t n = blockIdx.x * blockDim.x + threadIdx.x; n < N; n += gridDim.x * blockDim.x) {
    if (!chunk_active(act, n)) continue;  // no solid element around these nodes: zero
    const uint32_t q = dny.div(n), qz = dnx.div(q);
    const int gy = int(n - q * nny), gx = int(q - qz * nnx), gz = int(qz);
    T s = T(0);
#pragma unroll
    for (int a = 0; a < 8; ++a) {
      const int ey = gy - hex_ly(a), ex = gx - hex_lx(a), ez = gz - hex_lz(a);
      if (ey < 0 || ey >= g.ny || ex < 0 || ex >= g.nx || ez < 0 || ez >= g.nz) continue;
      s = s + srcE[ey + int64_t(g.ny) * (ex + int64_t(g.nx) * ez)] * T(0.125);
    }
    node[n] = s;
  }
}
template <typename T>
void launch_filter_e2n(cudaStream_t st, Grid g, const T* srcE, T* node, const uint32_t* act) {
  if (g.nnodes() >= (int64_t(1) << 32)) throw std::runtime_error("grid too large for 32-bit node indices");
  const FastDiv dny{uint32_t(g.ny + 1)}, dnx{uint32_t(g.nx + 1)};
  (k_filter_e2n<T><<<grid1d(g.nnodes(), 256), 256, 0, st>>>(g, srcE, node, dny, dnx, act), topx::count_launch());
  TOPX_CUDA_OK(cudaGetLastError());
}

// Jacobi preconditioner 1/diag (TOP3D_XL.m:855-867); 0 on absent nodes
template <typename T>
__global__ void k_filter_diag(Grid g, const uint8_t* __restrict__ solid, const FilterKe<double> kf, T* __restrict__ dp) {
  const int64_t N = g.nnodes();
  const int nny = g.ny + 1, nnx = g.nx + 1;
  for (int64_t n = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; n < N; n += int64_t(gridDim.x) * blockDim.x) {
    const int gy = int(n % nny), gx = int((n / nny) % nnx), gz = int(n / (int64_t(nny) * nnx));
    double s = 0.0;
    for (int a = 0; a < 8; ++a) {
      const int ey = gy - hex_ly(a), ex = gx - hex_lx(a), ez = gz - hex_lz(a);
      if (ey < 0 || ey >= g.ny || ex < 0 || ex >= g.nx || ez < 0 || ez >= g.nz) continue;
      if (solid[ey + int64_t(g.ny) * (ex + int64_t(g.nx) * ez)]) s += kf.v[a * 9];
    }
    dp[n] = s > 0.0 ? T(1.0 / s) : T(0);
  }
}
template <typename T>
void launch_filter_diag(cudaStream_t st, Grid g, const uint8_t* solid, const FilterKe<double>& kf, T* dp) {
  (k_filter_diag<T><<<grid1d(g.nnodes(), 256), 256, 0, st>>>(g, solid, kf, dp), topx::count_launch());
  TOPX_CUDA_OK(cudaGetLastError());
}

// Filter operator y = sum_e KF u_e over solid hexes (MatTimesVec_matrixFree_B, TOP3D_XL.m:904-917),
// node-centric: a CTA of 32x8 nodes marches FKZ node planes along z with a ring of three node
// planes and two planes of solid flags in shared memory; fused PCG direction update and p'q.
// The z-chunk zc is picked per grid so that small grids still give every SM a few CTAs.
constexpr int FKY = 32, FKX = 8, FNT = FKY * FKX;

template <typename T, int MODE>
__global__ void __launch_bounds__(FNT) k_filter_ku(Grid g, int zc, const FilterKe<T> kf, const T* __restrict__ in,
                                                    const T* __restrict__ zin, T* __restrict__ out,
                                                    const uint8_t* __restrict__ solid, PcgScalars* sc, RedScratch rs,
                                                    const uint32_t* __restrict__ active) {
  if (MODE != KU_PLAIN && sc->done) return;
  __shared__ T su[3][FKX + 2][FKY + 2];
  __shared__ T ss[2][FKX + 1][FKY + 1];
  const int nny = g.ny + 1, nnx = g.nx + 1, nnz = g.nz + 1;
  // the CTA's tile: blockIdx, or entry blockIdx.x of the list of tiles that own a node of the
  // domain (y-tile | x-tile << 10 | z-chunk << 20)
  int tyi = blockIdx.x, txi = blockIdx.y, tzi = blockIdx.z;
  if (active) {
    const uint32_t t = active[blockIdx.x];
    tyi = int(t & 1023u);
    txi = int((t >> 10) & 1023u);
    tzi = int(t >> 20);
  }
  const int y0 = tyi * FKY, x0 = txi * FKX, zc0 = tzi * zc;
  const int ty = threadIdx.x, tx = threadIdx.y;
  const int tid = ty + FKY * tx;
  const bool first = (MODE != KU_PLAIN) && sc->first;
  const T beta = (MODE != KU_PLAIN) ? T(sc->beta) : T(0);
  auto load_nodes = [&](int zp, int slot) {
    for (int i = tid; i < (FKX + 2) * (FKY + 2); i += FNT) {
      const int sy = i % (FKY + 2), sx = i / (FKY + 2);
      const int gy = y0 - 1 + sy, gx = x0 - 1 + sx;
      T v = T(0);
      if (zp >= 0 && zp < nnz && gy >= 0 && gy < nny && gx >= 0 && gx < nnx) {
        const int64_t n = gy + int64_t(nny) * (gx + int64_t(nnx) * zp);
        if (MODE == KU_PLAIN)
          v = in[n];
        else
          v = first ? zin[n] : zin[n] + beta * in[n];
      }
      su[slot][sx][sy] = v;
    }
  };
  auto load_solid = [&](int ez, int slot) {
    for (int i = tid; i < (FKX + 1) * (FKY + 1); i += FNT) {
      const int sy = i % (FKY + 1), sx = i / (FKY + 1);
      const int ey = y0 - 1 + sy, ex = x0 - 1 + sx;
      T v = T(0);
      if (ez >= 0 && ez < g.nz && ey >= 0 && ey < g.ny && ex >= 0 && ex < g.nx)
        v = solid[ey + int64_t(g.ny) * (ex + int64_t(g.nx) * ez)] ? T(1) : T(0);
      ss[slot][sx][sy] = v;
    }
  };
  load_nodes(zc0 - 1, 0);
  load_nodes(zc0, 1);
  load_solid(zc0 - 1, 0);
  const int gy = y0 + ty, gx = x0 + tx;
  const bool own = gy < nny && gx < nnx;
  double dot = 0.0;
  for (int k = 0; k < zc; ++k) {
    const int z = zc0 + k;
    if (z >= nnz) break;
    load_nodes(z + 1, (k + 2) % 3);
    load_solid(z, (k + 1) % 2);
    __syncthreads();
    if (own) {
      const T(*const pl[3])[FKY + 2] = {su[k % 3], su[(k + 1) % 3], su[(k + 2) % 3]};
      const T(*const el[2])[FKY + 1] = {ss[k % 2], ss[(k + 1) % 2]};
      T acc[8];
#pragma unroll
      for (int e = 0; e < 8; ++e) acc[e] = T(0);
#pragma unroll
      for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
        for (int dx = -1; dx <= 1; ++dx)
#pragma unroll
          for (int dy = -1; dy <= 1; ++dy) {
            const T u = pl[dz + 1][tx + 1 + dx][ty + 1 + dy];
#pragma unroll
            for (int e = 0; e < 8; ++e) {
              const int oy = (e & 1) ? 0 : -1, ox = (e & 2) ? 0 : -1, oz = (e & 4) ? 0 : -1;
              const int ly = dy - oy, lx = dx - ox, lz = dz - oz;
              if (ly < 0 || ly > 1 || lx < 0 || lx > 1 || lz < 0 || lz > 1) continue;
              const int a = hex_local(-oy, -ox, -oz), b = hex_local(ly, lx, lz);
              acc[e] = fma(kf.v[a * 8 + b], u, acc[e]);
            }
          }
      T y = T(0);
#pragma unroll
      for (int a = 0; a < 8; ++a) {
        const int oy = -hex_ly(a), ox = -hex_lx(a), oz = -hex_lz(a);
        const int e = (oy + 1) + 2 * (ox + 1) + 4 * (oz + 1);
        y = fma(el[oz + 1][tx + 1 + ox][ty + 1 + oy], acc[e], y);
      }
      const int64_t n = gy + int64_t(nny) * (gx + int64_t(nnx) * z);
      out[n] = y;
      if (MODE != KU_PLAIN) dot += double(pl[1][tx + 1][ty + 1]) * double(y);
    }
    __syncthreads();
  }
  if (MODE != KU_PLAIN) {
    double v[1] = {dot}, tot[1];
    if (reduce_publish<1>(v, rs, tot) && tid == 0) sc->pq = tot[0];
  }
}

// tiles of 32 x 8 nodes, each a z-chunk of zc planes (aim at four CTAs per SM)
struct FilterGeometry {
  dim3 grd;
  int zc;
};
static FilterGeometry filter_geometry(Grid g) {
  const int tiles = ((g.nny() + FKY - 1) / FKY) * ((g.nnx() + FKX - 1) / FKX);
  const int chunks = (148 * 4 + tiles - 1) / tiles;
  FilterGeometry f;
  f.zc = std::max(2, std::min(16, (g.nnz() + chunks - 1) / chunks));
  f.grd = dim3((g.nny() + FKY - 1) / FKY, (g.nnx() + FKX - 1) / FKX, (g.nnz() + f.zc - 1) / f.zc);
  return f;
}

std::vector<uint32_t> filter_active_tiles(Grid g, const std::vector<uint8_t>& present) {
  const FilterGeometry f = filter_geometry(g);
  const int nny = g.nny(), nnx = g.nnx(), nnz = g.nnz();
  if (f.grd.x > 1024 || f.grd.y > 1024 || f.grd.z > 4095) return {};
  std::vector<uint32_t> list;
  for (unsigned tz = 0; tz < f.grd.z; ++tz)
    for (unsigned tx = 0; tx < f.grd.y; ++tx)
      for (unsigned ty = 0; ty < f.grd.x; ++ty) {
        bool any = false;
        for (int z = int(tz) * f.zc; z < std::min(nnz, int(tz + 1) * f.zc) && !any; ++z)
          for (int x = int(tx) * FKX; x < std::min(nnx, int(tx + 1) * FKX) && !any; ++x)
            for (int y = int(ty) * FKY; y < std::min(nny, int(ty + 1) * FKY) && !any; ++y)
              any = present[size_t(y + int64_t(nny) * (x + int64_t(nnx) * z))] != 0;
        if (any) list.push_back(ty | (tx << 10) | (tz << 20));
      }
  return list;
}

template <typename T>
void launch_filter_ku(cudaStream_t st, KuMode mode, Grid g, const FilterKe<T>& kf, const T* in, const T* z, T* pout, T* out,
                      const uint8_t* solid, PcgScalars* sc, RedScratch rs, KuTiles tiles) {
  (void)pout;
  const FilterGeometry f = filter_geometry(g);
  dim3 blk(FKY, FKX, 1);
  const dim3 grd = tiles.list ? dim3(unsigned(tiles.n)) : f.grd;
  if (grd.x == 0) return;
  if (mode == KU_PLAIN)
    (k_filter_ku<T, KU_PLAIN><<<grd, blk, 0, st>>>(g, f.zc, kf, in, z, out, solid, sc, rs, tiles.list),
     topx::count_launch());
  else
    (k_filter_ku<T, KU_P_UPDATE><<<grd, blk, 0, st>>>(g, f.zc, kf, in, z, out, solid, sc, rs, tiles.list),
     topx::count_launch());
  TOPX_CUDA_OK(cudaGetLastError());
}

// r = b (y0 = 0), z = dp.*r, p = z, x1 = z'r, normB = ||b||
template <typename T>
__global__ void k_filter_init(Grid g, const T* __restrict__ b, const T* __restrict__ dp, T* __restrict__ r,
                              T* __restrict__ z, T* __restrict__ y, PcgScalars* sc, RedScratch rs, double tol,
                              int maxIT, const uint32_t* __restrict__ act) {
  const int64_t N = g.nnodes();
  double bb = 0.0, zr = 0.0;
  for (int64_t n = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; n < N; n += int64_t(gridDim.x) * blockDim.x) {
    if (!chunk_active(act, n)) continue;  // zero there and stays so
    const T bv = b[n];
    const T zv = dp[n] * bv;
    r[n] = bv;
    z[n] = zv;
    y[n] = T(0);
    bb += double(bv) * double(bv);
    zr += double(zv) * double(bv);
  }
  double v[2] = {bb, zr}, tot[2];
  if (reduce_publish<2>(v, rs, tot) && threadIdx.x == 0) {
    sc->normB = sqrt(tot[0]);
    sc->x1 = tot[1];
    sc->tol = tol;
    sc->maxIT = maxIT;
    sc->its = 0;
    sc->done = 0;
    sc->first = 1;
    sc->beta = 0.0;
  }
}
template <typename T>
void launch_filter_residual_init(cudaStream_t st, Grid g, const T* b, const T* dp, T* r, T* z, T* y, PcgScalars* sc,
                                 RedScratch rs, double tol, int maxIT, const uint32_t* act) {
  (k_filter_init<T><<<grid1d(g.nnodes(), 256), 256, 0, st>>>(g, b, dp, r, z, y, sc, rs, tol, maxIT, act),
   topx::count_launch());
  TOPX_CUDA_OK(cudaGetLastError());
}

// p = z (+ beta p); y += lam p; r -= lam q; stop test; z = dp.*r; beta = z'r / x1
template <typename T>
__global__ void k_filter_update(Grid g, T* __restrict__ y, T* __restrict__ p, T* __restrict__ r,
                                const T* __restrict__ q, const T* __restrict__ dp, T* __restrict__ z, PcgScalars* sc,
                                RedScratch rs, const uint32_t* __restrict__ act) {
  if (sc->done) return;
  const bool first = sc->first;
  const T beta = T(sc->beta);
  const double lam = sc->x1 / sc->pq;
  const T lamT = T(lam);
  const int64_t N = g.nnodes();
  double rr = 0.0, zr = 0.0;
  for (int64_t n = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; n < N; n += int64_t(gridDim.x) * blockDim.x) {
    if (!chunk_active(act, n)) continue;  // zero there and stays so
    const T pv = first ? z[n] : z[n] + beta * p[n];
    p[n] = pv;
    y[n] = y[n] + lamT * pv;
    const T rv = r[n] - lamT * q[n];
    r[n] = rv;
    const T zv = dp[n] * rv;
    z[n] = zv;
    rr += double(rv) * double(rv);
    zr += double(zv) * double(rv);
  }
  double v[2] = {rr, zr}, tot[2];
  if (reduce_publish<2>(v, rs, tot) && threadIdx.x == 0) {
    sc->rr = tot[0];
    sc->resnorm = sqrt(tot[0]) / sc->normB;
    sc->its += 1;
    sc->first = 0;
    if (sc->resnorm < sc->tol) {
      sc->done = 1;
    } else if (sc->its >= sc->maxIT) {
      sc->done = 2;
    } else {
      sc->beta = tot[1] / sc->x1;
      sc->x1 = tot[1];
    }
  }
}
template <typename T>
void launch_filter_update(cudaStream_t st, Grid g, T* y, T* p, T* r, const T* q, const T* dp, T* z, PcgScalars* sc,
                          RedScratch rs, const uint32_t* act) {
  (k_filter_update<T><<<grid1d(g.nnodes(), 256), 256, 0, st>>>(g, y, p, r, q, dp, z, sc, rs, act), topx::count_launch());
  TOPX_CUDA_OK(cudaGetLastError());
}

// node -> element mean (TOP3D_XL.m:894-901), compact element order
template <typename T>
__global__ void k_filter_n2e(Grid g, const T* __restrict__ node, const int32_t* __restrict__ emb0, int64_t Ne,
                             double* __restrict__ out) {
  const int nny = g.ny + 1, nnx = g.nx + 1;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < Ne; e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t id = emb0[e];
    const int ey = int(id % g.ny), ex = int((id / g.ny) % g.nx), ez = int(id / (int64_t(g.ny) * g.nx));
    double s = 0.0;
#pragma unroll
    for (int a = 0; a < 8; ++a)
      s += double(node[(ey + hex_ly(a)) + int64_t(nny) * ((ex + hex_lx(a)) + int64_t(nnx) * (ez + hex_lz(a)))]);
    out[e] = s * (1.0 / 8);
  }
}
template <typename T>
void launch_filter_n2e(cudaStream_t st, Grid g, const T* node, const int32_t* eleMapBack0, int64_t Ne, double* out) {
  (k_filter_n2e<T><<<grid1d(Ne, 256), 256, 0, st>>>(g, node, eleMapBack0, Ne, out), topx::count_launch());
  TOPX_CUDA_OK(cudaGetLastError());
}

template <typename T>
__global__ void k_scatter_elems(const double* __restrict__ src, const int32_t* __restrict__ emb0, int64_t Ne,
                                T* __restrict__ dst) {
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < Ne; e += int64_t(gridDim.x) * blockDim.x)
    dst[emb0[e]] = T(src[e]);
}
template <typename T>
void launch_scatter_elems_t(cudaStream_t st, const double* src, const int32_t* eleMapBack0, int64_t Ne, T* dstE) {
  (k_scatter_elems<T><<<grid1d(Ne, 256), 256, 0, st>>>(src, eleMapBack0, Ne, dstE), topx::count_launch());
  TOPX_CUDA_OK(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// objective and sensitivities (TOP3D_XL.m:124-130 / 323-328)
// ---------------------------------------------------------------------------
__global__ void k_objective(int64_t Ne, const double* __restrict__ ce, const double* __restrict__ xPhys, double cSolid,
                            double Emin, double E0, double penal, double* __restrict__ dc, ObjState* os,
                            RedScratch rs) {
  double sc = 0.0, sv = 0.0;
  const double dsimp = penal * (E0 - Emin);
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < Ne; e += int64_t(gridDim.x) * blockDim.x) {
    const double x = xPhys[e];
    const double cn = ce[e] / cSolid;
    const double E = Emin + pow(x, penal) * (E0 - Emin);
    sc += E * cn;
    sv += x;
    dc[e] = -(dsimp * pow(x, penal - 1)) * cn;
  }
  double v[2] = {sc, sv}, tot[2];
  if (reduce_publish<2>(v, rs, tot) && threadIdx.x == 0) {
    os->cObj = tot[0];
    os->xsum = tot[1];
  }
}
void launch_objective(cudaStream_t st, int64_t Ne, const double* ce, const double* xPhys, double cSolid, double Emin,
                      double E0, double penal, double* dc, ObjState* os, RedScratch rs) {
  (k_objective<<<grid1d(Ne, 256), 256, 0, st>>>(Ne, ce, xPhys, cSolid, Emin, E0, penal, dc, os, rs), topx::count_launch());
  TOPX_CUDA_OK(cudaGetLastError());
}

__global__ void k_dot(int64_t n, const double* __restrict__ a, const double* __restrict__ b, double* out,
                      RedScratch rs) {
  double s = 0.0;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    s += b ? a[i] * b[i] : a[i];
  double v[1] = {s}, tot[1];
  if (reduce_publish<1>(v, rs, tot) && threadIdx.x == 0) *out = tot[0];
}
void launch_sum(cudaStream_t st, int64_t n, const double* a, const double* b, double* out, RedScratch rs) {
  (k_dot<<<grid1d(n, 256), 256, 0, st>>>(n, a, b, out, rs), topx::count_launch());
  TOPX_CUDA_OK(cudaGetLastError());
}

__global__ void k_ewise(int op, int64_t n, const double* __restrict__ a, const double* __restrict__ b,
                        double* __restrict__ out, double s) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    double v;
    switch (op) {
      case EW_MUL:
        v = a[i] * b[i];
        break;
      case EW_DIV_MAXX:  // a ./ max(s, b)
        v = a[i] / fmax(s, b[i]);
        break;
      default:
        v = a[i];
    }
    out[i] = v;
  }
}
void launch_ewise(cudaStream_t st, int op, int64_t n, const double* a, const double* b, double* out, double s) {
  (k_ewise<<<grid1d(n, 256), 256, 0, st>>>(op, n, a, b, out, s), topx::count_launch());
  TOPX_CUDA_OK(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// OC update with Lagrange-multiplier bisection (TOP3D_XL.m:145-156).  Each
// launch evaluates kOcStepsPerLaunch bisection steps as one grid reduction; once
// the interval test fails the remaining launches return at once.
// ---------------------------------------------------------------------------
// x sqrt(-dc / lmid) evaluated as w * r with w = x sqrt(-dc) formed once per OC iteration
// (k_oc_prep) and r = 1 / sqrt(lmid) once per bisection step: the bisection then streams x and w
// with two multiplications per element instead of a division and a square root (the result
// differs from the reference's evaluation order by a few ulps).
__device__ __forceinline__ double oc_xnew(double x, double w, double r, double move) {
  return fmax(0.0, fmax(x - move, fmin(1.0, fmin(x + move, w * r))));
}

__global__ void k_oc_prep(int64_t Ne, const double* __restrict__ x, const double* __restrict__ dc,
                          double* __restrict__ w) {
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < Ne; e += int64_t(gridDim.x) * blockDim.x)
    w[e] = x[e] * sqrt(-dc[e]);
}
void launch_oc_prep(cudaStream_t st, int64_t Ne, const double* x, const double* dc, double* w) {
  (k_oc_prep<<<grid1d(Ne, 256), 256, 0, st>>>(Ne, x, dc, w), topx::count_launch());
  TOPX_CUDA_OK(cudaGetLastError());
}

// kOcStepsPerLaunch bisection steps per launch.  The multipliers the next D = kOcStepsPerLaunch
// steps can try form a binary tree below the current interval (l1, l2): node 0 is its midpoint,
// child 2j+1 the midpoint of node j's lower half (the step found the volume too low, l2 = lmid),
// child 2j+2 of its upper half (l1 = lmid).  One pass over x and w sums the volume change of all
// 2^D - 1 nodes; the last block then walks the tree taking exactly the decisions, interval test
// included, that D launches of a one-step kernel take.  Every node's midpoint and sum are
// formed as the one-step kernel forms them (same expressions, same per-thread order, same
// block-order reduction), so l1, l2, lmid and the step count come out bit-identical.
// In the per-element clamp, max(0, max(x - move, min(1, min(x + move, t)))) is regrouped as
// max(lo, min(hi, t)) with lo = max(0, x - move), hi = min(1, x + move) formed once per element,
// and the two outer selections are written as comparisons (a NaN t, from a positive dc, selects
// hi as fmin does): min and max select one operand exactly, so neither changes a value (up to
// the sign of a zero term of the sum).
constexpr int kOcNodes = (1 << kOcStepsPerLaunch) - 1;

__global__ void __launch_bounds__(256) k_oc_bisect(int64_t Ne, const double* __restrict__ x,
                                                   const double* __restrict__ w, const uint8_t* __restrict__ passive,
                                                   OcState* os, RedScratch rs, double move) {
  if (os->converged) return;
  // thread j < kOcNodes forms node j's 1/sqrt(lmid): its interval follows the path from the root
  __shared__ double sr[kOcNodes];
  if (threadIdx.x < kOcNodes) {
    const int j = threadIdx.x;
    int depth = 0;
    while ((j + 1) >> (depth + 1)) ++depth;  // node j sits at depth floor(log2(j + 1))
    double a = os->l1, b = os->l2;
    for (int d = depth - 1; d >= 0; --d) {  // the branch taken at each level, root first
      const int node = ((j + 1) >> (d + 1)) - 1;
      const double lmid = 0.5 * (b + a);
      if (j + 1 - ((node + 1) << (d + 1)) < (1 << d))  // lower half: l2 = lmid
        b = lmid;
      else
        a = lmid;
    }
    sr[j] = 1.0 / sqrt(0.5 * (b + a));
  }
  __syncthreads();
  double r[kOcNodes];
#pragma unroll
  for (int j = 0; j < kOcNodes; ++j) r[j] = sr[j];
  double s[kOcNodes];
#pragma unroll
  for (int j = 0; j < kOcNodes; ++j) s[j] = 0.0;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < Ne; e += int64_t(gridDim.x) * blockDim.x) {
    const double xv = x[e];
    if (passive && passive[e]) {
#pragma unroll
      for (int j = 0; j < kOcNodes; ++j) s[j] += 1.0 - xv;
    } else {
      const double wv = w[e];
      const double lo = fmax(0.0, xv - move), hi = fmin(1.0, xv + move);
#pragma unroll
      for (int j = 0; j < kOcNodes; ++j) {
        const double t = wv * r[j];
        const double u = t < hi ? t : hi;
        s[j] += (u > lo ? u : lo) - xv;
      }
    }
  }
  double tot[kOcNodes];
  if (reduce_publish<kOcNodes>(s, rs, tot, gridDim.x) && threadIdx.x == 0) {
    double l1 = os->l1, l2 = os->l2, lmid = os->lmid;
    int steps = os->steps, conv = 0, j = 0;
    for (int d = 0; d < kOcStepsPerLaunch; ++d) {
      lmid = 0.5 * (l2 + l1);
      const double gt = os->fval + tot[j];
      if (gt > 0) {
        l1 = lmid;
        j = 2 * j + 2;
      } else {
        l2 = lmid;
        j = 2 * j + 1;
      }
      steps += 1;
      if (!((l2 - l1) / (l1 + l2) > 1e-6)) {
        conv = 1;
        break;
      }
    }
    os->l1 = l1;
    os->l2 = l2;
    os->lmid = lmid;
    os->steps = steps;
    os->converged = conv;
  }
}
void launch_oc_bisect(cudaStream_t st, int64_t Ne, const double* x, const double* w, const uint8_t* passive,
                      OcState* os, RedScratch rs, double move) {
  const unsigned nb = grid1d(Ne, 256);
  static_assert(size_t(kOcNodes) * 148 * 16 <= size_t(kMaxRedBlocks) * kMaxRedSlots, "reduction slots");
  (k_oc_bisect<<<nb, 256, 0, st>>>(Ne, x, w, passive, os, rs, move), topx::count_launch());
  TOPX_CUDA_OK(cudaGetLastError());
}

// x = xnew(lmid); xPhys = x (passive = 1); change = max|xnew - x|; sharpness
__global__ void k_oc_final(int64_t Ne, double* __restrict__ x, const double* __restrict__ w,
                           const uint8_t* __restrict__ passive, double* __restrict__ xPhys, OcState* os,
                           RedScratch rs, RedScratch rs2, double move) {
  const double lmid = os->lmid;
  const double r = 1.0 / sqrt(lmid);
  double ch = 0.0, sh = 0.0;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < Ne; e += int64_t(gridDim.x) * blockDim.x) {
    const double xv = x[e];
    const bool pas = passive && passive[e];
    const double xn = pas ? 1.0 : oc_xnew(xv, w[e], r, move);
    ch = fmax(ch, fabs(xn - xv));
    x[e] = xn;
    xPhys[e] = xn;
    sh += xn * (1.0 - xn);
  }
  double v[1] = {sh}, tot[1];
  if (reduce_publish<1>(v, rs, tot) && threadIdx.x == 0) os->sharpsum = tot[0];
  double mx;
  if (reduce_publish_max(ch, rs2, mx) && threadIdx.x == 0) os->change = mx;
}
void launch_oc_final(cudaStream_t st, int64_t Ne, double* x, const double* w, const uint8_t* passive, double* xPhys,
                     OcState* os, RedScratch rs, RedScratch rs2, double move) {
  (k_oc_final<<<grid1d(Ne, 256), 256, 0, st>>>(Ne, x, w, passive, xPhys, os, rs, rs2, move), topx::count_launch());
  TOPX_CUDA_OK(cudaGetLastError());
}

template void launch_filter_e2n<double>(cudaStream_t, Grid, const double*, double*, const uint32_t*);
template void launch_filter_e2n<float>(cudaStream_t, Grid, const float*, float*, const uint32_t*);
template void launch_filter_diag<double>(cudaStream_t, Grid, const uint8_t*, const FilterKe<double>&, double*);
template void launch_filter_diag<float>(cudaStream_t, Grid, const uint8_t*, const FilterKe<double>&, float*);
template void launch_filter_ku<double>(cudaStream_t, KuMode, Grid, const FilterKe<double>&, const double*, const double*, double*, double*,
                                       const uint8_t*, PcgScalars*, RedScratch, KuTiles);
template void launch_filter_ku<float>(cudaStream_t, KuMode, Grid, const FilterKe<float>&, const float*, const float*, float*, float*,
                                      const uint8_t*, PcgScalars*, RedScratch, KuTiles);
template void launch_filter_residual_init<double>(cudaStream_t, Grid, const double*, const double*, double*, double*,
                                                  double*, PcgScalars*, RedScratch, double, int, const uint32_t*);
template void launch_filter_residual_init<float>(cudaStream_t, Grid, const float*, const float*, float*, float*,
                                                 float*, PcgScalars*, RedScratch, double, int, const uint32_t*);
template void launch_filter_update<double>(cudaStream_t, Grid, double*, double*, double*, const double*,
                                           const double*, double*, PcgScalars*, RedScratch, const uint32_t*);
template void launch_filter_update<float>(cudaStream_t, Grid, float*, float*, float*, const float*, const float*,
                                          float*, PcgScalars*, RedScratch, const uint32_t*);
template void launch_filter_n2e<double>(cudaStream_t, Grid, const double*, const int32_t*, int64_t, double*);
template void launch_filter_n2e<float>(cudaStream_t, Grid, const float*, const int32_t*, int64_t, double*);
template void launch_scatter_elems_t<double>(cudaStream_t, const double*, const int32_t*, int64_t, double*);
template void launch_scatter_elems_t<float>(cudaStream_t, const double*, const int32_t*, int64_t, float*);

}  // namespace topx

namespace topx {

// ---------------------------------------------------------------------------
// MMA with one constraint (MMAseq/GenSub/SolveDIP, TOP3D_XL.m:1804-2049).
// Elements flagged passive are not part of the subproblem (activeEles).
// ---------------------------------------------------------------------------
constexpr double kMmaFeps = 1.0e-6;
constexpr double kMmaC = 1000.0;

__global__ void k_mma_gensub(int64_t n, int iter, double move, const double* __restrict__ xval,
                             const uint8_t* __restrict__ passive, double* __restrict__ xold1,
                             double* __restrict__ xold2, double* __restrict__ low, double* __restrict__ upp,
                             const double* __restrict__ dfdx, const double* __restrict__ dgdx, double gx, int64_t nact,
                             double* __restrict__ alpha, double* __restrict__ beta, double* __restrict__ p0,
                             double* __restrict__ q0, double* __restrict__ pij, double* __restrict__ qij,
                             MmaState* ms, RedScratch rs) {
  double bs = 0.0;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < n; e += int64_t(gridDim.x) * blockDim.x) {
    if (passive && passive[e]) continue;
    const double xv = xval[e];
    const double xmn = fmax(0.0, xv - move), xmx = fmin(1.0, xv + move);
    const double xo1 = xold1[e], xo2 = xold2[e];
    double lo, up;
    if (iter < 3) {
      lo = xv - 0.5 * (xmx - xmn);
      up = xv + 0.5 * (xmx - xmn);
    } else {
      const double zzz = (xv - xo1) * (xo1 - xo2);
      const double gam = zzz > 0 ? 1.2 : (zzz < 0 ? 0.7 : 1.0);
      lo = xv - gam * (xo1 - low[e]);
      up = xv + gam * (upp[e] - xo1);
      lo = fmax(lo, xv - 10.0 * (xmx - xmn));
      lo = fmin(lo, xv - 0.01 * (xmx - xmn));
      up = fmin(up, xv + 10.0 * (xmx - xmn));
      up = fmax(up, xv + 0.01 * (xmx - xmn));
    }
    double al = 0.9 * lo + 0.1 * xv;
    if (al - xmn < 0) al = xmn;
    double be = 0.9 * up + 0.1 * xv;
    if (be - xmx > 0) be = xmx;
    const double df = dfdx[e], dg = dgdx[e];
    const double ux = up - xv, xl = xv - lo;
    const double dfp = df < 0.0 ? 0.0 : df, dfm = -df < 0.0 ? 0.0 : -df;
    const double P0 = ux * ux * (dfp + 0.001 * fabs(df) + 0.5 * kMmaFeps / (up - lo));
    const double Q0 = xl * xl * (dfm + 0.001 * fabs(df) + 0.5 * kMmaFeps / (up - lo));
    const double dgp = dg < 0.0 ? 0.0 : dg, dgm = -dg < 0.0 ? 0.0 : -dg;
    const double extra = 0.001 * fabs(dg) + 0.5 * kMmaFeps / (up - lo);
    const double Pij = ux * ux * (dgp + extra), Qij = xl * xl * (dgm + extra);
    bs += Pij / ux + Qij / xl;
    low[e] = lo;
    upp[e] = up;
    alpha[e] = al;
    beta[e] = be;
    p0[e] = P0;
    q0[e] = Q0;
    pij[e] = Pij;
    qij[e] = Qij;
    xold2[e] = xo1;
    xold1[e] = xv;
  }
  double v[1] = {bs}, tot[1];
  if (reduce_publish<1>(v, rs, tot) && threadIdx.x == 0) {
    ms->b = -gx + tot[0];
    ms->lam = kMmaC / 2.0;
    ms->mu = 1.0;
    ms->epsi = 1.0;
    ms->err = 1.0;
    ms->tol = 1.0e-9 * sqrt(double(nact) + 1.0);
    ms->inner = 0;
    ms->total = 0;
    ms->finished = 0;
  }
}

void launch_mma_gensub(cudaStream_t st, int64_t n, int iter, double move, const double* xval, const uint8_t* passive,
                       double* xold1, double* xold2, double* low, double* upp, const double* dfdx, const double* dgdx,
                       double gx, int64_t nact, double* alpha, double* beta, double* p0, double* q0, double* pij,
                       double* qij, MmaState* ms, RedScratch rs) {
  (k_mma_gensub<<<grid1d(n, 256), 256, 0, st>>>(n, iter, move, xval, passive, xold1, xold2, low, upp, dfdx, dgdx, gx,
                                                nact, alpha, beta, p0, q0, pij, qij, ms, rs), topx::count_launch());
  TOPX_CUDA_OK(cudaGetLastError());
}

__device__ __forceinline__ void mma_x(double lam, double lo, double up, double al, double be, double P0, double Q0,
                                      double Pij, double Qij, double& xcl, double& xun, double& pj, double& qj) {
  pj = P0 + Pij * lam;
  qj = Q0 + Qij * lam;
  const double sp = sqrt(pj), sq = sqrt(qj);
  xun = (sp * lo + sq * up) / (sp + sq);
  xcl = xun;
  if (xcl - al < 0) xcl = al;
  if (xcl - be > 0) xcl = be;
}

// one Newton step of the dual interior point method (XYZofLAMBDA, DualGrad,
// DualHess, DualLineSearch: TOP3D_XL.m:1930-2031)
__global__ void k_mma_newton(int64_t n, const uint8_t* __restrict__ passive, const double* __restrict__ low,
                             const double* __restrict__ upp, const double* __restrict__ alpha,
                             const double* __restrict__ beta, const double* __restrict__ p0,
                             const double* __restrict__ q0, const double* __restrict__ pij,
                             const double* __restrict__ qij, MmaState* ms, RedScratch rs) {
  if (ms->finished) return;
  const double lam = fmax(ms->lam, 0.0);
  double sg = 0.0, sh = 0.0;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < n; e += int64_t(gridDim.x) * blockDim.x) {
    if (passive && passive[e]) continue;
    const double lo = low[e], up = upp[e];
    double xc, xu, pj, qj;
    mma_x(lam, lo, up, alpha[e], beta[e], p0[e], q0[e], pij[e], qij[e], xc, xu, pj, qj);
    const double ux = up - xc, xl = xc - lo;
    sg += pij[e] / ux + qij[e] / xl;
    const double PQ = pij[e] / (ux * ux) - qij[e] / (xl * xl);
    double df2 = -1.0 / (2.0 * pj / (ux * ux * ux) + 2.0 * qj / (xl * xl * xl));
    if (xu - alpha[e] < 0) df2 = 0.0;
    if (xu - beta[e] > 0) df2 = 0.0;
    sh += PQ * df2 * PQ;
  }
  double v[2] = {sg, sh}, tot[2];
  if (reduce_publish<2>(v, rs, tot) && threadIdx.x == 0) {
    double L = lam, mu = ms->mu;
    const double epsi = ms->epsi;
    const double y = fmax(L - kMmaC, 0.0);
    double grad = -ms->b - 0.0 - y + tot[0];
    grad = -1.0 * grad - epsi / L;
    double H = tot[1];
    if (L > kMmaC) H -= 1.0;
    H -= mu / L;
    double corr = 1e-4 * H / 1.0;
    if (-1.0 * corr < 1.0e-7) corr = -1.0e-7;
    H += corr;
    const double s1 = grad / H;
    const double s2 = -mu + epsi / L - s1 * mu / L;
    double theta = 1.005;
    if (theta < -1.01 * s1 / L) theta = -1.01 * s1 / L;
    if (theta < -1.01 * s2 / mu) theta = -1.01 * s2 / mu;
    theta = 1.0 / theta;
    ms->lam = L + theta * s1;
    ms->mu = mu + theta * s2;
    ms->grad = grad;
    ms->hess = H;
  }
}

void launch_mma_newton(cudaStream_t st, int64_t n, const uint8_t* passive, const double* low, const double* upp,
                       const double* alpha, const double* beta, const double* p0, const double* q0, const double* pij,
                       const double* qij, MmaState* ms, RedScratch rs) {
  (k_mma_newton<<<grid1d(n, 256), 256, 0, st>>>(n, passive, low, upp, alpha, beta, p0, q0, pij, qij, ms, rs), topx::count_launch());
  TOPX_CUDA_OK(cudaGetLastError());
}

// XYZofLAMBDA + DualResidual (TOP3D_XL.m:1967-1984, 2033-2049) and the epsilon schedule
__global__ void k_mma_residual(int64_t n, const uint8_t* __restrict__ passive, const double* __restrict__ low,
                               const double* __restrict__ upp, const double* __restrict__ alpha,
                               const double* __restrict__ beta, const double* __restrict__ p0,
                               const double* __restrict__ q0, const double* __restrict__ pij,
                               const double* __restrict__ qij, double* __restrict__ x, MmaState* ms, RedScratch rs) {
  if (ms->finished) return;
  const double lam = fmax(ms->lam, 0.0);
  double sp = 0.0, sq = 0.0;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < n; e += int64_t(gridDim.x) * blockDim.x) {
    if (passive && passive[e]) continue;
    const double lo = low[e], up = upp[e];
    double xc, xu, pj, qj;
    mma_x(lam, lo, up, alpha[e], beta[e], p0[e], q0[e], pij[e], qij[e], xc, xu, pj, qj);
    x[e] = xc;
    sp += pij[e] / (up - xc);
    sq += qij[e] / (xc - lo);
  }
  double v[2] = {sp, sq}, tot[2];
  if (reduce_publish<2>(v, rs, tot) && threadIdx.x == 0) {
    ms->lam = lam;
    const double y = fmax(lam - kMmaC, 0.0);
    double r1 = -ms->b - 0.0 - y + ms->mu;
    r1 = r1 + tot[0] + tot[1];
    const double r2 = ms->mu * lam - ms->epsi;
    double err = 0.0;
    if (err < fabs(r1)) err = fabs(r1);
    if (err < fabs(r2)) err = fabs(r2);
    ms->err = err;
    ms->inner += 1;
    ms->total += 1;
    if (!(err > 0.9 * ms->epsi && ms->inner < 100)) {
      ms->epsi *= 0.1;
      ms->inner = 0;
      if (!(ms->epsi > ms->tol)) ms->finished = 1;
    }
  }
}

void launch_mma_residual(cudaStream_t st, int64_t n, const uint8_t* passive, const double* low, const double* upp,
                         const double* alpha, const double* beta, const double* p0, const double* q0,
                         const double* pij, const double* qij, double* x, MmaState* ms, RedScratch rs) {
  (k_mma_residual<<<grid1d(n, 256), 256, 0, st>>>(n, passive, low, upp, alpha, beta, p0, q0, pij, qij, x, ms, rs), topx::count_launch());
  TOPX_CUDA_OK(cudaGetLastError());
}

// x = xmma on active elements, 1 on passive ones; change = max |xmma - xval| (xval kept in xold1)
__global__ void k_mma_finish(int64_t n, const uint8_t* __restrict__ passive, const double* __restrict__ xmma,
                             const double* __restrict__ xold1, double* __restrict__ x, MmaState* ms, RedScratch rs) {
  double ch = 0.0;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < n; e += int64_t(gridDim.x) * blockDim.x) {
    if (passive && passive[e]) {
      x[e] = 1.0;
      continue;
    }
    ch = fmax(ch, fabs(xmma[e] - xold1[e]));
    x[e] = xmma[e];
  }
  double mx;
  if (reduce_publish_max(ch, rs, mx) && threadIdx.x == 0) ms->change = mx;
}

void launch_mma_finish(cudaStream_t st, int64_t n, const uint8_t* passive, const double* xmma, const double* xold1,
                       double* x, MmaState* ms, RedScratch rs) {
  (k_mma_finish<<<grid1d(n, 256), 256, 0, st>>>(n, passive, xmma, xold1, x, ms, rs), topx::count_launch());
  TOPX_CUDA_OK(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// LOCAL driver elementwise chain (TOP3D_XL.m:333-350, 380-382)
// ---------------------------------------------------------------------------
__global__ void k_pnorm(int64_t Ne, const double* __restrict__ xhat, double Ve0, double pP, double* out,
                        RedScratch rs) {
  double s = 0.0;
  const double vm = pow(Ve0, pP);
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < Ne; e += int64_t(gridDim.x) * blockDim.x)
    s += pow(xhat[e], pP) / vm;
  double v[1] = {s}, tot[1];
  if (reduce_publish<1>(v, rs, tot) && threadIdx.x == 0) *out = tot[0];
}
void launch_pnorm_terms(cudaStream_t st, int64_t Ne, const double* xhat, double Ve0, int pPIO, double* out_sum,
                        RedScratch rs) {
  (k_pnorm<<<grid1d(Ne, 256), 256, 0, st>>>(Ne, xhat, Ve0, double(pPIO), out_sum, rs), topx::count_launch());
  TOPX_CUDA_OK(cudaGetLastError());
}

__global__ void k_local_sens(int64_t Ne, const double* __restrict__ xhat, const double* __restrict__ xTilde,
                             const double* __restrict__ dc, double Ve0, double pP, double pn, double bt, double eta,
                             double* __restrict__ dfdx_pde, double* __restrict__ dx, double* __restrict__ dcdx) {
  const double f = pow(pn, 1.0 / pP - 1.0);
  const double vm = pow(Ve0, pP);
  const double den = tanh(bt * eta) + tanh(bt * (1 - eta));
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < Ne; e += int64_t(gridDim.x) * blockDim.x) {
    dfdx_pde[e] = f * (pow(xhat[e], pP - 1) / vm) / double(Ne);
    const double th = tanh(bt * (xTilde[e] - eta));
    const double d = bt * (1 - th * th) / den;
    dx[e] = d;
    dcdx[e] = dc[e] * d;
  }
}
void launch_local_sens(cudaStream_t st, int64_t Ne, const double* xhat, const double* xTilde, const double* dc,
                       double Ve0, int pPIO, double pn, double betaPIO, double etaPIO, double* dfdx_pde, double* dx,
                       double* dcdx) {
  (k_local_sens<<<grid1d(Ne, 256), 256, 0, st>>>(Ne, xhat, xTilde, dc, Ve0, double(pPIO), pn, betaPIO, etaPIO,
                                                dfdx_pde, dx, dcdx), topx::count_launch());
  TOPX_CUDA_OK(cudaGetLastError());
}

__global__ void k_heaviside(int64_t Ne, const double* __restrict__ xTilde, const uint8_t* __restrict__ passive,
                            double bt, double eta, double* __restrict__ xPhys, double* sharpsum, RedScratch rs) {
  const double a = tanh(bt * eta), den = tanh(bt * eta) + tanh(bt * (1 - eta));
  double s = 0.0;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < Ne; e += int64_t(gridDim.x) * blockDim.x) {
    double v = (a + tanh(bt * (xTilde[e] - eta))) / den;
    if (passive && passive[e]) v = 1.0;
    xPhys[e] = v;
    s += v * (1.0 - v);
  }
  double vv[1] = {s}, tot[1];
  if (reduce_publish<1>(vv, rs, tot) && threadIdx.x == 0) *sharpsum = tot[0];
}
void launch_heaviside(cudaStream_t st, int64_t Ne, const double* xTilde, const uint8_t* passive, double betaPIO,
                      double etaPIO, double* xPhys, double* sharpsum, RedScratch rs) {
  (k_heaviside<<<grid1d(Ne, 256), 256, 0, st>>>(Ne, xTilde, passive, betaPIO, etaPIO, xPhys, sharpsum, rs), topx::count_launch());
  TOPX_CUDA_OK(cudaGetLastError());
}

}  // namespace topx
