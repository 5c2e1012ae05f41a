// Level-1 elasticity kernels of the TOP3D_XL B200 path: matrix-free K*u,
// Jacobi diagonal, PCG vector algebra, trilinear multigrid transfers, SIMP,
// unit compliance.  FP64 (plain path) and FP32 (mixed path) instantiations.
#include <cmath>
#include <mutex>
#include <stdexcept>
#include <type_traits>
#include <vector>

#include "topx_ke_classes.h"
#include "topx_kernels.cuh"

namespace topx {

__constant__ double c_Ke64[576];
__constant__ float c_Ke32[576];

template <typename T>
__device__ __forceinline__ T ke(int i);
template <>
__device__ __forceinline__ double ke<double>(int i) {
  return c_Ke64[i];
}
template <>
__device__ __forceinline__ float ke<float>(int i) {
  return c_Ke32[i];
}

// The ten values of Ke (topx_ke_classes.h): the level-1 operator addresses these instead of
// 576 constants, so they stay in uniform registers for the whole launch.
__constant__ double c_Kc64[kKeClasses];
__constant__ float c_Kc32[kKeClasses];

template <typename T>
__device__ __forceinline__ T kcls(int c);
template <>
__device__ __forceinline__ double kcls<double>(int c) {
  return c_Kc64[c];
}
template <>
__device__ __forceinline__ float kcls<float>(int c) {
  return c_Kc32[c];
}
// entry idx of Ke from its class (idx is a compile-time constant once the loops are unrolled)
template <typename T>
__device__ __forceinline__ T kcl(int idx) {
  const int code = ke_class_code(idx);
  return code > 0 ? kcls<T>(code - 1) : -kcls<T>(-code - 1);
}

void upload_ke(const double* Ke576) {
  float f[576];
  for (int i = 0; i < 576; ++i) f[i] = float(Ke576[i]);
  TOPX_CUDA_OK(cudaMemcpyToSymbol(c_Ke64, Ke576, sizeof(double) * 576));
  TOPX_CUDA_OK(cudaMemcpyToSymbol(c_Ke32, f, sizeof(float) * 576));
  // class values from the first entry of each class; every other entry must agree to rounding
  double v[kKeClasses];
  bool seen[kKeClasses] = {};
  for (int i = 0; i < 576; ++i) {
    const int code = ke_class_code(i), c = (code > 0 ? code : -code) - 1;
    if (!seen[c]) {
      v[c] = code > 0 ? Ke576[i] : -Ke576[i];
      seen[c] = true;
    }
  }
  for (int i = 0; i < 576; ++i) {
    const int code = ke_class_code(i), c = (code > 0 ? code : -code) - 1;
    const double e = code > 0 ? v[c] : -v[c];
    if (!(std::fabs(Ke576[i] - e) <= 1e-13 * std::fabs(v[c])))
      throw std::runtime_error("element stiffness does not have the hex8 value classes");
  }
  float vf[kKeClasses];
  for (int c = 0; c < kKeClasses; ++c) vf[c] = float(v[c]);
  TOPX_CUDA_OK(cudaMemcpyToSymbol(c_Kc64, v, sizeof(v)));
  TOPX_CUDA_OK(cudaMemcpyToSymbol(c_Kc32, vf, sizeof(vf)));
}

static inline unsigned grid1d(int64_t n, int threads, int cap = 148 * 16) {
  int64_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > cap) b = cap;
  return unsigned(b);
}

// ---------------------------------------------------------------------------
// K*u, level 1 (Solving_KbyU_MatrixFree, TOP3D_XL.m:684-725).
//
// Node-centric gather: one thread per grid node owns its 3 DOFs.  A CTA of
// 32x8 nodes marches 16 node planes along z, keeping a ring of three
// (32+2)x(8+2) planes of u (masked by the free-DOF mask) and two planes of
// element moduli in shared memory, and sums, for each of the 8 surrounding
// hexes, the node's 3 rows of E_e*Ke times the hex's 24 DOFs (Ke addressed through
// its ten value classes, held in uniform registers).  No atomics: the result is deterministic.  The reference's per-element BC
// matrices (uniqueKesFree_/uniqueKesFixed_) reduce exactly to
//     y = m .* K_E (m .* u) + (1-m) .* cfix .* u
// with m the free-DOF mask and cfix(node) = sum over its hexes of 1/nAdj.
// The PCG mode forms the direction p = z (+ beta*p) on the fly (the update
// kernel stores it) and reduces p'q.
// ---------------------------------------------------------------------------
constexpr int KY = 32, KX = 8, KZC = 16;  // CTA = KY x KX nodes, marching KZC node planes along z
constexpr int KNT = KY * KX;

// Node value seen by the operator: u (plain) or the PCG direction p = z (+ beta p_old).
template <typename T, int MODE>
__device__ __forceinline__ void ku_fetch(const T* __restrict__ in, const T* __restrict__ zin, int64_t n, int64_t S,
                                         bool first, T beta, T& v0, T& v1, T& v2) {
  if (MODE == KU_PLAIN) {
    v0 = in[n];
    v1 = in[n + S];
    v2 = in[n + 2 * S];
  } else if (first) {
    v0 = zin[n];
    v1 = zin[n + S];
    v2 = zin[n + 2 * S];
  } else {
    v0 = zin[n] + beta * in[n];
    v1 = zin[n + S] + beta * in[n + S];
    v2 = zin[n + 2 * S] + beta * in[n + 2 * S];
  }
}

// Accumulate, for the four hexes on one side of the node plane (upper: oz = 0,
// lower: oz = -1), the node's 3 rows of Ke times the hex's 24 DOFs, then add
// E_e * acc to y in the reference's local-node order.  PL(dz, c, dx, dy) is the (masked)
// value of component c of the neighbour at offset (dy, dx, dz); EL(oz, ox, oy) the modulus of
// the hex whose lowest corner is at offset (oy, ox, oz).
template <typename T, int OZ, typename FPL, typename FEL>
__device__ __forceinline__ void ku_half(FPL&& PL, FEL&& EL, T (&y)[3]) {
  T acc[4][3];
#pragma unroll
  for (int e = 0; e < 4; ++e) acc[e][0] = acc[e][1] = acc[e][2] = T(0);
#pragma unroll
  for (int dz = OZ; dz <= OZ + 1; ++dz)
#pragma unroll
    for (int dx = -1; dx <= 1; ++dx)
#pragma unroll
      for (int dy = -1; dy <= 1; ++dy) {
        const T u0 = PL(dz, 0, dx, dy);
        const T u1 = PL(dz, 1, dx, dy);
        const T u2 = PL(dz, 2, dx, dy);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int oy = (e & 1) ? 0 : -1, ox = (e & 2) ? 0 : -1;
          const int ly = dy - oy, lx = dx - ox, lz = dz - OZ;
          if (ly < 0 || ly > 1 || lx < 0 || lx > 1 || lz < 0 || lz > 1) continue;
          const int a = hex_local(-oy, -ox, -OZ), b = hex_local(ly, lx, lz);
#pragma unroll
          for (int i = 0; i < 3; ++i) {
            T s = acc[e][i];
            s = fma(kcl<T>((3 * a + i) * 24 + 3 * b + 0), u0, s);
            s = fma(kcl<T>((3 * a + i) * 24 + 3 * b + 1), u1, s);
            s = fma(kcl<T>((3 * a + i) * 24 + 3 * b + 2), u2, s);
            acc[e][i] = s;
          }
        }
      }
#pragma unroll
  for (int a = (OZ == 0 ? 0 : 4); a < (OZ == 0 ? 4 : 8); ++a) {
    const int oy = -hex_ly(a), ox = -hex_lx(a);
    const int e = (oy + 1) + 2 * (ox + 1);
    const T Ee = EL(OZ, ox, oy);
#pragma unroll
    for (int i = 0; i < 3; ++i) y[i] = fma(Ee, acc[e][i], y[i]);
  }
}

// Plane loads are asynchronous copies one plane ahead: the raw values of node plane z+2
// (u, or z and p_old in PCG mode) land in a staging area and element plane z+1 in a third
// element slot while plane z is computed; the next iteration forms the masked values of
// the staged plane in the node ring.  Only the free-DOF bits ride in registers.
constexpr int KU_NP = (KX + 2) * (KY + 2), KU_EP = (KX + 1) * (KY + 1);
static_assert(KU_NP <= 2 * KNT && KU_EP <= 2 * KNT, "two staged positions per thread");

template <int BYTES>
__device__ __forceinline__ void cp_async_el(void* smem, const void* gmem, bool pred) {
  static_assert(BYTES == 4 || BYTES == 8, "element copy size");
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  const int n = pred ? BYTES : 0;  // 0: fill with zeros, read nothing
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;" ::"r"(s), "l"(gmem), "n"(BYTES), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// A tile of the launch: blockIdx, or entry blockIdx.x of a list of the tiles that own a node of
// the domain (y-tile | x-tile << 10 | z-chunk << 20); tiles of void alone are not launched.
__device__ __forceinline__ void ku_tile(const uint32_t* __restrict__ active, int& ty, int& tx, int& tz) {
  if (active) {
    const uint32_t t = active[blockIdx.x];
    ty = int(t & 1023u);
    tx = int((t >> 10) & 1023u);
    tz = int(t >> 20);
  } else {
    ty = blockIdx.x;
    tx = blockIdx.y;
    tz = blockIdx.z;
  }
}

// In PCG mode with yacc given, each node also takes the previous iteration's solution step
// y += lam p_in (p_in: that iteration's direction; none on the first step).
template <typename T>
__device__ __forceinline__ void ku_solution_step(double* __restrict__ yacc, const T* __restrict__ in, int64_t n,
                                                 int64_t S, double lam) {
#pragma unroll
  for (int c = 0; c < 3; ++c) yacc[n + c * S] = fma(lam, double(in[n + c * S]), yacc[n + c * S]);
}

// Shared memory of the tile kernel (dynamic: above the 48 KB of static shared memory in PCG mode)
template <typename T, int MODE>
struct KuSmem {
  T su[3][3][KX + 2][KY + 2];  // ring of 3 node planes: [slot][comp][x][y], masked by the free mask
  T se[3][KX + 1][KY + 1];     // ring of 3 element planes
  T sa[3][KU_NP];              // staged raw plane: u (plain) or z (PCG mode)
  T sb[MODE == KU_PLAIN ? 1 : 3][MODE == KU_PLAIN ? 1 : KU_NP];  // staged p_old (PCG mode)
  // PCG mode with the solution step: y at the thread's own node of the staged plane, and the
  // step length of the previous iteration (read where used: no register across the plane loop)
  double sy[MODE == KU_PLAIN ? 1 : 3][MODE == KU_PLAIN ? 1 : KNT];
  double s_lam;
};

template <typename T, int MODE>
__global__ void __launch_bounds__(KNT, 3) k_ku_l1(Grid g, int zc, const T* __restrict__ in, const T* __restrict__ zin,
                                                  T* __restrict__ pout, T* __restrict__ out, const T* __restrict__ E,
                                                  const uint8_t* __restrict__ fixbits, const T* __restrict__ cfix,
                                                  PcgScalars* sc, RedScratch rs, const uint32_t* __restrict__ active,
                                                  double* __restrict__ yacc, const uint32_t* __restrict__ zr) {
  if (MODE != KU_PLAIN && sc->done) return;
  extern __shared__ __align__(16) unsigned char ku_dyn_smem[];
  KuSmem<T, MODE>& sm = *reinterpret_cast<KuSmem<T, MODE>*>(ku_dyn_smem);
  auto& su = sm.su;
  auto& se = sm.se;
  auto& sa = sm.sa;
  auto& sb = sm.sb;
  auto& sy = sm.sy;
  double& s_lam = sm.s_lam;
  const int nny = g.ny + 1, nnx = g.nx + 1, nnz = g.nz + 1;
  const int64_t S = g.stride;
  int tyi, txi, tzi;
  ku_tile(active, tyi, txi, tzi);
  const int y0 = tyi * KY, x0 = txi * KX;
  int zc0 = tzi * zc, zend = min(zc0 + zc, nnz);
  if (active && zr) {  // only the planes of the chunk that hold a present node
    const uint32_t r = zr[blockIdx.x];
    zc0 = int(r & 0xffffu);
    zend = int(r >> 16);
  }
  const int ty = threadIdx.x, tx = threadIdx.y;
  const int tid = ty + KY * tx;
  const bool first = (MODE != KU_PLAIN) && sc->first;
  const T beta = (MODE != KU_PLAIN) ? T(sc->beta) : T(0);
  const T* const araw = MODE == KU_PLAIN ? in : zin;
  uint8_t fbs[2];
  const bool ystep = MODE != KU_PLAIN && yacc && !first;
  const bool yown = y0 + ty < nny && x0 + tx < nnx;
  if (ystep && tid == 0) s_lam = sc->lam;

  // issue the copies of node plane zp into the staging area (and its free bits into fbs)
  auto issue_nodes = [&](int zp) {
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      const int i = tid + s * KNT;
      fbs[s] = 0;
      if (i < KU_NP) {
        const int sy = i % (KY + 2), sx = i / (KY + 2);
        const int gy = y0 - 1 + sy, gx = x0 - 1 + sx;
        const bool ok = zp >= 0 && zp < nnz && gy >= 0 && gy < nny && gx >= 0 && gx < nnx;
        const int64_t n = ok ? gy + int64_t(nny) * (gx + int64_t(nnx) * zp) : 0;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          cp_async_el<sizeof(T)>(&sa[c][i], araw + n + c * S, ok);
          if (MODE != KU_PLAIN) cp_async_el<sizeof(T)>(&sb[c][i], in + n + c * S, ok && !first);
        }
        if (ok) fbs[s] = fixbits[n];
      }
    }
  };
  auto issue_elems = [&](int ez, int slot) {
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      const int i = tid + s * KNT;
      if (i < KU_EP) {
        const int sy = i % (KY + 1), sx = i / (KY + 1);
        const int ey = y0 - 1 + sy, ex = x0 - 1 + sx;
        const bool ok = ez >= 0 && ez < g.nz && ey >= 0 && ey < g.ny && ex >= 0 && ex < g.nx;
        const int64_t e = ok ? ey + int64_t(g.ny) * (ex + int64_t(g.nx) * ez) : 0;
        cp_async_el<sizeof(T)>(&se[slot][sx][sy], E + e, ok);
      }
    }
  };
  // The previous iteration's solution step y += lam p_in rides with the plane copies: y at the
  // thread's own node of plane zp is copied beside the staged plane, and when that plane is
  // formed the thread adds lam times the staged p_in there and stores y.
  auto issue_y = [&](int zp) {
    if (ystep && yown && zp >= zc0 && zp < zend) {
      const int64_t n = (y0 + ty) + int64_t(nny) * ((x0 + tx) + int64_t(nnx) * zp);
#pragma unroll
      for (int c = 0; c < 3; ++c) cp_async_el<8>(&sy[c][tid], yacc + n + c * S, true);
    }
  };
  auto step_y = [&](int zp) {
    if (ystep && yown && zp >= zc0 && zp < zend) {
      const int64_t n = (y0 + ty) + int64_t(nny) * ((x0 + tx) + int64_t(nnx) * zp);
      const int io = (ty + 1) + (KY + 2) * (tx + 1);  // the own node's staging position
      const double lam = s_lam;
#pragma unroll
      for (int c = 0; c < 3; ++c) yacc[n + c * S] = fma(lam, double(sb[c][io]), sy[c][tid]);
    }
  };
  // masked values of the staged plane into node slot `slot`
  auto form_nodes = [&](int slot) {
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      const int i = tid + s * KNT;
      if (i < KU_NP) {
        const int sy = i % (KY + 2), sx = i / (KY + 2);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          T v = sa[c][i];
          if (MODE != KU_PLAIN && !first) v = v + beta * sb[c][i];
          su[slot][c][sx][sy] = ((fbs[s] >> c) & 1) ? T(0) : v;
        }
      }
    }
  };

  // prologue: node planes zc0-1, zc0 formed; element planes zc0-1, zc0 and node plane zc0+1 in flight
  issue_nodes(zc0 - 1);
  cp_async_commit();
  cp_async_wait_all();
  __syncthreads();
  form_nodes(0);
  __syncthreads();
  issue_nodes(zc0);
  issue_y(zc0);
  cp_async_commit();
  cp_async_wait_all();
  __syncthreads();
  form_nodes(1);
  step_y(zc0);
  __syncthreads();
  issue_elems(zc0 - 1, 0);
  issue_elems(zc0, 1);
  issue_nodes(zc0 + 1);
  issue_y(zc0 + 1);
  cp_async_commit();
  const int gy = y0 + ty, gx = x0 + tx;
  const bool own = gy < nny && gx < nnx;
  double dot = 0.0;
  for (int k = 0; zc0 + k < zend; ++k) {
    const int z = zc0 + k;
    cp_async_wait_all();
    __syncthreads();
    form_nodes((k + 2) % 3);
    step_y(z + 1);
    __syncthreads();
    if (z + 1 < zend) {
      issue_nodes(z + 2);
      issue_y(z + 2);
      issue_elems(z + 1, (k + 2) % 3);
      cp_async_commit();
    }
    const int64_t n = gy + int64_t(nny) * (gx + int64_t(nnx) * z);
    const uint8_t fbo = own ? fixbits[n] : uint8_t(0);
    if (own) {
      const T(*const pl[3])[KX + 2][KY + 2] = {su[k % 3], su[(k + 1) % 3], su[(k + 2) % 3]};
      const T(*const el[2])[KY + 1] = {se[k % 3], se[(k + 1) % 3]};
      T y[3] = {T(0), T(0), T(0)};
      auto PL = [&](int dz, int c, int dx, int dy) { return pl[dz + 1][c][tx + 1 + dx][ty + 1 + dy]; };
      auto EL = [&](int oz, int ox, int oy) { return el[oz + 1][tx + 1 + ox][ty + 1 + oy]; };
      ku_half<T, 0>(PL, EL, y);   // hexes above the node: local nodes 1-4
      ku_half<T, -1>(PL, EL, y);  // hexes below the node: local nodes 5-8
      // the node's own value: masked copy in the ring for free DOFs, unmasked for fixed ones
      T p[3] = {pl[1][0][tx + 1][ty + 1], pl[1][1][tx + 1][ty + 1], pl[1][2][tx + 1][ty + 1]};
      if (fbo) {
        T p0, p1, p2;
        ku_fetch<T, MODE>(in, zin, n, S, first, beta, p0, p1, p2);
        const T cf = cfix[n];
        if (fbo & 1) {
          p[0] = p0;
          y[0] = cf * p0;
        }
        if (fbo & 2) {
          p[1] = p1;
          y[1] = cf * p1;
        }
        if (fbo & 4) {
          p[2] = p2;
          y[2] = cf * p2;
        }
      }
      out[n] = y[0];
      out[n + S] = y[1];
      out[n + 2 * S] = y[2];
      if (MODE != KU_PLAIN) {
        if (pout) {  // the direction p = z (+ beta p_old) for the PCG update (another buffer than in)
          pout[n] = p[0];
          pout[n + S] = p[1];
          pout[n + 2 * S] = p[2];
        }
        dot += double(p[0]) * double(y[0]) + double(p[1]) * double(y[1]) + double(p[2]) * double(y[2]);
      }
    }
  }
  cp_async_wait_all();
  if (MODE != KU_PLAIN) {
    double v[1] = {dot}, tot[1];
    if (reduce_publish<1>(v, rs, tot) && tid == 0) sc->pq = tot[0];
  }
}

// The last node row y = ny of the grid, when the tile kernel's y-tiles end exactly at it: with
// ny a multiple of the tile height the tile kernel would otherwise run whole tiles for this one
// row (node counts here are 2^k + 1).  A CTA takes 32 x 8 nodes of the row (x, z); its
// threads first stage, together, the masked values of rows y = ny - 1 and ny over the tile and
// a one-node halo, their free bits, and the moduli of element row ny - 1 in shared memory (with
// y the fastest index every node of this row sits in its own DRAM sectors, so the loads are
// issued all at once rather than one neighbour at a time), then each thread applies the same
// operator, in the same FMA order, as the tile kernel to its node.  The p'q partial sum is
// added to the tile kernel's.
constexpr int KLX = 32, KLZ = 8;

template <typename T, int MODE>
__global__ void __launch_bounds__(KLX * KLZ) k_ku_l1_lastrow(Grid g, const T* __restrict__ in, const T* __restrict__ zin,
                                                             T* __restrict__ pout, T* __restrict__ out,
                                                             const T* __restrict__ E, const uint8_t* __restrict__ fixbits,
                                                             const T* __restrict__ cfix, PcgScalars* sc, RedScratch rs,
                                                             double* __restrict__ yacc, const uint32_t* __restrict__ rows) {
  if (MODE != KU_PLAIN && sc->done) return;
  __shared__ T sp[3][KLZ + 2][KLX + 2][2];  // masked values, [comp][z][x][row y = ny - 1, ny]
  __shared__ T se[KLZ + 1][KLX + 1];        // moduli of element row ny - 1
  __shared__ uint8_t sfb[KLZ + 2][KLX + 2][2];
  const int nny = g.ny + 1, nnx = g.nx + 1, nnz = g.nz + 1;
  const int64_t S = g.stride;
  const bool first = (MODE != KU_PLAIN) && sc->first;
  const T beta = (MODE != KU_PLAIN) ? T(sc->beta) : T(0);
  const bool ystep = MODE != KU_PLAIN && yacc && !first;
  const double lam = ystep ? sc->lam : 0.0;
  const int Y = nny - 1;
  int bx = blockIdx.x, bz = blockIdx.y;
  if (rows) {  // entry blockIdx.x of the tiles that hold a present node of the row
    bx = int(rows[blockIdx.x] & 0xffffu);
    bz = int(rows[blockIdx.x] >> 16);
  }
  const int x0 = bx * KLX, z0 = bz * KLZ;
  const int tid = threadIdx.x;
  // stage: position i -> row (i & 1), halo x and z; the two rows of one (x, z) are adjacent in memory
  constexpr int NPOS = 2 * (KLX + 2) * (KLZ + 2);
  for (int i = tid; i < NPOS; i += KLX * KLZ) {
    const int row = i & 1, rest = i >> 1;
    const int sx = rest % (KLX + 2), sz = rest / (KLX + 2);
    const int gx = x0 - 1 + sx, gz = z0 - 1 + sz;
    const bool ok = gx >= 0 && gx < nnx && gz >= 0 && gz < nnz;
    T v0 = T(0), v1 = T(0), v2 = T(0);
    uint8_t fb = 0;
    if (ok) {
      const int64_t n = (Y - 1 + row) + int64_t(nny) * (gx + int64_t(nnx) * gz);
      ku_fetch<T, MODE>(in, zin, n, S, first, beta, v0, v1, v2);
      fb = fixbits[n];
    }
    sp[0][sz][sx][row] = (fb & 1) ? T(0) : v0;
    sp[1][sz][sx][row] = (fb & 2) ? T(0) : v1;
    sp[2][sz][sx][row] = (fb & 4) ? T(0) : v2;
    sfb[sz][sx][row] = fb;
  }
  for (int i = tid; i < (KLX + 1) * (KLZ + 1); i += KLX * KLZ) {
    const int sx = i % (KLX + 1), sz = i / (KLX + 1);
    const int ex = x0 - 1 + sx, ez = z0 - 1 + sz;
    const bool ok = ex >= 0 && ex < g.nx && ez >= 0 && ez < g.nz;
    se[sz][sx] = ok ? E[(Y - 1) + int64_t(g.ny) * (ex + int64_t(g.nx) * ez)] : T(0);
  }
  __syncthreads();
  const int lx = tid % KLX, lz = tid / KLX;
  const int x = x0 + lx, z = z0 + lz;
  double dot = 0.0;
  if (x < nnx && z < nnz) {
    // neighbours at y + 1 and hexes above the row lie outside the grid: zero
    auto PL = [&](int dz, int c, int dx, int dy) { return dy > 0 ? T(0) : sp[c][lz + 1 + dz][lx + 1 + dx][dy + 1]; };
    auto EL = [&](int oz, int ox, int oy) { return oy == 0 ? T(0) : se[lz + 1 + oz][lx + 1 + ox]; };
    T y[3] = {T(0), T(0), T(0)};
    ku_half<T, 0>(PL, EL, y);
    ku_half<T, -1>(PL, EL, y);
    const int64_t n = Y + int64_t(nny) * (x + int64_t(nnx) * z);
    const uint8_t fbo = sfb[lz + 1][lx + 1][1];
    T p[3] = {sp[0][lz + 1][lx + 1][1], sp[1][lz + 1][lx + 1][1], sp[2][lz + 1][lx + 1][1]};
    if (fbo) {
      T p0, p1, p2;
      ku_fetch<T, MODE>(in, zin, n, S, first, beta, p0, p1, p2);
      const T cf = cfix[n];
      if (fbo & 1) {
        p[0] = p0;
        y[0] = cf * p0;
      }
      if (fbo & 2) {
        p[1] = p1;
        y[1] = cf * p1;
      }
      if (fbo & 4) {
        p[2] = p2;
        y[2] = cf * p2;
      }
    }
    out[n] = y[0];
    out[n + S] = y[1];
    out[n + 2 * S] = y[2];
    if (ystep) ku_solution_step(yacc, in, n, S, lam);
    if (MODE != KU_PLAIN) {
      if (pout) {
        pout[n] = p[0];
        pout[n + S] = p[1];
        pout[n + 2 * S] = p[2];
      }
      dot += double(p[0]) * double(y[0]) + double(p[1]) * double(y[1]) + double(p[2]) * double(y[2]);
    }
  }
  if (MODE != KU_PLAIN) {
    double v[1] = {dot}, tot[1];
    if (reduce_publish<1>(v, rs, tot) && threadIdx.x == 0) sc->pq += tot[0];
  }
}

static int g_num_sms = 148;
// once per device and process: engines on several host threads share the attributes
void prepare_fem_kernels() {
  static std::mutex mu;
  static bool done[64] = {};
  int dev = 0;
  TOPX_CUDA_OK(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  if (dev >= 0 && dev < 64 && done[dev]) return;
  int n = 0;
  TOPX_CUDA_OK(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
  if (n > 0) g_num_sms = n;
  TOPX_CUDA_OK(cudaFuncSetAttribute(k_ku_l1<double, KU_PLAIN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    int(sizeof(KuSmem<double, KU_PLAIN>))));
  TOPX_CUDA_OK(cudaFuncSetAttribute(k_ku_l1<double, KU_P_UPDATE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    int(sizeof(KuSmem<double, KU_P_UPDATE>))));
  TOPX_CUDA_OK(cudaFuncSetAttribute(k_ku_l1<float, KU_PLAIN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    int(sizeof(KuSmem<float, KU_PLAIN>))));
  TOPX_CUDA_OK(cudaFuncSetAttribute(k_ku_l1<float, KU_P_UPDATE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    int(sizeof(KuSmem<float, KU_P_UPDATE>))));
  if (dev >= 0 && dev < 64) done[dev] = true;
}

// z-chunk length of the K*u launch: fewest (waves x halo-inclusive planes) for three CTAs per SM
static int ku_z_chunk(int nny, int nnx, int nnz) {
  const int64_t tiles = int64_t((nny + KY - 1) / KY) * ((nnx + KX - 1) / KX);
  const int64_t slots = int64_t(g_num_sms) * 3;
  int best = KZC;
  int64_t bestCost = -1;
  for (int zc = 1; zc <= 24; ++zc) {
    const int64_t ctas = tiles * ((nnz + zc - 1) / zc);
    const int64_t cost = ((ctas + slots - 1) / slots) * (zc + 2);
    if (bestCost < 0 || cost < bestCost) {
      bestCost = cost;
      best = zc;
    }
  }
  return best;
}

// Tile grid of the level-1 K*u launch: y-tiles (a last node row that would fill a tile on its own
// goes to k_ku_l1_lastrow instead), x-tiles and z-chunks.
struct KuGeometry {
  bool lastrow;
  int rows, zc;
  dim3 grd;
};
static KuGeometry ku_geometry(Grid g) {
  KuGeometry k;
  k.lastrow = g.ny >= KY && g.ny % KY == 0;
  k.rows = k.lastrow ? g.ny : g.nny();
  k.zc = ku_z_chunk(k.rows, g.nnx(), g.nnz());
  k.grd = dim3((k.rows + KY - 1) / KY, (g.nnx() + KX - 1) / KX, (g.nnz() + k.zc - 1) / k.zc);
  return k;
}

std::vector<uint32_t> ku_active_tiles(Grid g, const std::vector<uint8_t>& present, std::vector<uint32_t>* zranges) {
  const KuGeometry k = ku_geometry(g);
  const int nny = g.nny(), nnx = g.nnx(), nnz = g.nnz();
  if (k.grd.x > 1024 || k.grd.y > 1024 || k.grd.z > 4095 || nnz > 65535) return {};
  std::vector<uint32_t> list;
  if (zranges) zranges->clear();
  for (unsigned tz = 0; tz < k.grd.z; ++tz)
    for (unsigned tx = 0; tx < k.grd.y; ++tx)
      for (unsigned ty = 0; ty < k.grd.x; ++ty) {
        int lo = -1, hi = -1;
        for (int z = int(tz) * k.zc; z < std::min(nnz, int(tz + 1) * k.zc); ++z) {
          bool any = false;
          for (int x = int(tx) * KX; x < std::min(nnx, int(tx + 1) * KX) && !any; ++x)
            for (int y = int(ty) * KY; y < std::min(k.rows, int(ty + 1) * KY) && !any; ++y)
              any = present[size_t(y + int64_t(nny) * (x + int64_t(nnx) * z))] != 0;
          if (any) {
            if (lo < 0) lo = z;
            hi = z + 1;
          }
        }
        if (lo >= 0) {
          list.push_back(ty | (tx << 10) | (tz << 20));
          if (zranges) zranges->push_back(uint32_t(lo) | (uint32_t(hi) << 16));
        }
      }
  return list;
}

std::vector<uint32_t> ku_active_row_tiles(Grid g, const std::vector<uint8_t>& present) {
  const KuGeometry k = ku_geometry(g);
  std::vector<uint32_t> list;
  if (!k.lastrow) return list;
  const int nny = g.nny(), nnx = g.nnx(), nnz = g.nnz(), Y = nny - 1;
  for (int bz = 0; bz < (nnz + KLZ - 1) / KLZ; ++bz)
    for (int bx = 0; bx < (nnx + KLX - 1) / KLX; ++bx) {
      bool any = false;
      for (int z = bz * KLZ; z < std::min(nnz, (bz + 1) * KLZ) && !any; ++z)
        for (int x = bx * KLX; x < std::min(nnx, (bx + 1) * KLX) && !any; ++x)
          any = present[size_t(Y + int64_t(nny) * (x + int64_t(nnx) * z))] != 0;
      if (any) list.push_back(uint32_t(bx) | (uint32_t(bz) << 16));
    }
  return list;
}

template <typename T>
void launch_ku(cudaStream_t st, KuMode mode, Grid g, const T* in, const T* z, T* pout, T* out, const T* E,
               const uint8_t* fixbits, const T* cfix, PcgScalars* sc, RedScratch rs, KuTiles tiles, double* yacc) {
  if (mode == KU_PLAIN) yacc = nullptr;
  const KuGeometry k = ku_geometry(g);
  const bool lastrow = k.lastrow;
  const int zc = k.zc;
  dim3 blk(KY, KX, 1);
  dim3 grd = tiles.list ? dim3(unsigned(tiles.n)) : k.grd;
  if (tiles.list && tiles.n == 0) grd = dim3(0);
  if (grd.x == 0) {
  } else if (mode == KU_PLAIN)
    (k_ku_l1<T, KU_PLAIN><<<grd, blk, sizeof(KuSmem<T, KU_PLAIN>), st>>>(g, zc, in, z, pout, out, E, fixbits, cfix,
                                                                       sc, rs, tiles.list, yacc, tiles.zr),
     topx::count_launch());
  else
    (k_ku_l1<T, KU_P_UPDATE><<<grd, blk, sizeof(KuSmem<T, KU_P_UPDATE>), st>>>(g, zc, in, z, pout, out, E, fixbits,
                                                                             cfix, sc, rs, tiles.list, yacc, tiles.zr),
     topx::count_launch());
  if (lastrow && !(tiles.list && tiles.rows && tiles.nrows == 0)) {
    const uint32_t* rows = tiles.list ? tiles.rows : nullptr;
    const dim3 nb = rows ? dim3(unsigned(tiles.nrows)) : dim3((g.nnx() + KLX - 1) / KLX, (g.nnz() + KLZ - 1) / KLZ);
    if (mode == KU_PLAIN)
      (k_ku_l1_lastrow<T, KU_PLAIN><<<nb, KLX * KLZ, 0, st>>>(g, in, z, pout, out, E, fixbits, cfix, sc, rs, yacc, rows),
       topx::count_launch());
    else
      (k_ku_l1_lastrow<T, KU_P_UPDATE><<<nb, KLX * KLZ, 0, st>>>(g, in, z, pout, out, E, fixbits, cfix, sc, rs, yacc, rows),
       topx::count_launch());
  }
  TOPX_CUDA_OK(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// Finest-level Jacobi diagonal (TOP3D_XL.m:1020-1050): sum over the node's
// hexes, in local-node order, of E_e * diag(Ke); fixed DOFs take cfix.  Stored
// as its reciprocal (0 on absent nodes) so the smoother multiplies.
// ---------------------------------------------------------------------------
template <typename TE, typename T>
__global__ void k_diag_l1(Grid g, const TE* __restrict__ E, const uint8_t* __restrict__ fixbits,
                          const TE* __restrict__ cfix, const uint8_t* __restrict__ present, T* __restrict__ d) {
  const int64_t N = g.nnodes();
  const int nny = g.ny + 1, nnx = g.nx + 1;
  for (int64_t n = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; n < N; n += int64_t(gridDim.x) * blockDim.x) {
    double v[3] = {0.0, 0.0, 0.0};
    if (present[n]) {
      const int gy = int(n % nny), gx = int((n / nny) % nnx), gz = int(n / (int64_t(nny) * nnx));
      double s[3] = {0.0, 0.0, 0.0};
      for (int a = 0; a < 8; ++a) {
        const int ey = gy - hex_ly(a), ex = gx - hex_lx(a), ez = gz - hex_lz(a);
        if (ey < 0 || ey >= g.ny || ex < 0 || ex >= g.nx || ez < 0 || ez >= g.nz) continue;
        const double Ee = double(E[ey + int64_t(g.ny) * (ex + int64_t(g.nx) * ez)]);
        for (int c = 0; c < 3; ++c) s[c] += double(ke<double>((3 * a + c) * 25)) * Ee;
      }
      const uint8_t fb = fixbits[n];
      for (int c = 0; c < 3; ++c) v[c] = 1.0 / ((fb >> c) & 1 ? double(cfix[n]) : s[c]);
    }
    for (int c = 0; c < 3; ++c) d[n + c * g.stride] = T(v[c]);
  }
}

template <typename TE, typename T>
void launch_diag_l1(cudaStream_t st, Grid g, const TE* E, const uint8_t* fixbits, const TE* cfix,
                    const uint8_t* present, T* d) {
  (k_diag_l1<TE, T><<<grid1d(g.nnodes(), 256), 256, 0, st>>>(g, E, fixbits, cfix, present, d), topx::count_launch());
  TOPX_CUDA_OK(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// PCG vector algebra (TOP3D_XL.m:613-622)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_residual_init(Grid g, const T* __restrict__ b, const T* __restrict__ Ay, T* __restrict__ r,
                                PcgScalars* sc, RedScratch rs, double tol, int maxIT) {
  const int64_t N = g.nnodes(), S = g.stride;
  double bb = 0.0;
  for (int64_t n = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; n < N; n += int64_t(gridDim.x) * blockDim.x) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const T bv = b[n + c * S];
      r[n + c * S] = bv - Ay[n + c * S];
      bb += double(bv) * double(bv);
    }
  }
  double v[1] = {bb}, tot[1];
  if (reduce_publish<1>(v, rs, tot) && threadIdx.x == 0) {
    sc->normB = sqrt(tot[0]);
    sc->tol = tol;
    sc->maxIT = maxIT;
    sc->its = 0;
    sc->done = 0;
    sc->first = 1;
    sc->beta = 0.0;
  }
}

template <typename T>
void launch_residual_init(cudaStream_t st, Grid g, const T* b, const T* Ay, T* r, PcgScalars* sc, RedScratch rs,
                          double tol, int maxIT) {
  (k_residual_init<T><<<grid1d(g.nnodes(), 256), 256, 0, st>>>(g, b, Ay, r, sc, rs, tol, maxIT), topx::count_launch());
  TOPX_CUDA_OK(cudaGetLastError());
}

template <typename T>
struct Vec2;
template <>
struct Vec2<double> {
  using type = double2;
};
template <>
struct Vec2<float> {
  using type = float2;
};

// PGIVEN: p already holds the new direction (written by K*u), z is not read and p not written,
// and the solution step y += lambda p is left to the next K*u (which reads this p as its p_in) or
// to launch_pcg_flush after the last iteration: lambda goes to sc->lam and y is not touched here
template <typename T, typename TY, bool PGIVEN>
__global__ void k_pcg_update(Grid g, TY* __restrict__ y, const T* __restrict__ z, T* __restrict__ p,
                             T* __restrict__ r, const T* __restrict__ q, PcgScalars* sc, RedScratch rs,
                             const uint32_t* __restrict__ act) {
  if (sc->done) return;
  const bool first = sc->first;
  const T beta = T(sc->beta);
  const double lam = sc->x1 / sc->pq;
  const T lamT = T(lam);
  const TY lamY = TY(lam);
  const int64_t S = g.stride;  // a multiple of 32, so node pairs are aligned
  const int64_t npair = (g.nnodes() + 1) / 2;
  double rr = 0.0;
  using V2 = typename Vec2<T>::type;
  using Y2 = typename Vec2<TY>::type;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < npair; i += int64_t(gridDim.x) * blockDim.x) {
    if (!chunk_active(act, 2 * i)) continue;  // both nodes of the pair lie in one chunk
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int64_t k = 2 * i + c * S;
      V2 pv = *reinterpret_cast<const V2*>(p + k);
      if (!PGIVEN) {
        const V2 zv = *reinterpret_cast<const V2*>(z + k);
        pv.x = first ? zv.x : zv.x + beta * pv.x;
        pv.y = first ? zv.y : zv.y + beta * pv.y;
        *reinterpret_cast<V2*>(p + k) = pv;
      }
      if (!PGIVEN) {
        Y2 yv = *reinterpret_cast<const Y2*>(y + k);
        yv.x = fma(lamY, TY(pv.x), yv.x);
        yv.y = fma(lamY, TY(pv.y), yv.y);
        *reinterpret_cast<Y2*>(y + k) = yv;
      }
      const V2 qv = *reinterpret_cast<const V2*>(q + k);
      V2 rv = *reinterpret_cast<const V2*>(r + k);
      rv.x = rv.x - lamT * qv.x;
      rv.y = rv.y - lamT * qv.y;
      *reinterpret_cast<V2*>(r + k) = rv;
      rr += double(rv.x) * double(rv.x) + double(rv.y) * double(rv.y);
    }
  }
  double v[1] = {rr}, tot[1];
  if (reduce_publish<1>(v, rs, tot) && threadIdx.x == 0) {
    sc->lam = lam;
    sc->rr = tot[0];
    sc->resnorm = sqrt(tot[0]) / sc->normB;
    sc->its += 1;
    sc->first = 0;
    if (sc->resnorm < sc->tol)
      sc->done = 1;
    else if (sc->its >= sc->maxIT)
      sc->done = 2;
  }
}

// y += sc->lam * p over every node: the solution step of the last PCG iteration (PGIVEN updates
// leave it to the next K*u)
__global__ void k_pcg_flush(Grid g, double* __restrict__ y, const double* __restrict__ p, const PcgScalars* sc,
                            const uint32_t* __restrict__ act) {
  const double lam = sc->lam;
  const int64_t S = g.stride;
  const int64_t npair = (g.nnodes() + 1) / 2;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < npair; i += int64_t(gridDim.x) * blockDim.x) {
    if (!chunk_active(act, 2 * i)) continue;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int64_t k = 2 * i + c * S;
      const double2 pv = *reinterpret_cast<const double2*>(p + k);
      double2 yv = *reinterpret_cast<const double2*>(y + k);
      yv.x = fma(lam, pv.x, yv.x);
      yv.y = fma(lam, pv.y, yv.y);
      *reinterpret_cast<double2*>(y + k) = yv;
    }
  }
}

void launch_pcg_flush(cudaStream_t st, Grid g, double* y, const double* p, const PcgScalars* sc,
                      const uint32_t* act) {
  (k_pcg_flush<<<grid1d(g.nnodes(), 256), 256, 0, st>>>(g, y, p, sc, act), topx::count_launch());
  TOPX_CUDA_OK(cudaGetLastError());
}

template <typename T, typename TY>
void launch_pcg_update(cudaStream_t st, Grid g, TY* y, const T* z, T* p, T* r, const T* q, PcgScalars* sc,
                       RedScratch rs, const uint32_t* act) {
  if (z)
    (k_pcg_update<T, TY, false><<<grid1d(g.nnodes(), 256), 256, 0, st>>>(g, y, z, p, r, q, sc, rs, act),
     topx::count_launch());
  else
    (k_pcg_update<T, TY, true><<<grid1d(g.nnodes(), 256), 256, 0, st>>>(g, y, z, p, r, q, sc, rs, act),
     topx::count_launch());
  TOPX_CUDA_OK(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// Trilinear restriction R = P^T (Solving_RestrictResidual, TOP3D_XL.m:783-798)
// as three separable passes (y, x, z).  Weights (S-|d|)/S are exact in binary,
// equal to the reference's multiGridOperatorRI entries.
// ---------------------------------------------------------------------------
template <typename TI, typename T, int S, int AXIS>
__global__ void k_restrict_axis(const TI* __restrict__ in, int64_t istr, int iny, int inx, int inz,
                                T* __restrict__ out, int64_t ostr, int ony, int onx, int onz, FastDiv fdy,
                                FastDiv fdx, const uint32_t* __restrict__ cols) {
  const uint32_t N = uint32_t(ony) * onx * onz;
  for (uint32_t n = blockIdx.x * blockDim.x + threadIdx.x; n < N; n += gridDim.x * blockDim.x) {
    const uint32_t q = fdy.div(n), oz = fdx.div(q);
    const int oy = int(n - q * uint32_t(ony)), ox = int(q - oz * uint32_t(onx));
    T acc[3] = {T(0), T(0), T(0)};
    // y pass with a column mask: an input (x, z) column without a present node is zero, and so
    // is the output (written without reading the column)
    if (AXIS == 0 && cols && ((__ldg(cols + (q >> 5)) >> (q & 31)) & 1u) == 0u) {
#pragma unroll
      for (int c = 0; c < 3; ++c) out[n + c * ostr] = T(0);
      continue;
    }
#pragma unroll
    for (int d = -(S - 1); d <= S - 1; ++d) {
      int iy = oy, ix = ox, iz = int(oz);
      int lim;
      if (AXIS == 0) {
        iy = S * oy + d;
        lim = iny;
      } else if (AXIS == 1) {
        ix = S * ox + d;
        lim = inx;
      } else {
        iz = S * int(oz) + d;
        lim = inz;
      }
      const int ia = AXIS == 0 ? iy : (AXIS == 1 ? ix : iz);
      if (ia < 0 || ia >= lim) continue;
      const T w = T(S - (d < 0 ? -d : d)) / T(S);
      const int64_t k = iy + int64_t(iny) * (ix + int64_t(inx) * iz);
#pragma unroll
      for (int c = 0; c < 3; ++c) acc[c] = fma(w, T(in[k + c * istr]), acc[c]);
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) out[n + c * ostr] = acc[c];
  }
}

// The restriction in one pass, for small grids (launch-latency bound): L threads per coarse node,
// one per (x, z) column of its (2S-1)^3 fine taps.  Thread (dx, dz) forms the column's y sum as the
// first axis pass does (a column without a present node is zero, unread), thread dz of the node
// the x sum of its columns as the second pass does, and thread 0 the z sum as the third; each sum
// keeps the pass's element type and tap order, so the result equals the three passes bit for bit.
template <int S>
struct RestrictCoop {
  static constexpr int W = 2 * S - 1;           // taps per axis
  static constexpr int L = S == 4 ? 64 : 16;    // threads per coarse node (>= W * W)
  static constexpr int NODES = 256 / L;         // coarse nodes per block
};
template <int S, typename TI, typename T>
__global__ void __launch_bounds__(256) k_restrict_coop(const TI* __restrict__ in, int64_t istr, int iny, int inx,
                                                      int inz, T* __restrict__ out, int64_t ostr, int ony, int onx,
                                                      int onz, FastDiv fdy, FastDiv fdx,
                                                      const uint32_t* __restrict__ cols) {
  using RC = RestrictCoop<S>;
  constexpr int W = RC::W, L = RC::L, NODES = RC::NODES;
  static_assert(W * W <= L, "a thread per tap column");
  __shared__ T sy[NODES][W * W][3];  // y sums of the node's (dx, dz) columns
  __shared__ T sx[NODES][W][3];      // x sums per dz
  const int sub = threadIdx.x / L, lane = threadIdx.x % L;
  const uint32_t N = uint32_t(ony) * onx * onz;
  for (uint32_t base = blockIdx.x * uint32_t(NODES); base < N; base += gridDim.x * uint32_t(NODES)) {
    const uint32_t n = base + uint32_t(sub);
    const bool valid = n < N;
    const uint32_t q = valid ? fdy.div(n) : 0u, oz = valid ? fdx.div(q) : 0u;
    const int oy = int(n - q * uint32_t(ony)), ox = int(q - oz * uint32_t(onx));
    if (valid && lane < W * W) {
      const int ix = S * ox + lane % W - (S - 1), iz = S * int(oz) + lane / W - (S - 1);
      T t[3] = {T(0), T(0), T(0)};
      if (ix >= 0 && ix < inx && iz >= 0 && iz < inz) {
        const uint32_t col = uint32_t(ix) + uint32_t(inx) * uint32_t(iz);
        if (!cols || ((__ldg(cols + (col >> 5)) >> (col & 31)) & 1u) != 0u) {
#pragma unroll
          for (int dy = -(S - 1); dy <= S - 1; ++dy) {
            const int iy = S * oy + dy;
            if (iy < 0 || iy >= iny) continue;
            const T w = T(S - (dy < 0 ? -dy : dy)) / T(S);
            const int64_t k = iy + int64_t(iny) * (ix + int64_t(inx) * iz);
#pragma unroll
            for (int c = 0; c < 3; ++c) t[c] = fma(w, T(in[k + c * istr]), t[c]);
          }
        }
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) sy[sub][lane][c] = t[c];
    }
    __syncthreads();
    if (valid && lane < W) {
      T t[3] = {T(0), T(0), T(0)};
#pragma unroll
      for (int dx = -(S - 1); dx <= S - 1; ++dx) {
        const int ix = S * ox + dx;
        if (ix < 0 || ix >= inx) continue;
        const T w = T(S - (dx < 0 ? -dx : dx)) / T(S);
#pragma unroll
        for (int c = 0; c < 3; ++c) t[c] = fma(w, sy[sub][lane * W + dx + (S - 1)][c], t[c]);
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) sx[sub][lane][c] = t[c];
    }
    __syncthreads();
    if (valid && lane == 0) {
      T acc[3] = {T(0), T(0), T(0)};
#pragma unroll
      for (int dz = -(S - 1); dz <= S - 1; ++dz) {
        const int iz = S * int(oz) + dz;
        if (iz < 0 || iz >= inz) continue;
        const T w = T(S - (dz < 0 ? -dz : dz)) / T(S);
#pragma unroll
        for (int c = 0; c < 3; ++c) acc[c] = fma(w, sx[sub][dz + (S - 1)][c], acc[c]);
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) out[n + c * ostr] = acc[c];
    }
    __syncthreads();  // the next nodes' sums reuse the shared arrays
  }
}

template <typename TI, typename T>
void launch_restrict(cudaStream_t st, int span, const TI* in, Grid gf, T* tmp1, T* tmp2, T* out, Grid gc,
                     const uint32_t* cols) {
  const int fy = gf.nny(), fx = gf.nnx(), fz = gf.nnz();
  const int cy = gc.nny(), cx = gc.nnx(), cz = gc.nnz();
  const int64_t s1 = int64_t(cy) * fx * fz, s2 = int64_t(cy) * cx * fz;
  if (gf.nnodes() >= (int64_t(1) << 32)) throw std::runtime_error("grid too large for 32-bit node indices");
  const FastDiv dcy{uint32_t(cy)}, dfx{uint32_t(fx)}, dcx{uint32_t(cx)};
  if (gf.nnodes() <= (int64_t(1) << 21) && (span == 2 || span == 4)) {
    // small grids are launch-latency bound: one launch, a thread per tap column of a coarse node
    if (span == 4)
      (k_restrict_coop<4, TI, T><<<grid1d(gc.nnodes() * RestrictCoop<4>::L, 256), 256, 0, st>>>(
           in, gf.stride, fy, fx, fz, out, gc.stride, cy, cx, cz, dcy, dcx, cols),
       topx::count_launch());
    else
      (k_restrict_coop<2, TI, T><<<grid1d(gc.nnodes() * RestrictCoop<2>::L, 256), 256, 0, st>>>(
           in, gf.stride, fy, fx, fz, out, gc.stride, cy, cx, cz, dcy, dcx, cols),
       topx::count_launch());
  } else if (span == 4) {
    (k_restrict_axis<TI, T, 4, 0><<<grid1d(s1, 256), 256, 0, st>>>(in, gf.stride, fy, fx, fz, tmp1, s1, cy, fx, fz, dcy, dfx, cols), topx::count_launch());
    (k_restrict_axis<T, T, 4, 1><<<grid1d(s2, 256), 256, 0, st>>>(tmp1, s1, cy, fx, fz, tmp2, s2, cy, cx, fz, dcy, dcx, nullptr), topx::count_launch());
    (k_restrict_axis<T, T, 4, 2><<<grid1d(gc.nnodes(), 256), 256, 0, st>>>(tmp2, s2, cy, cx, fz, out, gc.stride, cy,
                                                                             cx, cz, dcy, dcx, nullptr), topx::count_launch());
  } else {
    (k_restrict_axis<TI, T, 2, 0><<<grid1d(s1, 256), 256, 0, st>>>(in, gf.stride, fy, fx, fz, tmp1, s1, cy, fx, fz, dcy, dfx, cols), topx::count_launch());
    (k_restrict_axis<T, T, 2, 1><<<grid1d(s2, 256), 256, 0, st>>>(tmp1, s1, cy, fx, fz, tmp2, s2, cy, cx, fz, dcy, dcx, nullptr), topx::count_launch());
    (k_restrict_axis<T, T, 2, 2><<<grid1d(gc.nnodes(), 256), 256, 0, st>>>(tmp2, s2, cy, cx, fz, out, gc.stride, cy,
                                                                             cx, cz, dcy, dcx, nullptr), topx::count_launch());
  }
  TOPX_CUDA_OK(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// Prolongation + Jacobi up-smoothing of the 'Adapted' V-cycle
// (TOP3D_XL.m:757-778, Solving_InterpolationDeviation 800-814):
//   x = omega*(r./d) + P*xc + (omega*r)./d   on present fine nodes.
// The level-1 instance also reduces z'r and updates beta/x1 (TOP3D_XL.m:626-630).
// ---------------------------------------------------------------------------
// SMOOTH = false (the 'Standard' V-cycle) stops after omega*(r/d) + P(xc); the Jacobi
// correction against K x follows in k_jacobi_correct.
template <typename TX, typename T, typename TD, int S, bool DOT, bool SMOOTH = true>
__global__ void __launch_bounds__(256) k_prolong_smooth(const TX* __restrict__ xc, Grid gc, const T* __restrict__ r,
                                                        const TD* __restrict__ dinv,
                                                        const uint8_t* __restrict__ present, T* __restrict__ x,
                                                        Grid gf, FastDiv dny, FastDiv dnx, T omega, PcgScalars* sc,
                                                        RedScratch rs, int init, const uint32_t* __restrict__ act) {
  if ((DOT || !SMOOTH) && sc->done) return;
  const uint32_t fny = uint32_t(gf.nny()), fnx = uint32_t(gf.nnx());
  const uint32_t nn = uint32_t(gf.nnodes());  // < 2^32 (checked at launch)
  const int cny = gc.nny(), cnx = gc.nnx();
  double zr = 0.0;
  // grid-stride over the flattened fine grid: no idle lanes on odd extents, and one
  // reduction tail per CTA instead of one per 256 nodes
  for (uint32_t n = blockIdx.x * blockDim.x + threadIdx.x; n < nn; n += gridDim.x * blockDim.x) {
    if (!chunk_active(act, n)) continue;  // x is zero there and stays so
    T rv[3], di[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      rv[c] = r[n + c * gf.stride];
      di[c] = T(dinv[n + c * gf.stride]);
    }
    T v[3] = {T(0), T(0), T(0)};
    if (present[n]) {
      const uint32_t q = dny.div(n);
      const int fy = int(n - q * fny);
      const uint32_t fzu = dnx.div(q);
      const int fz = int(fzu);
      const int fx = int(q - fzu * fnx);
      const int Y = fy / S, X = fx / S, Z = fz / S;
      const int ty = fy - S * Y, tx = fx - S * X, tz = fz - S * Z;
      T pc[3] = {T(0), T(0), T(0)};
#pragma unroll
      for (int a = 0; a < 8; ++a) {
        // corner a of the coarse hex, summed in the reference's local-node order
        const int oy = hex_ly(a), ox = hex_lx(a), oz = hex_lz(a);
        if ((oy && ty == 0) || (ox && tx == 0) || (oz && tz == 0)) continue;
        const T wy = oy ? T(ty) / T(S) : T(S - ty) / T(S);
        const T wx = ox ? T(tx) / T(S) : T(S - tx) / T(S);
        const T wz = oz ? T(tz) / T(S) : T(S - tz) / T(S);
        const T w = wy * wx * wz;
        const int64_t k = (Y + oy) + int64_t(cny) * ((X + ox) + int64_t(cnx) * (Z + oz));
#pragma unroll
        for (int c = 0; c < 3; ++c) pc[c] = fma(w, T(xc[k + c * gc.stride]), pc[c]);
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        T t = omega * (rv[c] * di[c]);
        t = t + pc[c];
        if (SMOOTH) t = t + (omega * rv[c]) * di[c];
        v[c] = t;
        if (DOT) zr += double(t) * double(rv[c]);
      }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) x[n + c * gf.stride] = v[c];
  }
  if (DOT) {
    double vv[1] = {zr}, tot[1];
    if (reduce_publish<1>(vv, rs, tot) && threadIdx.x == 0) {
      if (init) {
        sc->x1 = tot[0];
      } else {
        sc->beta = tot[0] / sc->x1;
        sc->x1 = tot[0];
      }
    }
  }
}

template <typename TX, typename T, typename TD>
void launch_prolong_smooth(cudaStream_t st, int span, const TX* xc, Grid gc, const T* r, const TD* d,
                           const uint8_t* present, T* x, Grid gf, double omega, bool dot, bool init,
                           PcgScalars* sc, RedScratch rs, const uint32_t* act) {
  if (gf.nnodes() >= (int64_t(1) << 32)) throw std::runtime_error("grid too large for 32-bit node indices");
  const unsigned nb = grid1d(gf.nnodes(), 256, 148 * 8);
  const T w = T(omega);
  const FastDiv dny{uint32_t(gf.nny())}, dnx{uint32_t(gf.nnx())};
  if (span == 4) {
    if (dot)
      (k_prolong_smooth<TX, T, TD, 4, true><<<nb, 256, 0, st>>>(xc, gc, r, d, present, x, gf, dny, dnx, w, sc, rs, init, act),
       topx::count_launch());
    else
      (k_prolong_smooth<TX, T, TD, 4, false><<<nb, 256, 0, st>>>(xc, gc, r, d, present, x, gf, dny, dnx, w, sc, rs, init, act),
       topx::count_launch());
  } else {
    if (dot)
      (k_prolong_smooth<TX, T, TD, 2, true><<<nb, 256, 0, st>>>(xc, gc, r, d, present, x, gf, dny, dnx, w, sc, rs, init, act),
       topx::count_launch());
    else
      (k_prolong_smooth<TX, T, TD, 2, false><<<nb, 256, 0, st>>>(xc, gc, r, d, present, x, gf, dny, dnx, w, sc, rs, init, act),
       topx::count_launch());
  }
  TOPX_CUDA_OK(cudaGetLastError());
}

template <typename TX, typename T, typename TD>
void launch_prolong_add(cudaStream_t st, int span, const TX* xc, Grid gc, const T* r, const TD* d,
                        const uint8_t* present, T* x, Grid gf, double omega, PcgScalars* sc) {
  const unsigned nb = grid1d(gf.nnodes(), 256, 148 * 8);
  const T w = T(omega);
  RedScratch none{nullptr, nullptr};
  if (gf.nnodes() >= (int64_t(1) << 32)) throw std::runtime_error("grid too large for 32-bit node indices");
  const FastDiv dny{uint32_t(gf.nny())}, dnx{uint32_t(gf.nnx())};
  if (span == 4)
    (k_prolong_smooth<TX, T, TD, 4, false, false><<<nb, 256, 0, st>>>(xc, gc, r, d, present, x, gf, dny, dnx, w, sc,
                                                                      none, 0, nullptr),
     topx::count_launch());
  else
    (k_prolong_smooth<TX, T, TD, 2, false, false><<<nb, 256, 0, st>>>(xc, gc, r, d, present, x, gf, dny, dnx, w, sc,
                                                                      none, 0, nullptr),
     topx::count_launch());
  TOPX_CUDA_OK(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// 'Standard' V-cycle pieces (TOP3D_XL.m:758-763, 772-777): pre-smoothing from zero, the
// residual r - K x, and the Jacobi correction after the coarse-grid correction.  All return at
// once when the PCG has finished (sc->done), like the prolongation that writes the V-cycle
// output.
// ---------------------------------------------------------------------------
// x = omega*(r/d) on present nodes (the first line of the restriction loop, TX:757)
template <typename TR, typename T, typename TD>
__global__ void k_jacobi_pre(Grid g, const TR* __restrict__ r, const TD* __restrict__ dinv,
                             const uint8_t* __restrict__ present, T* __restrict__ x, T omega, const PcgScalars* sc) {
  if (sc->done) return;
  const int64_t N = g.nnodes();
  for (int64_t n = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; n < N; n += int64_t(gridDim.x) * blockDim.x) {
    const bool pres = present[n] != 0;
#pragma unroll
    for (int c = 0; c < 3; ++c)
      x[n + c * g.stride] = pres ? omega * (T(r[n + c * g.stride]) * T(dinv[n + c * g.stride])) : T(0);
  }
}
template <typename TR, typename T, typename TD>
void launch_jacobi_pre(cudaStream_t st, Grid g, const TR* r, const TD* d, const uint8_t* present, T* x, double omega,
                       const PcgScalars* sc) {
  (k_jacobi_pre<TR, T, TD><<<grid1d(g.nnodes(), 256), 256, 0, st>>>(g, r, d, present, x, T(omega), sc),
   topx::count_launch());
  TOPX_CUDA_OK(cudaGetLastError());
}

// q = r - q: the residual after pre-smoothing, restricted next (TX:761-762)
template <typename TR, typename T>
__global__ void k_residual_inplace(Grid g, const TR* __restrict__ r, T* __restrict__ q, const PcgScalars* sc) {
  if (sc->done) return;
  const int64_t N = g.nnodes();
  for (int64_t n = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; n < N; n += int64_t(gridDim.x) * blockDim.x) {
#pragma unroll
    for (int c = 0; c < 3; ++c) q[n + c * g.stride] = T(r[n + c * g.stride]) - q[n + c * g.stride];
  }
}
template <typename TR, typename T>
void launch_residual_inplace(cudaStream_t st, Grid g, const TR* r, T* q, const PcgScalars* sc) {
  (k_residual_inplace<TR, T><<<grid1d(g.nnodes(), 256), 256, 0, st>>>(g, r, q, sc), topx::count_launch());
  TOPX_CUDA_OK(cudaGetLastError());
}

// x = x + omega*(r - q)/d on present nodes, q = K x (TX:775-776); the finest instance also
// reduces z'r and updates beta/x1 like the 'Adapted' prolongation (TX:626-630)
template <typename TR, typename T, typename TD, bool DOT>
__global__ void __launch_bounds__(256) k_jacobi_correct(Grid g, const TR* __restrict__ r, const T* __restrict__ q,
                                                        const TD* __restrict__ dinv,
                                                        const uint8_t* __restrict__ present, T* __restrict__ x,
                                                        T omega, PcgScalars* sc, RedScratch rs, int init) {
  if (sc->done) return;
  const int64_t N = g.nnodes();
  double zr = 0.0;
  for (int64_t n = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; n < N; n += int64_t(gridDim.x) * blockDim.x) {
    const bool pres = present[n] != 0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int64_t i = n + c * g.stride;
      const T rv = T(r[i]);
      const T t = pres ? x[i] + (omega * (rv - q[i])) * T(dinv[i]) : T(0);
      x[i] = t;
      if (DOT) zr += double(t) * double(rv);
    }
  }
  if (DOT) {
    double vv[1] = {zr}, tot[1];
    if (reduce_publish<1>(vv, rs, tot) && threadIdx.x == 0) {
      if (init) {
        sc->x1 = tot[0];
      } else {
        sc->beta = tot[0] / sc->x1;
        sc->x1 = tot[0];
      }
    }
  }
}
template <typename TR, typename T, typename TD>
void launch_jacobi_correct(cudaStream_t st, Grid g, const TR* r, const T* q, const TD* d, const uint8_t* present,
                           T* x, double omega, bool dot, bool init, PcgScalars* sc, RedScratch rs) {
  const unsigned nb = grid1d(g.nnodes(), 256, 148 * 8);
  if (dot)
    (k_jacobi_correct<TR, T, TD, true><<<nb, 256, 0, st>>>(g, r, q, d, present, x, T(omega), sc, rs, init ? 1 : 0),
     topx::count_launch());
  else
    (k_jacobi_correct<TR, T, TD, false><<<nb, 256, 0, st>>>(g, r, q, d, present, x, T(omega), sc, rs, init ? 1 : 0),
     topx::count_launch());
  TOPX_CUDA_OK(cudaGetLastError());
}

// K*u on a coarse level with its stored Galerkin matrices (Solving_KbyU_MatrixFree for
// iLevel > 1, TOP3D_XL.m:727-743).  One thread per node: for each hex around it, in
// local-node order (the order accumarray adds them), the product of the node's three rows of
// Ks_e with the hex's 24 DOFs, then the sum over hexes.  Deterministic, no atomics.  The
// reference forms u_e' Ks_e; the Galerkin matrices are symmetric, so rows serve for columns (up
// to the rounding of their assembly).
__global__ void __launch_bounds__(256) k_ku_coarse(Grid g, const double* __restrict__ Ks,
                                                   const uint8_t* __restrict__ epresent,
                                                   const uint8_t* __restrict__ present, const double* __restrict__ u,
                                                   double* __restrict__ y, const PcgScalars* sc) {
  if (sc->done) return;
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
        if (!epresent[e]) continue;
        const double* K = Ks + e * 576 + (3 * a) * 24;  // rows 3a .. 3a + 2
        double t[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int b = 0; b < 8; ++b) {
          const int64_t m = (ey + hex_ly(b)) + int64_t(nny) * ((ex + hex_lx(b)) + int64_t(nnx) * (ez + hex_lz(b)));
          const double u0 = u[m], u1 = u[m + g.stride], u2 = u[m + 2 * g.stride];
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            t[c] = fma(K[c * 24 + 3 * b], u0, t[c]);
            t[c] = fma(K[c * 24 + 3 * b + 1], u1, t[c]);
            t[c] = fma(K[c * 24 + 3 * b + 2], u2, t[c]);
          }
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) s[c] += t[c];
      }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) y[n + c * g.stride] = s[c];
  }
}
void launch_ku_coarse(cudaStream_t st, Grid g, const double* Ks, const uint8_t* epresent, const uint8_t* present,
                      const double* u, double* y, const PcgScalars* sc) {
  (k_ku_coarse<<<grid1d(g.nnodes(), 256), 256, 0, st>>>(g, Ks, epresent, present, u, y, sc), topx::count_launch());
  TOPX_CUDA_OK(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// conversions between the reference's compact numbering and the dense grid
// ---------------------------------------------------------------------------
template <typename TA, typename TB>
__global__ void k_convert(const TA* __restrict__ a, TB* __restrict__ b, int64_t n) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    b[i] = TB(a[i]);
}
template <typename TA, typename TB>
void launch_convert(cudaStream_t st, const TA* a, TB* b, int64_t n) {
  (k_convert<TA, TB><<<grid1d(n, 256), 256, 0, st>>>(a, b, n), topx::count_launch());
  TOPX_CUDA_OK(cudaGetLastError());
}

// interleaved compact DOF vector (3k+c) -> SoA dense grid field
template <typename T>
__global__ void k_c2g_nodes(const double* __restrict__ src, T* __restrict__ dst, Grid g,
                            const int32_t* __restrict__ nmb0, int64_t nn) {
  for (int64_t k = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; k < nn; k += int64_t(gridDim.x) * blockDim.x) {
    const int64_t n = nmb0[k];
    for (int c = 0; c < 3; ++c) dst[n + c * g.stride] = T(src[3 * k + c]);
  }
}
template <typename T>
void launch_compact_to_grid_nodes(cudaStream_t st, const double* src, T* dst, Grid g, const int32_t* nodMapBack0,
                                  int64_t numNodes) {
  (k_c2g_nodes<T><<<grid1d(numNodes, 256), 256, 0, st>>>(src, dst, g, nodMapBack0, numNodes), topx::count_launch());
  TOPX_CUDA_OK(cudaGetLastError());
}
template <typename T>
__global__ void k_g2c_nodes(const T* __restrict__ src, double* __restrict__ dst, Grid g,
                            const int32_t* __restrict__ nmb0, int64_t nn) {
  for (int64_t k = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; k < nn; k += int64_t(gridDim.x) * blockDim.x) {
    const int64_t n = nmb0[k];
    for (int c = 0; c < 3; ++c) dst[3 * k + c] = double(src[n + c * g.stride]);
  }
}
template <typename T>
void launch_grid_to_compact_nodes(cudaStream_t st, const T* src, double* dst, Grid g, const int32_t* nodMapBack0,
                                  int64_t numNodes) {
  (k_g2c_nodes<T><<<grid1d(numNodes, 256), 256, 0, st>>>(src, dst, g, nodMapBack0, numNodes), topx::count_launch());
  TOPX_CUDA_OK(cudaGetLastError());
}

// SIMP moduli E = Emin + xPhys^p (E0 - Emin), compact -> dense (TOP3D_XL.m:107,116)
__global__ void k_simp_scatter(const double* __restrict__ x, const int32_t* __restrict__ emb0, int64_t Ne,
                               double Emin, double E0, double penal, double* __restrict__ Ed,
                               float* __restrict__ Ef) {
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < Ne; e += int64_t(gridDim.x) * blockDim.x) {
    const double v = Emin + pow(x[e], penal) * (E0 - Emin);
    const int64_t k = emb0[e];
    Ed[k] = v;
    if (Ef) Ef[k] = float(v);
  }
}
void launch_simp_scatter(cudaStream_t st, const double* xPhys, const int32_t* eleMapBack0, int64_t Ne, double Emin,
                         double E0, double penal, double* Ed, float* Ef) {
  (k_simp_scatter<<<grid1d(Ne, 256), 256, 0, st>>>(xPhys, eleMapBack0, Ne, Emin, E0, penal, Ed, Ef), topx::count_launch());
  TOPX_CUDA_OK(cudaGetLastError());
}

// TopOpti_ComputeUnitCompliance (TOP3D_XL.m:579-598): ce_e = u_e^T Ke u_e with the
// unmodified Ke, one thread per element (compact order), FP64.
__global__ void k_unit_compliance(Grid g, const double* __restrict__ U, const int32_t* __restrict__ emb0,
                                  int64_t Ne, FastDiv dy, FastDiv dx, double w, int acc, double* __restrict__ ce) {
  const int nny = g.ny + 1, nnx = g.nx + 1;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < Ne; e += int64_t(gridDim.x) * blockDim.x) {
    const uint32_t id = uint32_t(emb0[e]);  // element id on the full box, < 2^31
    const uint32_t q = dy.div(id), ez = dx.div(q);
    const int ey = int(id - q * uint32_t(g.ny)), ex = int(q - ez * uint32_t(g.nx));
    double u[24];
#pragma unroll
    for (int a = 0; a < 8; ++a) {
      const int64_t n = (ey + hex_ly(a)) + int64_t(nny) * ((ex + hex_lx(a)) + int64_t(nnx) * (ez + hex_lz(a)));
#pragma unroll
      for (int c = 0; c < 3; ++c) u[3 * a + c] = U[n + c * g.stride];
    }
    // Ke is symmetric: u^T Ke u = sum_j u_j (Ke_jj u_j + 2 sum_{i<j} Ke_ij u_i), 324 FMA for 600
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < 24; ++j) {
      double t = 0.0;
#pragma unroll
      for (int i = 0; i < j; ++i) t = fma(u[i], c_Ke64[i * 24 + j], t);
      s = fma(u[j], fma(2.0, t, c_Ke64[j * 24 + j] * u[j]), s);
    }
    ce[e] = acc ? ce[e] + w * s : w * s;
  }
}
void launch_unit_compliance(cudaStream_t st, Grid g, const double* U, const int32_t* eleMapBack0, int64_t Ne,
                            double weight, bool accumulate, double* ce) {
  const FastDiv dy{uint32_t(g.ny)}, dx{uint32_t(g.nx)};
  (k_unit_compliance<<<grid1d(Ne, 128), 128, 0, st>>>(g, U, eleMapBack0, Ne, dy, dx, weight, accumulate ? 1 : 0, ce),
   topx::count_launch());
  TOPX_CUDA_OK(cudaGetLastError());
}

// explicit instantiations
#define TOPX_INST(T)                                                                                             \
  template void launch_ku<T>(cudaStream_t, KuMode, Grid, const T*, const T*, T*, T*, const T*, const uint8_t*,   \
                             const T*, PcgScalars*, RedScratch, KuTiles, double*);                               \
  template void launch_diag_l1<T, T>(cudaStream_t, Grid, const T*, const uint8_t*, const T*, const uint8_t*, T*); \
  template void launch_residual_init<T>(cudaStream_t, Grid, const T*, const T*, T*, PcgScalars*, RedScratch,     \
                                        double, int);                                                            \
  template void launch_restrict<T, T>(cudaStream_t, int, const T*, Grid, T*, T*, T*, Grid, const uint32_t*);     \
  template void launch_prolong_smooth<T, T, T>(cudaStream_t, int, const T*, Grid, const T*, const T*,            \
                                               const uint8_t*, T*, Grid, double, bool, bool, PcgScalars*,        \
                                               RedScratch, const uint32_t*);                                     \
  template void launch_compact_to_grid_nodes<T>(cudaStream_t, const double*, T*, Grid, const int32_t*, int64_t); \
  template void launch_grid_to_compact_nodes<T>(cudaStream_t, const T*, double*, Grid, const int32_t*, int64_t);
TOPX_INST(double)
TOPX_INST(float)
template void launch_pcg_update<double, double>(cudaStream_t, Grid, double*, const double*, double*, double*,
                                                const double*, PcgScalars*, RedScratch, const uint32_t*);
template void launch_pcg_update<float, float>(cudaStream_t, Grid, float*, const float*, float*, float*, const float*,
                                              PcgScalars*, RedScratch, const uint32_t*);
template void launch_diag_l1<double, float>(cudaStream_t, Grid, const double*, const uint8_t*, const double*,
                                           const uint8_t*, float*);
template void launch_restrict<double, float>(cudaStream_t, int, const double*, Grid, float*, float*, float*, Grid,
                                             const uint32_t*);
template void launch_prolong_smooth<float, double, float>(cudaStream_t, int, const float*, Grid, const double*,
                                                          const float*, const uint8_t*, double*, Grid, double, bool,
                                                          bool, PcgScalars*, RedScratch, const uint32_t*);
template void launch_prolong_add<double, double, double>(cudaStream_t, int, const double*, Grid, const double*,
                                                        const double*, const uint8_t*, double*, Grid, double,
                                                        PcgScalars*);
template void launch_jacobi_pre<double, double, double>(cudaStream_t, Grid, const double*, const double*,
                                                        const uint8_t*, double*, double, const PcgScalars*);
template void launch_residual_inplace<double, double>(cudaStream_t, Grid, const double*, double*, const PcgScalars*);
template void launch_jacobi_correct<double, double, double>(cudaStream_t, Grid, const double*, const double*,
                                                            const double*, const uint8_t*, double*, double, bool,
                                                            bool, PcgScalars*, RedScratch);
template void launch_convert<double, float>(cudaStream_t, const double*, float*, int64_t);
template void launch_convert<float, double>(cudaStream_t, const float*, double*, int64_t);
template void launch_convert<double, double>(cudaStream_t, const double*, double*, int64_t);

}  // namespace topx

namespace topx {

// E = val on every solid element (compact -> dense); the solid-domain solve of
// TOP3D_XL.m:94-104 uses repmat(modulus_) rather than SIMP(1).
__global__ void k_fill_scatter(const int32_t* __restrict__ emb0, int64_t Ne, double val, double* __restrict__ Ed,
                               float* __restrict__ Ef) {
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < Ne; e += int64_t(gridDim.x) * blockDim.x) {
    Ed[emb0[e]] = val;
    if (Ef) Ef[emb0[e]] = float(val);
  }
}
void launch_fill_scatter(cudaStream_t st, const int32_t* eleMapBack0, int64_t Ne, double val, double* Ed, float* Ef) {
  (k_fill_scatter<<<grid1d(Ne, 256), 256, 0, st>>>(eleMapBack0, Ne, val, Ed, Ef), topx::count_launch());
  TOPX_CUDA_OK(cudaGetLastError());
}

}  // namespace topx
