// Shared device helpers for the TOP3D_XL B200 path.
//
// Layout in HBM (all levels): a dense padded voxel grid per multigrid level,
// MATLAB column-major (y fastest, then x, then z) exactly like the reference's
// element/node numbering; nodal DOF fields are structure-of-arrays
// (component c of grid node n at p[c*stride + n]); absent nodes hold zero.
#pragma once

#include <cuda_runtime.h>
#include <atomic>
#include <cstdint>
#include <cstdio>

namespace topx {

constexpr int kWarp = 32;

// Process-wide count of this library's kernel launches.  Every launch site adds one;
// launches recorded into a CUDA graph are taken back out after the capture, and each
// replay of that graph adds its kernel-node count instead.
inline std::atomic<long long>& launch_counter() {
  static std::atomic<long long> c{0};
  return c;
}
inline void count_launch() { launch_counter().fetch_add(1, std::memory_order_relaxed); }

// Device-resident scalars of one PCG solve (TOP3D_XL.m:600-639).  Written by
// the last block of each reduction kernel, read by every later kernel, so a
// whole PCG iteration runs without a host round trip.
struct PcgScalars {
  double normB;
  double x1;       // z'r of the previous iteration
  double pq;       // p'q
  double rr;       // r'r
  double resnorm;  // ||r|| / ||b||
  double beta;     // x2 / x1
  double lam;      // x1 / pq of the last update: its step y += lam p is applied by the next K*u
                   // (or, after the last iteration, by launch_pcg_flush)
  double tol;
  int its;
  int maxIT;
  int done;  // 0 running, 1 converged, 2 hit maxIT
  int first;
};

// Reduction scratch: per-block partials and a ticket counter.
struct RedScratch {
  double* partials;  // >= kMaxRedBlocks * kMaxRedSlots
  unsigned* ticket;
};
constexpr int kMaxRedBlocks = 1 << 18;
constexpr int kMaxRedSlots = 4;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Block-wide sum of NS values; result valid in thread 0.  blockDim.x*y*z <= 1024.
template <int NS>
__device__ __forceinline__ void block_sum(double (&v)[NS]) {
  __shared__ double sh[NS][32];
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nth = blockDim.x * blockDim.y * blockDim.z;
  const int lane = tid & 31, wid = tid >> 5, nw = (nth + 31) >> 5;
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    double w = warp_sum(v[s]);
    if (lane == 0) sh[s][wid] = w;
  }
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      double w = lane < nw ? sh[s][lane] : 0.0;
      v[s] = warp_sum(w);
    }
  }
  __syncthreads();
}

__device__ __forceinline__ double block_max(double v) {
  __shared__ double sh[32];
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nth = blockDim.x * blockDim.y * blockDim.z;
  const int lane = tid & 31, wid = tid >> 5, nw = (nth + 31) >> 5;
  double w = warp_max(v);
  if (lane == 0) sh[wid] = w;
  __syncthreads();
  if (wid == 0) {
    w = lane < nw ? sh[lane] : -1.0e300;
    v = warp_max(w);
  }
  __syncthreads();
  return v;
}

// Publish this block's NS partial sums; returns true in every thread of the
// block that finishes last.  That block then holds the NS totals (summed over
// blocks in block-index order, so the result is deterministic) in out[].
// Slot s of block b sits at partials[s * stride + b]: the default stride serves
// up to kMaxRedSlots slots of any grid; more slots need stride >= the grid's
// block count and NS * stride <= kMaxRedBlocks * kMaxRedSlots.
template <int NS>
__device__ __forceinline__ bool reduce_publish(double (&v)[NS], RedScratch rs, double (&out)[NS],
                                               unsigned stride = kMaxRedBlocks) {
  block_sum<NS>(v);
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nth = blockDim.x * blockDim.y * blockDim.z;
  const unsigned nb = gridDim.x * gridDim.y * gridDim.z;
  const unsigned bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
  __shared__ bool amLast;
  if (tid == 0) {
#pragma unroll
    for (int s = 0; s < NS; ++s) rs.partials[size_t(s) * stride + bid] = v[s];
    __threadfence();
    const unsigned t = atomicAdd(rs.ticket, 1u);
    amLast = (t == nb - 1);
  }
  __syncthreads();
  if (!amLast) return false;
  __threadfence();
  double acc[NS];
#pragma unroll
  for (int s = 0; s < NS; ++s) acc[s] = 0.0;
  // every slot of a block in one iteration: the loads of all slots are in flight together
#pragma unroll 4
  for (unsigned b = tid; b < nb; b += nth) {
#pragma unroll
    for (int s = 0; s < NS; ++s) acc[s] += __ldcg(&rs.partials[size_t(s) * stride + b]);
  }
  block_sum<NS>(acc);
  __shared__ double tot[NS];
  if (tid == 0) {
#pragma unroll
    for (int s = 0; s < NS; ++s) tot[s] = acc[s];
    *rs.ticket = 0u;
  }
  __syncthreads();
#pragma unroll
  for (int s = 0; s < NS; ++s) out[s] = tot[s];
  return true;
}

// Max-reduction analogue of reduce_publish (one slot).
__device__ __forceinline__ bool reduce_publish_max(double v, RedScratch rs, double& out) {
  v = block_max(v);
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nth = blockDim.x * blockDim.y * blockDim.z;
  const unsigned nb = gridDim.x * gridDim.y * gridDim.z;
  const unsigned bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
  __shared__ bool amLast;
  if (tid == 0) {
    rs.partials[bid] = v;
    __threadfence();
    const unsigned t = atomicAdd(rs.ticket, 1u);
    amLast = (t == nb - 1);
  }
  __syncthreads();
  if (!amLast) return false;
  __threadfence();
  double acc = -1.0e300;
  for (unsigned b = tid; b < nb; b += nth) acc = fmax(acc, __ldcg(&rs.partials[b]));
  acc = block_max(acc);
  __shared__ double tot;
  if (tid == 0) {
    tot = acc;
    *rs.ticket = 0u;
  }
  __syncthreads();
  out = tot;
  return true;
}

// Division of 32-bit unsigned integers by an invariant divisor d >= 1 through a multiply-high
// and shifts (Granlund and Montgomery, "Division by invariant integers using multiplication",
// 1994): with l = ceil(log2 d) and m = floor(2^32 (2^l - d) / d) + 1,
//   q = (t + ((n - t) >> 1)) >> (l - 1),  t = mulhi(m, n)    (l >= 1; d = 1 returns n)
// exact for every n < 2^32.
// Chunk mask of a node grid on an irregular domain: bit c of word c / 32 is set when nodes
// [32 c, 32 c + 32) of the dense grid hold a present node.  Nodes outside every present chunk are
// zero in every vector and stay so, so elementwise passes skip their chunks (a warp's 32
// consecutive nodes share one bit).  A null mask means every chunk is present.
__device__ __forceinline__ bool chunk_active(const uint32_t* __restrict__ act, int64_t n) {
  return !act || ((__ldg(act + (n >> 10)) >> ((n >> 5) & 31)) & 1u) != 0u;
}

struct FastDiv {
  uint32_t d = 1, m = 0;
  int l = 0;
  FastDiv() = default;
  explicit FastDiv(uint32_t dd) : d(dd) {
    while ((uint64_t(1) << l) < d) ++l;
    m = l == 0 ? 0u : uint32_t(((uint64_t(1) << 32) * ((uint64_t(1) << l) - d)) / d + 1);
  }
  __host__ __device__ __forceinline__ uint32_t div(uint32_t n) const {
    if (l == 0) return n;
#ifdef __CUDA_ARCH__
    const uint32_t t = __umulhi(m, n);
#else
    const uint32_t t = uint32_t((uint64_t(m) * n) >> 32);
#endif
    return (t + ((n - t) >> 1)) >> (l - 1);
  }
};

// Local node index (0..7) of the node at corner (ly, lx, lz) of a hex, using
// the reference's local numbering (TOP3D_XL.m:1697): node 1 = (y+1, x, z),
// node 2 = (y+1, x+1, z), node 3 = (y, x+1, z), node 4 = (y, x, z), 5-8 = z+1.
__host__ __device__ constexpr int hex_local(int ly, int lx, int lz) {
  return 4 * lz + (ly ? (lx ? 1 : 0) : (lx ? 2 : 3));
}
__host__ __device__ constexpr int hex_ly(int a) { return ((a & 3) == 0 || (a & 3) == 1) ? 1 : 0; }
__host__ __device__ constexpr int hex_lx(int a) { return ((a & 3) == 1 || (a & 3) == 2) ? 1 : 0; }
__host__ __device__ constexpr int hex_lz(int a) { return a >> 2; }

}  // namespace topx

#define TOPX_CUDA_OK(expr)                                                               \
  do {                                                                                   \
    cudaError_t _e = (expr);                                                             \
    if (_e != cudaSuccess) throw topx::CudaError(_e, #expr, __FILE__, __LINE__);         \
  } while (0)
