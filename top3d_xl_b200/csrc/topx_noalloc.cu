// Allocation-free level-1 operator application (topx_ku_noalloc in include/topx.h).
//
// topx_ku copies its host vectors through device buffers that it allocates on every call.
// Some callers cannot allow that: a host whose device memory is all handed out by its own
// pool or allocator (MATLAB's gpuArray manager, a framework's caching allocator capped to a
// fraction of the GPU), or a real-time loop that must not call cudaMalloc/cudaFree, which
// synchronise the device.  For them this file keeps the two grid-layout vectors that the
// operator needs as scratch in one fixed, file-scope device array instead of allocating them.
//
// Limit: the array holds kNoAllocScratchBytes = 32 MiB = 4,194,304 doubles, and the two vectors
// need 2 * 3 * stride of them, so the level-1 grid may have at most 699,040 nodes after padding
// (stride: grid nodes rounded up to 32), e.g. an 87x87x87-element cuboid (88^3 nodes).
// Every GPU on which the library's module is loaded holds the array until the process exits.
#include <cuda_runtime.h>

#include <mutex>
#include <stdexcept>
#include <string>

#include "topx_engine.hpp"
#include "topx_kernels.cuh"

namespace topx {
constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;
constexpr int kNoAllocMaxDevices = 64;
}  // namespace topx

// The scratch itself.  In host code this name is only a handle for cudaGetSymbolAddress,
// never a device address.
static __device__ __align__(256) double topx_noalloc_scratch[topx::kNoAllocScratchBytes / sizeof(double)];

namespace topx {
namespace {
std::mutex g_noalloc_mu;
double* g_noalloc_addr[kNoAllocMaxDevices] = {};
}  // namespace

size_t noalloc_scratch_bytes() { return kNoAllocScratchBytes; }

// Device address of the scratch on `device`, which must be the current device.  Looked up
// with cudaGetSymbolAddress on the first call for that device and cached afterwards.
double* noalloc_scratch(int device) {
  if (device < 0 || device >= kNoAllocMaxDevices)
    throw std::invalid_argument("device ordinal out of range for the fixed scratch table");
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_addr[device]) {
    void* p = nullptr;
    TOPX_CUDA_OK(cudaGetSymbolAddress(&p, topx_noalloc_scratch));
    g_noalloc_addr[device] = static_cast<double*>(p);
  }
  return g_noalloc_addr[device];
}

// y = K u with u and y compact interleaved DOF vectors in device memory (the reference's DOF
// order, like apply_K); grid_u and grid_y are caller-provided scratch of 3 * stride doubles.
void Engine::apply_K_device(const double* d_u, double* d_y, double* grid_u, double* grid_y) {
  const Grid& g = G[0];
  // The engine stream is non-blocking, so nothing orders it after work the caller still has
  // queued on the legacy default stream (a gpuArray kernel, an asynchronous copy into u):
  // wait for that work first.  Work on the caller's own non-blocking or per-thread streams is
  // not seen here; the caller synchronises it before the call.
  TOPX_CUDA_OK(cudaEventRecord(ev_legacy, cudaStreamLegacy));
  TOPX_CUDA_OK(cudaStreamWaitEvent(st, ev_legacy, 0));
  // the scratch keeps the previous call's contents: grid nodes outside the domain must read 0
  TOPX_CUDA_OK(cudaMemsetAsync(grid_u, 0, sizeof(double) * size_t(g.stride) * 3, st));
  launch_compact_to_grid_nodes<double>(st, d_u, grid_u, g, nodMapBack0.p, Nn);
  launch_ku<double>(st, KU_PLAIN, g, grid_u, nullptr, nullptr, grid_y, E64.p, fixbits.p, cfix64.p, nullptr,
                    RedScratch{nullptr, nullptr});
  launch_grid_to_compact_nodes<double>(st, grid_y, d_y, g, nodMapBack0.p, Nn);
  TOPX_CUDA_OK(cudaStreamSynchronize(st));
}

}  // namespace topx
