// Kernel-launch accounting.  libgre_gpu.so is linked with -Wl,--wrap=cudaLaunchKernel, so every
// kernel launch issued by this library's code (its own kernels and the CUB primitives compiled
// into it) passes through __wrap_cudaLaunchKernel, which counts it and forwards to the CUDA
// runtime.  gre_launch_count() reports the running total (used by benchmarks to state how many
// of the library's kernels ran in a timed region).
#include <cuda_runtime.h>

#include <atomic>

#include "../../include/gre_gpu.h"

static std::atomic<unsigned long long> g_launches{0};

extern "C" {

cudaError_t __real_cudaLaunchKernel(const void* func, dim3 grid, dim3 block, void** args, size_t smem, cudaStream_t stream);

cudaError_t __wrap_cudaLaunchKernel(const void* func, dim3 grid, dim3 block, void** args, size_t smem, cudaStream_t stream) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return __real_cudaLaunchKernel(func, grid, block, args, smem, stream);
}

uint64_t gre_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

}  // extern "C"

namespace gre {
// Kernels run from a CUDA graph do not pass through cudaLaunchKernel: a recorded sequence takes
// back the launches counted while it was captured (they did not run then) and adds them again
// at every replay.
void launch_count_add(long long k) { g_launches.fetch_add((unsigned long long)k, std::memory_order_relaxed); }
}  // namespace gre
