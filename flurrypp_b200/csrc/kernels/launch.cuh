// Kernel launches with programmatic dependent launch (PDL) for small cases.
//
// A small case (a served request, a P-multigrid coarse level) runs hundreds
// of kernels per step, each a few microseconds long, so the gaps between
// dependent launches dominate.  With PDL a kernel may be launched while its
// predecessor on the stream is still finishing: every kernel of this library
// calls pdl_wait() before it touches global memory (it returns once the
// predecessor grid has completed and its writes are visible) and then
// pdl_trigger(), which lets its own successor start launching.  Launched
// without the PDL attribute both are no-ops.  The attribute is set only for
// cases whose grids fit in about one wave (set_pdl), where an early successor
// cannot take SM slots from later waves of its predecessor.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <utility>

namespace frk {

__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Maximum that keeps a NaN of either operand (fmax returns the other one), so
// a blown-up residual reaches the host's NaN check through a max-norm.
__device__ __forceinline__ double nan_max(double a, double b) { return (a != a || a > b) ? a : b; }

// Asynchronous copy of one 8-byte (double) or 4-byte (float) word global ->
// shared (cp.async); a thread's copies complete in commit-group order.
template <typename R>
__device__ __forceinline__ void cp_async_word(R *dst, const R *src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  if constexpr (sizeof(R) == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// wait until at most N of this thread's newest groups are pending
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

inline int current_device() {
  int d = 0;
  cudaGetDevice(&d);
  return d;
}
// streaming multiprocessors of device d (queried once per device)
inline int sm_count(int d) {
  static std::atomic<int> cache[64];
  if (d < 0 || d >= 64) return 148;
  int v = cache[d].load(std::memory_order_relaxed);
  if (v > 0) return v;
  cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, d);
  if (v <= 0) v = 148;
  cache[d].store(v, std::memory_order_relaxed);
  return v;
}

// Launch policy of the calling host thread (set by the case around its
// launch sequences, graph captures included).
void set_pdl(bool on);
bool pdl_enabled();

// Opts kernel k into `bytes` of dynamic shared memory on the current device.
// The attribute belongs to the device's context, so it is set once per
// device; `done` (one per kernel, at the call site) records the devices.
template <typename... KArgs>
inline void smem_attr(void (*k)(KArgs...), int bytes, std::atomic<unsigned long long> &done) {
  int dev = 0;
  cudaGetDevice(&dev);
  const unsigned long long bit = 1ull << (dev & 63);
  if (done.load(std::memory_order_acquire) & bit) return;
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  done.fetch_or(bit, std::memory_order_acq_rel);
}

template <typename... KArgs, typename... Args>
inline void launch_k(void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, Args &&...args) {
  if (!pdl_enabled()) {
    k<<<grid, block, smem, st>>>(std::forward<Args>(args)...);
    return;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, k, std::forward<Args>(args)...);
}

}  // namespace frk
