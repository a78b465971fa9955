// Shared device/host helpers for the btorch_b200 kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>
#include <vector>

#include "../../include/btorch_b200.h"

// Set the thread-local error text and return `status` (defined in layout.cpp).
extern "C" int bt_set_error(int status, const char* fmt, ...);

#define BT_CHECK_ARG(cond, ...)                                  \
  do {                                                           \
    if (!(cond)) return bt_set_error(BT_ERR_INVALID, __VA_ARGS__); \
  } while (0)

// Report a failed launch (configuration errors surface here, asynchronous
// faults surface at the caller's next synchronisation).
#define BT_CHECK_LAUNCH(what)                                              \
  do {                                                                     \
    cudaError_t err_ = cudaGetLastError();                                 \
    if (err_ != cudaSuccess)                                               \
      return bt_set_error(BT_ERR_CUDA, "%s: %s", what, cudaGetErrorString(err_)); \
  } while (0)

namespace bt {

constexpr int kWarp = 32;
constexpr uint32_t kIdMask = (1u << BT_BIN_SHIFT) - 1u;

__host__ __device__ inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

// Single-rounding IEEE fp32 operations.  The intrinsics are never fused into
// FMA by the compiler, so the device evaluates exactly the rounding sequence of
// the reference's eager CPU operators (one rounding per torch op).
__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }

__device__ __forceinline__ float ld(const bt_param& p, int64_t i) { return __ldg(p.ptr + i * p.stride); }

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }

// L2 eviction-priority hints (PTX createpolicy + .L2::cache_hint, sm_80+).
// Data read once per step (edge lists, the step's input current) is loaded
// evict-first so that it does not push the small, reused accumulators out of
// L2; reductions into those accumulators are issued evict-last.
__device__ __forceinline__ uint64_t l2_evict_first() {
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t l2_evict_last() {
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
// Read-only (non-coherent) loads with an L2 policy; not volatile, so the
// compiler may batch them ahead of their uses.
__device__ __forceinline__ uint4 ld_nc_u4(const void* ptr, uint64_t pol) {
  uint4 v;
  asm("ld.global.nc.L2::cache_hint.v4.u32 {%0, %1, %2, %3}, [%4], %5;"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "l"(ptr), "l"(pol));
  return v;
}
__device__ __forceinline__ uint2 ld_nc_u2(const void* ptr, uint64_t pol) {
  uint2 v;
  asm("ld.global.nc.L2::cache_hint.v2.u32 {%0, %1}, [%2], %3;" : "=r"(v.x), "=r"(v.y) : "l"(ptr), "l"(pol));
  return v;
}
__device__ __forceinline__ uint32_t ld_nc_u32(const void* ptr, uint64_t pol) {
  uint32_t v;
  asm("ld.global.nc.L2::cache_hint.u32 %0, [%1], %2;" : "=r"(v) : "l"(ptr), "l"(pol));
  return v;
}
__device__ __forceinline__ float ld_nc_f32(const float* ptr, uint64_t pol) {
  float v;
  asm("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(ptr), "l"(pol));
  return v;
}
// Coherent fp32 load / store with an L2 policy.
__device__ __forceinline__ float ld_f32(const float* ptr, uint64_t pol) {
  float v;
  asm volatile("ld.global.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(ptr), "l"(pol));
  return v;
}
__device__ __forceinline__ void st_f32(float* ptr, float v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.f32 [%0], %1, %2;" ::"l"(ptr), "f"(v), "l"(pol) : "memory");
}
// fp32 reduction (no return value) with an L2 policy.
__device__ __forceinline__ void red_add_f32(float* ptr, float v, uint64_t pol) {
  // no "memory" clobber: nothing in the issuing kernel reads the target, so
  // independent loads may be scheduled across the reduction
  asm volatile("red.global.add.L2::cache_hint.f32 [%0], %1, %2;" ::"l"(ptr), "f"(v), "l"(pol));
}

// Launch set-ups already checked (kernel, device, dynamic shared memory,
// blocks): the attribute calls and occupancy queries of a persistent launch
// run once per set-up, not on every call -- they cost the host far more
// than a short launch takes on the device.
struct LaunchSetup {
  const void* kern;
  int dev;
  size_t smem;
  int blocks;
};
inline std::mutex& launch_setup_mutex() {
  static std::mutex m;
  return m;
}
inline std::vector<LaunchSetup>& launch_setups() {
  static std::vector<LaunchSetup> v;
  return v;
}
inline bool launch_setup_known(const void* kern, int dev, size_t smem, int blocks) {
  std::lock_guard<std::mutex> g(launch_setup_mutex());
  for (const LaunchSetup& e : launch_setups())
    if (e.kern == kern && e.dev == dev && e.smem == smem && e.blocks == blocks) return true;
  return false;
}
// The dynamic shared memory to allow a kernel: at least `smem` and never less
// than a set-up already checked on this device asked for (the attribute is
// the kernel's, shared by all its set-ups).
inline size_t launch_smem_allow(const void* kern, int dev, size_t smem) {
  std::lock_guard<std::mutex> g(launch_setup_mutex());
  for (const LaunchSetup& e : launch_setups())
    if (e.kern == kern && e.dev == dev && e.smem > smem) smem = e.smem;
  return smem;
}
inline void launch_setup_add(const void* kern, int dev, size_t smem, int blocks) {
  std::lock_guard<std::mutex> g(launch_setup_mutex());
  launch_setups().push_back(LaunchSetup{kern, dev, smem, blocks});
}

}  // namespace bt
