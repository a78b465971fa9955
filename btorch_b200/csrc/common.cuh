// Shared device/host helpers for the btorch_b200 kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

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

}  // namespace bt
