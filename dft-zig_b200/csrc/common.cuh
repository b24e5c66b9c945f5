// Shared types and helpers for libdftcuda (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>
#include <string>

#include "../../include/dftcuda.h"

namespace dftcuda {

// Interleaved complex {re, im}: the reference's math.Complex layout
// (src/features/math/complex.zig:3-6) for double; float2 for the FP32 path.
template <typename T> struct cplx_t;
template <> struct cplx_t<double> { using type = double2; };
template <> struct cplx_t<float> { using type = float2; };
template <typename T> using cplx = typename cplx_t<T>::type;

template <typename C> __host__ __device__ __forceinline__ C mk(double re, double im);
template <> __host__ __device__ __forceinline__ double2 mk<double2>(double re, double im) { return make_double2(re, im); }
template <> __host__ __device__ __forceinline__ float2 mk<float2>(double re, double im) {
  return make_float2((float)re, (float)im);
}

template <typename C> __host__ __device__ __forceinline__ C cadd(C a, C b) { C r; r.x = a.x + b.x; r.y = a.y + b.y; return r; }
template <typename C> __host__ __device__ __forceinline__ C csub(C a, C b) { C r; r.x = a.x - b.x; r.y = a.y - b.y; return r; }
template <typename C> __host__ __device__ __forceinline__ C cmul(C a, C b) {
  C r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}
template <typename C, typename S> __host__ __device__ __forceinline__ C cscale(C a, S s) { C r; r.x = a.x * s; r.y = a.y * s; return r; }
template <typename C> __host__ __device__ __forceinline__ C cconj(C a) { C r; r.x = a.x; r.y = -a.y; return r; }
// sigma * i * a, sigma = +1 or -1
template <typename C, typename S> __host__ __device__ __forceinline__ C cmuli(C a, S sigma) {
  C r; r.x = -sigma * a.y; r.y = sigma * a.x; return r;
}

struct Error {
  int status;
  std::string msg;
};

void set_last_error(int status, const std::string& msg);

#define DFT_CUDA_TRY(expr)                                                                    \
  do {                                                                                        \
    cudaError_t e__ = (expr);                                                                 \
    if (e__ != cudaSuccess) {                                                                 \
      ::dftcuda::set_last_error(DFTCUDA_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e__)); \
      return DFTCUDA_ERR_CUDA;                                                                \
    }                                                                                         \
  } while (0)

#define DFT_TRY(expr)         \
  do {                        \
    int s__ = (expr);         \
    if (s__ != DFTCUDA_OK) return s__; \
  } while (0)

inline int fail(int status, const std::string& msg) {
  set_last_error(status, msg);
  return status;
}

inline unsigned ceil_div(size_t a, size_t b) { return (unsigned)((a + b - 1) / b); }

// Count of kernels this library has launched (all contexts); every launch site calls count_launch().
uint64_t launches_total();
void count_launch(int n = 1);

// Every device allocation of the library goes through dev_malloc.  dftcuda_debug_fail_alloc(k) makes
// the k-th following one fail once, as cudaMalloc does when the device is out of memory, so that
// tests can check that each entry point reports DFTCUDA_ERR_OUT_OF_MEMORY and keeps its context usable.
bool alloc_should_fail();
template <typename T> inline cudaError_t dev_malloc(T** p, size_t bytes) {
  if (alloc_should_fail()) {
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  return cudaMalloc(reinterpret_cast<void**>(p), bytes);
}

// True when p is device (or managed) memory, false for host memory (pageable or pinned).
bool is_device_pointer(const void* p);

// cudaFuncSetAttribute(MaxDynamicSharedMemorySize) once per (device, kernel, size), under a lock: the
// attribute belongs to the device, so a process that drives several GPUs sets it on each of them.
int ensure_max_dynamic_smem(const void* kernel, int bytes);

// Failure injection for the bounded device waits (dftcuda_debug_set_wait_limits): polls > 0 replaces
// the grid barrier's poll budget; unreachable raises every barrier target by one arrival no block makes.
struct WaitLimits {
  long polls;
  bool unreachable;
};
WaitLimits wait_limits();
// Value a timed-out grid barrier writes to its status flag (the Jacobi solver writes 1 for "not
// converged"), so callers can tell a timeout from a numerical failure.
constexpr int kBarrierTimeoutFlag = 2;

// Makes `dev` the current device for the guard's lifetime (no-op when it already is, or dev < 0)
// and restores the caller's device afterwards.  status is DFTCUDA_OK unless the switch failed.
struct DeviceGuard {
  int prev = -1;
  bool switched = false;
  int status = DFTCUDA_OK;
  explicit DeviceGuard(int dev);
  ~DeviceGuard();
  DeviceGuard(const DeviceGuard&) = delete;
  DeviceGuard& operator=(const DeviceGuard&) = delete;
};

}  // namespace dftcuda
