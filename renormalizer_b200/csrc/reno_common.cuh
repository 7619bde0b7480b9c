// Shared definitions for the sweep-engine kernels (sm_100a).
//
// Every C-ABI entry point returns an int status (RENO_OK == 0).  Errors are
// recorded in the context (reno_last_error) so the Python shim can raise the
// exception type the reference raises for the same condition.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>
#include <atomic>
#include "../../include/reno_b200.h"

struct reno_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  int num_sms = 148;
  std::string last_error;
  // pinned host slots for scalars read back by the host (Krylov alpha/beta ...)
  double* host_scalars = nullptr;
};

namespace reno {

// Wall-clock limit of every bounded device wait (pipeline mbarriers of the
// tensor-core GEMM, grid barriers of the eigensolver reduction), passed to
// the kernels at launch; reno_set_wait_limit_ns changes it.
inline std::atomic<unsigned long long> g_wait_ns{2000000000ull};
// Test hooks of the failure path (reno_test_skip_arrival), consumed by the
// next launch of the kernel they name: CTA 0 of that launch leaves one wait
// without its arrival, so the bounded wait runs out and the kernel returns
// with its error status set.  -1 = none.
inline std::atomic<int> g_skip_split_stage{-1};
// K elements per promoted accumulation chunk of the split GEMM (0 = off),
// reno_set_split_accumulation_chunk
inline std::atomic<int> g_split_chunk_k{0};
inline std::atomic<int> g_skip_hetrd_column{-1};

// every kernel launch of the library bumps this (host-side, per process)
inline std::atomic<long long> g_launches{0};
inline void count_launch(long long n = 1) { g_launches.fetch_add(n, std::memory_order_relaxed); }

inline int set_error(reno_ctx* ctx, int code, const std::string& msg) {
  if (ctx) ctx->last_error = msg;
  return code;
}

inline int check_cuda(reno_ctx* ctx, cudaError_t e, const char* what) {
  if (e == cudaSuccess) return RENO_OK;
  std::string m = std::string(what) + ": " + cudaGetErrorString(e);
  return set_error(ctx, e == cudaErrorMemoryAllocation ? RENO_ERR_OOM : RENO_ERR_CUDA, m);
}

#define RENO_LAUNCH_CHECK(ctx, what)                                     \
  do {                                                                   \
    cudaError_t _e = cudaGetLastError();                                 \
    if (_e != cudaSuccess) return ::reno::check_cuda((ctx), _e, (what)); \
  } while (0)

__host__ __device__ inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

// Opt a kernel into `bytes` of dynamic shared memory once per device:
// function attributes belong to each device's context, so a process that
// drives several GPUs sets them on each (bit d of `done` = device d).
template <typename Kernel>
inline cudaError_t smem_optin_once(Kernel* kernel, int bytes, std::atomic<unsigned long long>& done) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const unsigned long long bit = (dev >= 0 && dev < 64) ? (1ull << dev) : 0ull;
  if (bit && (done.load(std::memory_order_acquire) & bit)) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess && bit) done.fetch_or(bit, std::memory_order_release);
  return e;
}

// SM count of the current device, read once per device (entry d of a
// per-process table; 0 = not read yet) and safe under concurrent first calls.
inline int sm_count_current_device() {
  static std::atomic<int> table[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 148;
  if (dev < 0 || dev >= 64) {
    int n = 0;
    return (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && n > 0) ? n : 148;
  }
  int n = table[dev].load(std::memory_order_relaxed);
  if (n > 0) return n;
  if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
  table[dev].store(n, std::memory_order_relaxed);
  return n;
}

}  // namespace reno
