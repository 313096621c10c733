// common.cuh -- shared device helpers for libufvm (sm_100a).
//
// Floating-point contract: every FP64 kernel in this library is compiled with
// --fmad=false and evaluates each expression in the left-to-right order of the MATLAB
// source it restates, so results are reproducible bit for bit against a sequential
// evaluation of the same expression. Reductions over many rows (sums of |r|, r^2) use a
// fixed two-stage tree and are deterministic run to run.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <string>
#include <vector>

#include "../../include/ufvm.h"

namespace ufvm {

constexpr int kBlock = 256;

// error state (thread-local message for ufvm_last_error)
void set_error(const std::string& msg);
const char* get_error();

#define UFVM_CUDA(call)                                                                   \
  do {                                                                                    \
    cudaError_t _e = (call);                                                              \
    if (_e != cudaSuccess) {                                                              \
      ::ufvm::set_error(std::string(#call) + ": " + cudaGetErrorString(_e));             \
      return UFVM_E_CUDA;                                                                 \
    }                                                                                     \
  } while (0)

#define UFVM_CHECK(expr)                 \
  do {                                   \
    int _s = (expr);                     \
    if (_s != UFVM_OK) return _s;        \
  } while (0)

#define UFVM_LAUNCH_CHECK() UFVM_CUDA(cudaGetLastError())

inline int nblocks(long long n, int bs = kBlock) { return (int)((n + bs - 1) / bs); }

__device__ __forceinline__ double dmax(double a, double b) { return (a < b) ? b : a; }
__device__ __forceinline__ double dmin(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double dot3(double a0, double a1, double a2, double b0, double b1, double b2) {
  return (a0 * b0 + a1 * b1) + a2 * b2;
}

// Bytes of device memory this host thread holds through dalloc (freed by dfree). The batched
// service takes differences of it around each case's allocations to learn the case's HBM
// footprint.
inline thread_local long long t_dev_bytes = 0;
// Host time (ms) this thread has spent inside device allocation and free calls.
inline thread_local double t_alloc_ms = 0.0;

// Stream-ordered allocation. A thread inside an AllocStreamScope allocates from the device's
// default memory pool on the scope's stream (cudaMallocAsync) and frees there (cudaFreeAsync):
// neither call waits for the device, while cudaFree waits for the whole device and cudaMalloc
// goes through the driver's allocator. The batched service builds hundreds of cases' meshes and
// AMG hierarchies on several host threads at once (hundreds of allocations per case), so it
// allocates this way; everything else uses cudaMalloc. An array remembers how it was allocated.
// An allocation is ordered on the scope's stream: work on another stream that uses it first
// waits for that stream (the service's builders synchronise their streams before the service
// stream uses what they made).
inline thread_local cudaStream_t t_alloc_stream = nullptr;
struct AllocStreamScope {
  cudaStream_t prev;
  explicit AllocStreamScope(cudaStream_t s) : prev(t_alloc_stream) { t_alloc_stream = s; }
  ~AllocStreamScope() { t_alloc_stream = prev; }
  AllocStreamScope(const AllocStreamScope&) = delete;
  AllocStreamScope& operator=(const AllocStreamScope&) = delete;
};
// The scope's stream, or null when this thread should use cudaMalloc (no scope, or the stream is
// being captured into a graph, where an asynchronous allocation would become a graph node).
inline cudaStream_t alloc_stream_now() {
  if (!t_alloc_stream) return nullptr;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(t_alloc_stream, &cs) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return cs == cudaStreamCaptureStatusNone ? t_alloc_stream : nullptr;
}
double host_ms_now();

// Device array owned by a case; freed by its owner.
template <typename T>
struct DArr {
  T* p = nullptr;
  size_t n = 0;
  bool async = false;  // allocated by cudaMallocAsync (stream-ordered), else cudaMalloc
};

template <typename T>
void dfree(DArr<T>& a) {
  if (a.p) {
    const double t0 = host_ms_now();
    if (!a.async) {
      cudaFree(a.p);
    } else if (cudaStream_t s = alloc_stream_now()) {
      cudaFreeAsync(a.p, s);
    } else {
      // outside a scope nothing orders the free after the array's last use: wait for it
      cudaDeviceSynchronize();
      cudaFree(a.p);
    }
    t_alloc_ms += host_ms_now() - t0;
    t_dev_bytes -= (long long)(a.n * sizeof(T));
  }
  a.p = nullptr;
  a.n = 0;
  a.async = false;
}

template <typename T>
int dalloc(DArr<T>& a, size_t n) {
  if (a.p && a.n >= n) return UFVM_OK;
  dfree(a);
  if (n == 0) n = 1;
  const double t0 = host_ms_now();
  cudaStream_t s = alloc_stream_now();
  cudaError_t e = s ? cudaMallocAsync((void**)&a.p, n * sizeof(T), s) : cudaMalloc((void**)&a.p, n * sizeof(T));
  t_alloc_ms += host_ms_now() - t0;
  if (e != cudaSuccess) {
    a.p = nullptr;
    cudaGetLastError();  // an out-of-memory report is not sticky: clear it for later checks
    set_error(std::string(s ? "cudaMallocAsync: " : "cudaMalloc: ") + cudaGetErrorString(e));
    return UFVM_E_OOM;
  }
  a.n = n;
  a.async = s != nullptr;
  t_dev_bytes += (long long)(n * sizeof(T));
  return UFVM_OK;
}

// Programmatic dependent launch. A kernel launched with programmatic stream serialization may
// start once every block of the kernel before it has executed pdl_trigger; pdl_wait then blocks
// until that kernel has completed and its writes are visible. Without the launch attribute both
// are no-ops. A kernel that waits before touching memory any earlier kernel writes behaves as
// an ordinary launch, minus the launch gap.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// ---- block reductions (fixed shape => deterministic) ----
__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = dmax(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_min(double v) {
  for (int o = 16; o > 0; o >>= 1) v = dmin(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}

// reduce over the block; result valid in thread 0. sh must hold blockDim/32 doubles.
template <int OP>  // 0 sum, 1 max, 2 min
__device__ __forceinline__ double block_reduce(double v, double* sh) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  v = OP == 0 ? warp_sum(v) : (OP == 1 ? warp_max(v) : warp_min(v));
  __syncthreads();
  if (lane == 0) sh[w] = v;
  __syncthreads();
  const int nw = blockDim.x >> 5;
  if (w == 0) {
    double x = lane < nw ? sh[lane] : (OP == 0 ? 0.0 : (OP == 1 ? -INFINITY : INFINITY));
    x = OP == 0 ? warp_sum(x) : (OP == 1 ? warp_max(x) : warp_min(x));
    v = x;
  }
  return v;
}

// Grid-wide barrier for cooperatively launched kernels (all blocks co-resident).
// The wait is bounded; on timeout the error flag is raised and the caller must return.
struct GridBarrier {
  unsigned int* count;  // zero-initialised
  unsigned int* gen;    // generation counter
  int* err;             // set to 1 on timeout
};

__device__ __forceinline__ bool grid_sync(const GridBarrier& b, unsigned int& local_gen) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    bool ok = true;
    const unsigned int nb = gridDim.x * gridDim.y * gridDim.z;
    __threadfence();
    const unsigned int my = local_gen;
    if (atomicAdd(b.count, 1u) == nb - 1) {
      *b.count = 0;
      __threadfence();
      atomicAdd(b.gen, 1u);
    } else {
      long long spins = 0;
      while (((volatile unsigned int*)b.gen)[0] == my) {
        if (++spins > (1ll << 26)) {  // bounded: raise the flag instead of waiting forever
          atomicExch(b.err, 1);
          ok = false;
          break;
        }
        __nanosleep(32);
      }
    }
    __threadfence();
    s_ok = ok && (((volatile int*)b.err)[0] == 0);
  }
  local_gen += 1;
  __syncthreads();
  return s_ok != 0;
}

// Thread 0 of each block reads the barrier generation once at kernel start.
__device__ __forceinline__ unsigned int grid_gen0(const GridBarrier& b) {
  __shared__ unsigned int s_gen;
  if (threadIdx.x == 0) s_gen = ((volatile unsigned int*)b.gen)[0];
  __syncthreads();
  return s_gen;
}

}  // namespace ufvm
