// noalloc.cu -- ufvm_solve_sor_noalloc: one symmetric natural-order Gauss-Seidel sweep
// (solve/cfdSolveSOR.m:13-29, the same operation as ufvm_solve_sor) that allocates no device
// memory.
//
// Why it exists: some callers cannot allocate device memory at the moment they call the
// smoother. A MATLAB MEX gateway that runs inside a caller-owned device-memory budget, a host
// application whose device memory is handed out only by its own pool allocator after start-up,
// or code that must not trigger the implicit device synchronisation of cudaMalloc/cudaFree in the
// middle of its own pipelined work. ufvm_solve_sor builds its level schedules in freshly allocated
// buffers; this variant keeps all of its scratch (row levels, level-sorted row lists, level
// offsets, counters) in one fixed array compiled into the library, so a call allocates nothing.
//
// Limits and sharing rules:
//   * at most kNaMaxRows rows (262,144, a 64^3 mesh); larger systems are rejected with
//     UFVM_E_INVALID before any device work;
//   * the scratch array is shared by every call in the process on a device and keeps what the
//     previous call left in it; each call clears the parts that must start at zero. Calls whose
//     device work overlaps (different streams, or different host threads) race on the scratch
//     and give wrong results: serialise them;
//   * the matrix must be structurally symmetric (a face couples both of its cells, so every
//     finite-volume matrix is): the dependency levels come from each row's lower neighbours,
//     which orders the sweep correctly only when a row's upper neighbours list it in turn;
//     ufvm_solve_sor makes the same assumption;
//   * every call reads the level schedule's size back to the host and synchronises its stream
//     (it builds the schedule on the device, then sizes the launches from it), so it cannot be
//     captured into a CUDA graph; the first call on a device also looks up the scratch array's
//     device address with cudaGetSymbolAddress (with that device current) and caches it.
//
// The sweep runs one kernel launch per dependency level (forward levels, then backward levels),
// so every row sees exactly the neighbour values the sequential sweep would see, and each row
// evaluates v = bc - sum(anb * x) in cconn order, then x = v / ac: the results are bit-identical
// to ufvm_solve_sor's.
#include <mutex>

#include "common.cuh"

namespace ufvm {
namespace {

constexpr int kNaMaxRows = 262144;
constexpr int kNaMaxDevices = 64;

// Scratch layout (int32 words): lvl[max], rows[max], start[max + 2], cursor[max + 2],
// flags[64] (0: changed, 1: max level, 2: widest level).
constexpr size_t kNaLvl = 0;
constexpr size_t kNaRows = kNaLvl + kNaMaxRows;
constexpr size_t kNaStart = kNaRows + kNaMaxRows;
constexpr size_t kNaCursor = kNaStart + kNaMaxRows + 2;
constexpr size_t kNaFlags = kNaCursor + kNaMaxRows + 2;
constexpr size_t kNaWords = kNaFlags + 64;

// About 4 MiB of device memory, reserved when the library's device code is loaded.
static __device__ __align__(256) int g_na_scratch[kNaWords];

std::mutex g_na_mutex;
int* g_na_ptr[kNaMaxDevices] = {nullptr};

// Device address of the scratch array on the current device (looked up once per device).
int na_scratch(int** out) {
  int dev = 0;
  UFVM_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNaMaxDevices) {
    set_error("ufvm_solve_sor_noalloc: device index out of range");
    return UFVM_E_INVALID;
  }
  std::lock_guard<std::mutex> lock(g_na_mutex);
  if (!g_na_ptr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_na_scratch);
    if (e != cudaSuccess || !p) {
      set_error(std::string("ufvm_solve_sor_noalloc: cudaGetSymbolAddress of the scratch array failed: ") +
                cudaGetErrorString(e));
      return UFVM_E_CUDA;
    }
    g_na_ptr[dev] = static_cast<int*>(p);
  }
  *out = g_na_ptr[dev];
  return UFVM_OK;
}

// Longest-path levels: fwd lvl[i] = 1 + max lvl[j] over lower neighbours j < i (0 if none),
// bwd the same over upper neighbours. Relaxed to the fixed point from lvl = 0.
template <bool FWD>
__global__ void k_na_level(int n, const int* __restrict__ rp, const int* __restrict__ col, int* lvl, int* flags) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int m = 0;
  for (int k = rp[i]; k < rp[i + 1]; ++k) {
    const int j = col[k];
    if (FWD ? (j < i) : (j > i)) m = max(m, __ldcg(lvl + j) + 1);
  }
  if (m != __ldcg(lvl + i)) {
    __stcg(lvl + i, m);
    flags[0] = 1;
  }
}

__global__ void k_na_count(int n, const int* __restrict__ lvl, int* cnt, int* flags) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  atomicAdd(cnt + lvl[i], 1);
  atomicMax(flags + 1, lvl[i]);
}

// One block: exclusive scan of the level counts into start (and cursor), widest level into
// flags[2]. nl = number of levels.
__global__ void __launch_bounds__(1024) k_na_scan(int nl, int* cnt_to_start, int* cursor, int* flags) {
  __shared__ int sh[1024];
  __shared__ int carry, widest;
  if (threadIdx.x == 0) { carry = 0; widest = 0; }
  __syncthreads();
  for (int base = 0; base < nl; base += 1024) {
    const int i = base + threadIdx.x;
    const int v = i < nl ? cnt_to_start[i] : 0;
    if (v > 0) atomicMax(&widest, v);
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {  // inclusive Hillis-Steele scan
      const int t = threadIdx.x >= off ? sh[threadIdx.x - off] : 0;
      __syncthreads();
      sh[threadIdx.x] += t;
      __syncthreads();
    }
    const int excl = carry + sh[threadIdx.x] - v;
    if (i < nl) { cnt_to_start[i] = excl; cursor[i] = excl; }
    __syncthreads();
    if (threadIdx.x == 1023) carry += sh[1023];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    cnt_to_start[nl] = carry;
    flags[2] = widest;
  }
}

__global__ void k_na_fill(int n, const int* __restrict__ lvl, int* cursor, int* rows) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  rows[atomicAdd(cursor + lvl[i], 1)] = i;
}

// The rows of one level, each with the operation order of the sequential sweep.
__global__ void k_na_gs_level(int l, const int* __restrict__ start, const int* __restrict__ rows,
                              const int* __restrict__ rp, const int* __restrict__ col, const double* __restrict__ ac,
                              const double* __restrict__ anb, const double* __restrict__ bc, double* x) {
  const int s = start[l], e = start[l + 1];
  const int idx = s + blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= e) return;
  const int i = rows[idx];
  double v = bc[i];
  for (int k = rp[i]; k < rp[i + 1]; ++k) v = v - anb[k] * x[col[k]];
  x[i] = v / ac[i];
}

template <bool FWD>
int na_half_sweep(int n, const int* rp, const int* col, const double* ac, const double* anb, const double* bc,
                  double* x, int* scratch, cudaStream_t st) {
  int* lvl = scratch + kNaLvl;
  int* rows = scratch + kNaRows;
  int* start = scratch + kNaStart;
  int* cursor = scratch + kNaCursor;
  int* flags = scratch + kNaFlags;
  // what a previous call left behind is cleared first
  UFVM_CUDA(cudaMemsetAsync(lvl, 0, (size_t)n * sizeof(int), st));
  UFVM_CUDA(cudaMemsetAsync(flags, 0, 64 * sizeof(int), st));
  int changed = 1, passes = 0;
  while (changed) {
    UFVM_CUDA(cudaMemsetAsync(flags, 0, sizeof(int), st));
    for (int k = 0; k < 8; ++k) k_na_level<FWD><<<nblocks(n), kBlock, 0, st>>>(n, rp, col, lvl, flags);
    UFVM_LAUNCH_CHECK();
    UFVM_CUDA(cudaMemcpyAsync(&changed, flags, sizeof(int), cudaMemcpyDeviceToHost, st));
    UFVM_CUDA(cudaStreamSynchronize(st));
    passes += 8;
    if (passes > n + 16) {
      set_error("ufvm_solve_sor_noalloc: level schedule did not converge");
      return UFVM_E_INVALID;
    }
  }
  UFVM_CUDA(cudaMemsetAsync(start, 0, (size_t)(n + 2) * sizeof(int), st));
  UFVM_CUDA(cudaMemsetAsync(flags + 1, 0, 2 * sizeof(int), st));
  k_na_count<<<nblocks(n), kBlock, 0, st>>>(n, lvl, start, flags);
  UFVM_LAUNCH_CHECK();
  int maxl = 0;
  UFVM_CUDA(cudaMemcpyAsync(&maxl, flags + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
  UFVM_CUDA(cudaStreamSynchronize(st));
  const int nl = maxl + 1;
  k_na_scan<<<1, 1024, 0, st>>>(nl, start, cursor, flags);
  k_na_fill<<<nblocks(n), kBlock, 0, st>>>(n, lvl, cursor, rows);
  UFVM_LAUNCH_CHECK();
  int widest = 0;
  UFVM_CUDA(cudaMemcpyAsync(&widest, flags + 2, sizeof(int), cudaMemcpyDeviceToHost, st));
  UFVM_CUDA(cudaStreamSynchronize(st));
  const int nb = std::max(1, nblocks(widest));
  for (int l = 0; l < nl; ++l) k_na_gs_level<<<nb, kBlock, 0, st>>>(l, start, rows, rp, col, ac, anb, bc, x);
  UFVM_LAUNCH_CHECK();
  return UFVM_OK;
}

}  // namespace
}  // namespace ufvm

using namespace ufvm;

extern "C" int ufvm_solve_sor_noalloc(int32_t n, const int32_t* rowptr, const int32_t* col, const double* ac,
                                      const double* anb, const double* bc, double* dphi, void* stream) {
  if (n <= 0 || !rowptr || !col || !ac || !anb || !bc || !dphi) {
    set_error("ufvm_solve_sor_noalloc: bad argument");
    return UFVM_E_INVALID;
  }
  if (n > kNaMaxRows) {
    set_error("ufvm_solve_sor_noalloc: " + std::to_string(n) + " rows exceed the fixed scratch limit of " +
              std::to_string(kNaMaxRows) + " rows; use ufvm_solve_sor");
    return UFVM_E_INVALID;
  }
  int* scratch = nullptr;
  UFVM_CHECK(na_scratch(&scratch));
  cudaStream_t st = (cudaStream_t)stream;
  UFVM_CHECK(na_half_sweep<true>(n, rowptr, col, ac, anb, bc, dphi, scratch, st));
  UFVM_CHECK(na_half_sweep<false>(n, rowptr, col, ac, anb, bc, dphi, scratch, st));
  UFVM_CUDA(cudaStreamSynchronize(st));
  return UFVM_OK;
}
