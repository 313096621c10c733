// linsolve.cu -- residual, smoothers and grid transfers of uFVM's linear solve.
//
//   residual      compute/cfdComputeResidualsArray.m:9-17
//   GS ('SOR')    solve/cfdSolveSOR.m:13-29   (natural order, level scheduled: identical
//                 arithmetic to the sequential sweep because a row's lower neighbours sit in
//                 earlier levels and its upper neighbours in later ones)
//   DILU ('ILU')  solve/cfdFactorizeILU.m:5-47, solve/cfdSolveILU.m:18-93 (level scheduled)
//   MCGS          multicolour symmetric GS (greedy first-fit colouring in natural order)
//   smoother loop solve/cfdSolveAlgebraicSystem.m:11-66
//   restriction   solve/AMG/cfdUpdateRHS.m:10-17, prolongation cfdCorrectFinerLevelSolution.m:11-14
//
// Roofline: residual / one GS half-sweep are HBM-bound; algorithmic bytes per row =
// 8 (ac) + 8 (bc) + 8 (x) + 8 (r or x write) + 4 (rowptr) + nnz_row * (8 anb + 4 col).
#include "linsolve.cuh"

namespace ufvm {

int LinCtx::ensure(int n) {
  const int nb = nblocks(n) + 2;
  UFVM_CHECK(dalloc(part, std::max(nb, 64) * 2));
  UFVM_CHECK(dalloc(red, 16));
  UFVM_CHECK(dalloc(iflag, 16));
  UFVM_CHECK(dalloc(iscan, nblocks(n, 1024) * 2 + 64));
  if (!bar.p) {
    UFVM_CHECK(dalloc(bar, 2));
    UFVM_CUDA(cudaMemsetAsync(bar.p, 0, 2 * sizeof(unsigned int), stream));
  }
  if (!berr.p) {
    UFVM_CHECK(dalloc(berr, 1));
    UFVM_CUDA(cudaMemsetAsync(berr.p, 0, sizeof(int), stream));
  }
  return UFVM_OK;
}

void LinCtx::release() {
  dfree(part); dfree(red); dfree(iflag); dfree(iscan); dfree(bar); dfree(berr);
}

// ---------------------------------------------------------------- scan (exclusive, int)
__global__ void k_scan_block(const int* __restrict__ in, int* out, int n, int* bsum) {
  __shared__ int sh[1024];
  const int base = blockIdx.x * 1024;
  for (int t = threadIdx.x; t < 1024; t += blockDim.x) sh[t] = base + t < n ? in[base + t] : 0;
  __syncthreads();
  // Hillis-Steele on 1024 entries with 1024 threads
  for (int o = 1; o < 1024; o <<= 1) {
    int v = 0;
    if (threadIdx.x >= o) v = sh[threadIdx.x - o];
    __syncthreads();
    sh[threadIdx.x] += v;
    __syncthreads();
  }
  const int incl = sh[threadIdx.x];
  const int x = base + threadIdx.x < n ? in[base + threadIdx.x] : 0;
  if (base + threadIdx.x < n) out[base + threadIdx.x] = incl - x;
  if (threadIdx.x == 1023) bsum[blockIdx.x] = incl;
}

__global__ void k_scan_add(int* out, int n, const int* __restrict__ boff) {
  const int i = blockIdx.x * 1024 + threadIdx.x;
  if (i < n) out[i] += boff[blockIdx.x];
}

static int scan_rec(LinCtx& c, const int* in, int* out, int n, int* tmp, size_t tmpcap) {
  const int nb = nblocks(n, 1024);
  if ((size_t)(2 * nb + 2) > tmpcap) { set_error("scan scratch too small"); return UFVM_E_INVALID; }
  int* bsum = tmp;
  int* boff = tmp + nb;
  k_scan_block<<<nb, 1024, 0, c.stream>>>(in, out, n, bsum);
  UFVM_LAUNCH_CHECK();
  if (nb == 1) return UFVM_OK;
  UFVM_CHECK(scan_rec(c, bsum, boff, nb, tmp + 2 * nb, tmpcap - 2 * nb));
  k_scan_add<<<nb, 1024, 0, c.stream>>>(out, n, boff);
  UFVM_LAUNCH_CHECK();
  return UFVM_OK;
}

__global__ void k_scan_total(const int* __restrict__ in, const int* __restrict__ out, int n, int* total_slot) {
  *total_slot = n > 0 ? out[n - 1] + in[n - 1] : 0;
}

// out has n + 1 entries; out[n] = total.
int scan_exclusive(LinCtx& c, const int* in, int* out, int n, int* total_host) {
  size_t need = 0;
  for (int m = n; m > 1; m = nblocks(m, 1024)) need += 2 * (size_t)nblocks(m, 1024) + 2;
  need += 8;
  UFVM_CHECK(dalloc(c.iscan, std::max(need, c.iscan.n)));
  if (n > 0) UFVM_CHECK(scan_rec(c, in, out, n, c.iscan.p, c.iscan.n));
  k_scan_total<<<1, 1, 0, c.stream>>>(in, out, n, out + n);
  UFVM_LAUNCH_CHECK();
  if (total_host) {
    UFVM_CUDA(cudaMemcpyAsync(total_host, out + n, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    UFVM_CUDA(cudaStreamSynchronize(c.stream));
  }
  return UFVM_OK;
}

// ---------------------------------------------------------------- residual
// One row per thread. Everything a row needs apart from the neighbour values (its row
// pointers, bc, ac, x_i) is loaded at once, then its entries kResChunk at a time (the L1
// serves the warp's neighbouring rows from the same sectors), then the neighbour values:
// three dependent memory round trips per row. v = bc - ac x_i, then v = v - anb x_j in cconn
// order, with each product rounded before the subtraction as in the sequential loop.
constexpr int kResChunk = 4;
constexpr int kResBlock = 128;

__device__ __forceinline__ double row_residual(int i, const int* __restrict__ rp, const int* __restrict__ col,
                                               const double* __restrict__ ac, const double* __restrict__ anb,
                                               const double* __restrict__ bc, const double* __restrict__ x) {
  const int k0 = rp[i], k1 = rp[i + 1];
  double v = bc[i] - ac[i] * x[i];
  for (int k = k0; k < k1; k += kResChunk) {
    double p[kResChunk];
#pragma unroll
    for (int t = 0; t < kResChunk; ++t) p[t] = k + t < k1 ? anb[k + t] * x[col[k + t]] : 0.0;
#pragma unroll
    for (int t = 0; t < kResChunk; ++t)
      if (k + t < k1) v = v - p[t];
  }
  return v;
}

__global__ void __launch_bounds__(kResBlock) k_residual(int n, const int* __restrict__ rp,
                                                        const int* __restrict__ col, const double* __restrict__ ac,
                                                        const double* __restrict__ anb,
                                                        const double* __restrict__ bc,
                                                        const double* __restrict__ x, double* __restrict__ r) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) r[i] = row_residual(i, rp, col, ac, anb, bc, x);
}

// sum_i |r_i| : block partials (stage 1)
__global__ void __launch_bounds__(kBlock) k_sumabs_res(int n, const int* __restrict__ rp, const int* __restrict__ col,
                                                       const double* __restrict__ ac, const double* __restrict__ anb,
                                                       const double* __restrict__ bc, const double* __restrict__ x,
                                                       double* part) {
  __shared__ double sh[32];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double v = i < n ? fabs(row_residual(i, rp, col, ac, anb, bc, x)) : 0.0;
  v = block_reduce<0>(v, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = v;
}

// stage 2: fixed-order sum of the partials
__global__ void k_sum_partials(int np, const double* __restrict__ part, double* out) {
  __shared__ double sh[32];
  double v = 0.0;
  for (int k = threadIdx.x; k < np; k += blockDim.x) v = v + part[k];
  v = block_reduce<0>(v, sh);
  if (threadIdx.x == 0) *out = v;
}

int residual(LinCtx& c, const Level& L, const double* x, double* r) {
  k_residual<<<nblocks(L.n, kResBlock), kResBlock, 0, c.stream>>>(L.n, L.rowptr.p, L.col.p, L.ac.p, L.anb.p,
                                                                   L.bc.p, x, r);
  UFVM_LAUNCH_CHECK();
  return UFVM_OK;
}

int sum_abs_residual(LinCtx& c, const Level& L, const double* x, double* out_host) {
  UFVM_CHECK(c.ensure(L.n));
  const int nb = nblocks(L.n);
  k_sumabs_res<<<nb, kBlock, 0, c.stream>>>(L.n, L.rowptr.p, L.col.p, L.ac.p, L.anb.p, L.bc.p, x, c.part.p);
  UFVM_LAUNCH_CHECK();
  k_sum_partials<<<1, 1024, 0, c.stream>>>(nb, c.part.p, c.red.p);
  UFVM_LAUNCH_CHECK();
  UFVM_CUDA(cudaMemcpyAsync(out_host, c.red.p, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  UFVM_CUDA(cudaStreamSynchronize(c.stream));
  return UFVM_OK;
}

// ---------------------------------------------------------------- level schedules
// fwd: lvl[i] = 1 + max lvl[j] over lower neighbours j < i (0 if none); bwd: upper.
template <bool FWD>
__global__ void k_level_iter(int n, const int* __restrict__ rp, const int* __restrict__ col, int* lvl, int* changed) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int m = 0;
  for (int k = rp[i]; k < rp[i + 1]; ++k) {
    const int j = col[k];
    if (FWD ? (j < i) : (j > i)) m = max(m, __ldcg(lvl + j) + 1);
  }
  if (m != __ldcg(lvl + i)) {
    __stcg(lvl + i, m);
    *changed = 1;
  }
}

__global__ void k_level_hist(int n, const int* __restrict__ lvl, int* cnt, int* maxl) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  atomicAdd(cnt + lvl[i], 1);
  atomicMax(maxl, lvl[i]);
}

__global__ void k_level_fill(int n, const int* __restrict__ lvl, int* cur, int* rows) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  rows[atomicAdd(cur + lvl[i], 1)] = i;
}

static int one_schedule(LinCtx& c, Level& L, bool fwd, DArr<int>& rows, DArr<int>& start, int& nlev) {
  const int n = L.n;
  UFVM_CHECK(dalloc(L.lvl, n));
  UFVM_CUDA(cudaMemsetAsync(L.lvl.p, 0, n * sizeof(int), c.stream));
  int changed = 1, iters = 0;
  while (changed) {
    // run a few relaxation passes between host checks
    UFVM_CUDA(cudaMemsetAsync(c.iflag.p, 0, sizeof(int), c.stream));
    for (int k = 0; k < 8; ++k) {
      if (fwd) k_level_iter<true><<<nblocks(n), kBlock, 0, c.stream>>>(n, L.rowptr.p, L.col.p, L.lvl.p, c.iflag.p);
      else k_level_iter<false><<<nblocks(n), kBlock, 0, c.stream>>>(n, L.rowptr.p, L.col.p, L.lvl.p, c.iflag.p);
    }
    UFVM_LAUNCH_CHECK();
    UFVM_CUDA(cudaMemcpyAsync(&changed, c.iflag.p, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    UFVM_CUDA(cudaStreamSynchronize(c.stream));
    iters += 8;
    if (iters > n + 16) { set_error("level schedule did not converge"); return UFVM_E_INVALID; }
  }
  // counting sort of rows by level
  DArr<int> cnt;
  UFVM_CHECK(dalloc(cnt, n + 2));
  UFVM_CUDA(cudaMemsetAsync(cnt.p, 0, (n + 2) * sizeof(int), c.stream));
  UFVM_CUDA(cudaMemsetAsync(c.iflag.p + 1, 0, sizeof(int), c.stream));
  k_level_hist<<<nblocks(n), kBlock, 0, c.stream>>>(n, L.lvl.p, cnt.p, c.iflag.p + 1);
  UFVM_LAUNCH_CHECK();
  int maxl = 0;
  UFVM_CUDA(cudaMemcpyAsync(&maxl, c.iflag.p + 1, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  UFVM_CUDA(cudaStreamSynchronize(c.stream));
  nlev = maxl + 1;
  UFVM_CHECK(dalloc(start, nlev + 1));
  UFVM_CHECK(scan_exclusive(c, cnt.p, start.p, nlev, nullptr));
  UFVM_CUDA(cudaMemcpyAsync(cnt.p, start.p, nlev * sizeof(int), cudaMemcpyDeviceToDevice, c.stream));
  UFVM_CHECK(dalloc(rows, n));
  k_level_fill<<<nblocks(n), kBlock, 0, c.stream>>>(n, L.lvl.p, cnt.p, rows.p);
  UFVM_LAUNCH_CHECK();
  // widest level (host) to size the cooperative launch
  std::vector<int> hs(nlev + 1);
  UFVM_CUDA(cudaMemcpyAsync(hs.data(), start.p, (nlev + 1) * sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  UFVM_CUDA(cudaStreamSynchronize(c.stream));
  for (int l = 0; l < nlev; ++l) L.maxw = std::max(L.maxw, hs[l + 1] - hs[l]);
  dfree(cnt);
  return UFVM_OK;
}

// tpos[k]: position of the transposed entry (j, i) for entry k = (i, j).
__global__ void k_tpos(int n, const int* __restrict__ rp, const int* __restrict__ col, int* tpos) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int k = rp[i]; k < rp[i + 1]; ++k) {
    const int j = col[k];
    int p = -1;
    for (int q = rp[j]; q < rp[j + 1]; ++q)
      if (col[q] == i) { p = q; break; }
    tpos[k] = p;
  }
}

int build_tpos(LinCtx& c, Level& L) {
  UFVM_CHECK(dalloc(L.tpos, std::max(L.nnz, 1)));
  k_tpos<<<nblocks(L.n), kBlock, 0, c.stream>>>(L.n, L.rowptr.p, L.col.p, L.tpos.p);
  UFVM_LAUNCH_CHECK();
  return UFVM_OK;
}

// lord: for each row, the CSR positions of its lower neighbours in increasing column order
// (the order in which the reference's outer loop over i1 delivers them), then -1 in the row's
// remaining slots. Built once per pattern by repeated minimum search.
__global__ void k_lower_order(int n, const int* __restrict__ rp, const int* __restrict__ col, int* lord) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int k0 = rp[i], k1 = rp[i + 1];
  int t = k0, prev = -1;
  while (true) {
    int best = 0x7fffffff, bk = -1;
    for (int k = k0; k < k1; ++k) {
      const int j = col[k];
      if (j < i && j > prev && j < best) { best = j; bk = k; }
    }
    if (bk < 0) break;
    prev = best;
    lord[t++] = bk;
  }
  for (; t < k1; ++t) lord[t] = -1;
}

int build_schedule(LinCtx& c, Level& L) {
  if (L.sched_valid) return UFVM_OK;
  UFVM_CHECK(c.ensure(L.n));
  L.maxw = 0;
  UFVM_CHECK(one_schedule(c, L, true, L.fwdRows, L.fwdStart, L.nfwd));
  UFVM_CHECK(one_schedule(c, L, false, L.bwdRows, L.bwdStart, L.nbwd));
  UFVM_CHECK(build_tpos(c, L));
  UFVM_CHECK(dalloc(L.lord, std::max(L.nnz, 1)));
  k_lower_order<<<nblocks(L.n), kBlock, 0, c.stream>>>(L.n, L.rowptr.p, L.col.p, L.lord.p);
  UFVM_LAUNCH_CHECK();
  L.sched_valid = true;
  L.dc_epoch = 0;
  for (int k = 0; k < 4; ++k) L.sell_valid[k] = false;
  return UFVM_OK;
}

// ---------------------------------------------------------------- level-scheduled sweeps
enum { OP_GS = 0, OP_ILU_FACT = 1, OP_ILU_FWD = 2, OP_ILU_BWD = 3 };

struct SweepArgs {
  int n, nlev, quirks;
  const int *lstart, *rows, *rp, *col, *tpos, *lord;
  const double *ac, *anb, *bc;
  double *x, *dc, *rc;
};

// One row of a sweep, with the reference's operation order. The products that a row
// subtracts do not depend on one another, so they are formed kChunk at a time (their loads
// in flight together) and then subtracted one by one in the reference's order: the same
// operations on the same operands, so the same bits.
constexpr int kChunk = 8;

template <int OP>
__device__ __forceinline__ void row_op(int i, const SweepArgs& a) {
  const int k0 = a.rp[i], k1 = a.rp[i + 1];
  if (OP == OP_GS) {
    // solve/cfdSolveSOR.m:13-29: v = bc - sum anb * x in cconn order, x = v / ac
    double v = a.bc[i];
    for (int k = k0; k < k1; k += kChunk) {
      double p[kChunk];
#pragma unroll
      for (int t = 0; t < kChunk; ++t) p[t] = k + t < k1 ? a.anb[k + t] * __ldcg(a.x + a.col[k + t]) : 0.0;
#pragma unroll
      for (int t = 0; t < kChunk; ++t)
        if (k + t < k1) v = v - p[t];
    }
    __stcg(a.x + i, v / a.ac[i]);
  } else if (OP == OP_ILU_FACT) {
    // solve/cfdFactorizeILU.m:5-47: d = ac - sum over lower j (increasing) of anb(i,j) dc_j anb(j,i)
    double d = a.ac[i];
    for (int k = k0; k < k1; k += kChunk) {
      double p[kChunk];
      bool use[kChunk];
      bool done = false;
#pragma unroll
      for (int t = 0; t < kChunk; ++t) {
        const int q = k + t < k1 ? a.lord[k + t] : -1;
        done |= q < 0;
        int j = q >= 0 ? a.col[q] : -1;
        // Q7: the reference's factorisation loop skips row N-1 (1-based), i.e. row n-2
        const bool skip = (a.quirks & UFVM_Q7_ILU_SKIP_ROW) && j == a.n - 2;
        const int tk = q >= 0 ? a.tpos[q] : -1;  // the pattern is structurally symmetric, so tk >= 0
        use[t] = q >= 0 && !skip && tk >= 0;
        p[t] = use[t] ? a.anb[q] * __ldcg(a.dc + j) * a.anb[tk] : 0.0;
      }
#pragma unroll
      for (int t = 0; t < kChunk; ++t)
        if (use[t]) d = d - p[t];
      if (done) break;
    }
    __stcg(a.dc + i, 1.0 / d);
  } else if (OP == OP_ILU_FWD) {
    // solve/cfdSolveILU.m:33-70 forward substitution over lower j in increasing order
    double v = __ldcg(a.rc + i);
    for (int k = k0; k < k1; k += kChunk) {
      double p[kChunk];
      bool use[kChunk];
      bool done = false;
#pragma unroll
      for (int t = 0; t < kChunk; ++t) {
        const int q = k + t < k1 ? a.lord[k + t] : -1;
        done |= q < 0;
        use[t] = q >= 0;
        if (use[t]) {
          const int j = a.col[q];
          const double mat1 = __ldcg(a.dc + j) * __ldcg(a.rc + j);
          p[t] = a.anb[q] * mat1;
        } else {
          p[t] = 0.0;
        }
      }
#pragma unroll
      for (int t = 0; t < kChunk; ++t)
        if (use[t]) v = v - p[t];
      if (done) break;
    }
    __stcg(a.rc + i, v);
  } else {  // OP_ILU_BWD (solve/cfdSolveILU.m:72-93): upper j in cconn order, then the update
    double v = __ldcg(a.rc + i);
    if (i < a.n - 1) {
      for (int k = k0; k < k1; k += kChunk) {
        double p[kChunk];
        bool use[kChunk];
#pragma unroll
        for (int t = 0; t < kChunk; ++t) {
          const int j = k + t < k1 ? a.col[k + t] : -1;
          use[t] = j > i;
          p[t] = use[t] ? a.anb[k + t] * __ldcg(a.rc + j) : 0.0;
        }
#pragma unroll
        for (int t = 0; t < kChunk; ++t)
          if (use[t]) v = v - p[t];
      }
    }
    const double mat1 = __ldcg(a.dc + i) * v;
    __stcg(a.rc + i, mat1);
    a.x[i] = a.x[i] + mat1;
  }
}

// Wide schedules: one cooperative grid, a software grid barrier between dependency levels.
template <int OP>
__global__ void k_sched_sweep(SweepArgs a, GridBarrier bar) {
  unsigned int gen = grid_gen0(bar);
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
  for (int L = 0; L < a.nlev; ++L) {
    const int s = a.lstart[L], e = a.lstart[L + 1];
    for (int idx = s + tid; idx < e; idx += nth) row_op<OP>(a.rows[idx], a);
    if (L + 1 < a.nlev)
      if (!grid_sync(bar, gen)) return;
  }
}

// Narrow schedules (every level at most a few thousand rows, as in the natural-order sweeps
// of structured meshes and of every coarse AMG level): one CTA, or one thread-block cluster
// of up to 8 CTAs, with the hardware barrier between levels. Writes of a level are made at
// L2 (st.global.cg) and read back from L2 (ld.global.cg); the CTA barrier, or the cluster
// barrier's release/acquire pair, orders them. Every thread of every CTA executes every
// barrier (no early exit), so the barrier cannot wait on a missing CTA.
__device__ __forceinline__ void cluster_barrier() {
  asm volatile("barrier.cluster.arrive.release;\n\tbarrier.cluster.wait.acquire;\n" ::: "memory");
}

template <int OP, bool CLUSTER>
__global__ void __launch_bounds__(1024) k_sched_sweep_cl(SweepArgs a) {
  unsigned int rank = 0, size = 1;
  if (CLUSTER) {
    asm("mov.u32 %0, %%cluster_ctarank;" : "=r"(rank));
    asm("mov.u32 %0, %%cluster_nctarank;" : "=r"(size));
  }
  const int tid = (int)rank * blockDim.x + threadIdx.x, nth = (int)size * blockDim.x;
  for (int L = 0; L < a.nlev; ++L) {
    const int s = a.lstart[L], e = a.lstart[L + 1];
    for (int idx = s + tid; idx < e; idx += nth) row_op<OP>(a.rows[idx], a);
    if (L + 1 < a.nlev) {
      if (CLUSTER) cluster_barrier();
      else __syncthreads();
    }
  }
}

// ILU: r = b - A x (into rc) before the triangular solves
__global__ void k_ilu_res(int n, const int* __restrict__ rp, const int* __restrict__ col, const double* __restrict__ ac,
                          const double* __restrict__ anb, const double* __restrict__ bc, const double* __restrict__ x,
                          double* rc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double res = -ac[i] * x[i] + bc[i];
  for (int k = rp[i]; k < rp[i + 1]; ++k) res = res - anb[k] * x[col[k]];
  rc[i] = res;
}

// ---------------------------------------------------------------- position-ordered sweeps
// The narrow sweeps read each row through a position-ordered ELL copy: schedule position p
// (row i = rows[p]) keeps its entries at [t * n + p], so one coalesced load per array brings a
// level's rows, and nothing but the neighbour values is left to load after the barrier. The
// next level's rows are fetched between the barrier's arrive and its wait (cluster form) or
// before it (single CTA). Each row performs the same operations on the same operands, in the
// same order, as row_op: same bits.
enum { SELL_GS_FWD = 0, SELL_GS_BWD = 1, SELL_ILU_FWD = 2, SELL_ILU_BWD = 3 };

// Entries of row i for one kind, in the kind's order: callback(t, q) with q the CSR position.
template <int KIND, typename F>
__device__ __forceinline__ int sell_entries(int i, const int* __restrict__ rp, const int* __restrict__ col,
                                            const int* __restrict__ lord, F f) {
  const int k0 = rp[i], k1 = rp[i + 1];
  int t = 0;
  if (KIND == SELL_GS_FWD || KIND == SELL_GS_BWD) {
    for (int k = k0; k < k1; ++k) f(t++, k);
  } else if (KIND == SELL_ILU_FWD) {
    for (int k = k0; k < k1; ++k) {
      const int q = lord[k];
      if (q < 0) break;
      f(t++, q);
    }
  } else {
    for (int k = k0; k < k1; ++k)
      if (col[k] > i) f(t++, k);
  }
  return t;
}

template <int KIND>
__global__ void k_sell_width(int n, const int* __restrict__ rows, const int* __restrict__ rp,
                             const int* __restrict__ col, const int* __restrict__ lord, int* wmax) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int w = sell_entries<KIND>(rows[p], rp, col, lord, [](int, int) {});
  atomicMax(wmax, w);
}

// VALUES = false: columns (-1 past the end); true: coefficients.
template <int KIND, bool VALUES>
__global__ void k_sell_fill(int n, int W, const int* __restrict__ rows, const int* __restrict__ rp,
                            const int* __restrict__ col, const int* __restrict__ lord,
                            const double* __restrict__ anb, int* scol, double* sa) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int i = rows[p];
  const int cnt = sell_entries<KIND>(i, rp, col, lord, [&](int t, int q) {
    if (VALUES) sa[(size_t)t * n + p] = anb[q];
    else scol[(size_t)t * n + p] = col[q];
  });
  for (int t = cnt; t < W; ++t) {
    if (VALUES) sa[(size_t)t * n + p] = 0.0;
    else scol[(size_t)t * n + p] = -1;
  }
}

struct SellArgs {
  int n, nlev, W;
  const int *lstart, *rows, *scol;
  const double *sa, *ac, *bc, *dc;
  double *x, *rc;
};

constexpr int kSellPre = 4;

// What a row needs that no other row of the sweep writes: its own values and its first
// kSellPre entries.
struct SellRow {
  int i;
  double own0, own1, own2;
  int c[kSellPre];
  double w[kSellPre];
};

template <int OP>
__device__ __forceinline__ void sell_load(SellRow& r, const SellArgs& a, int p) {
  r.i = -1;
  if (p < 0) return;
  const int i = a.rows[p];
  r.i = i;
  if (OP == OP_GS) {
    r.own0 = a.bc[i];
    r.own1 = a.ac[i];
  } else if (OP == OP_ILU_FWD) {
    r.own0 = __ldcg(a.rc + i);
  } else {  // OP_ILU_BWD
    r.own0 = __ldcg(a.rc + i);
    r.own1 = a.dc[i];
    r.own2 = a.x[i];
  }
#pragma unroll
  for (int t = 0; t < kSellPre; ++t) {
    const bool in = t < a.W;
    r.c[t] = in ? a.scol[(size_t)t * a.n + p] : -1;
    r.w[t] = in ? a.sa[(size_t)t * a.n + p] : 0.0;
  }
}

template <int OP>
__device__ __forceinline__ void sell_finish(const SellRow& r, const SellArgs& a, int p) {
  const int i = r.i;
  // neighbour values (and, for the DILU forward substitution, the factor of the neighbour)
  double g[kSellPre], h[kSellPre];
#pragma unroll
  for (int t = 0; t < kSellPre; ++t) {
    const bool in = r.c[t] >= 0;
    g[t] = in ? (OP == OP_GS ? __ldcg(a.x + r.c[t]) : __ldcg(a.rc + r.c[t])) : 0.0;
    if (OP == OP_ILU_FWD) h[t] = in ? a.dc[r.c[t]] : 0.0;
  }
  double v = r.own0;
  bool end = false;
  if (OP == OP_ILU_BWD && i >= a.n - 1) end = true;  // the reference skips the last row's sum
#pragma unroll
  for (int t = 0; t < kSellPre; ++t) {
    end |= r.c[t] < 0;
    if (!end) {
      if (OP == OP_ILU_FWD) {
        const double mat1 = h[t] * g[t];
        v = v - r.w[t] * mat1;
      } else {
        v = v - r.w[t] * g[t];
      }
    }
  }
  if (!end) {
    for (int t = kSellPre; t < a.W; ++t) {
      const int j = a.scol[(size_t)t * a.n + p];
      if (j < 0) break;
      const double wt = a.sa[(size_t)t * a.n + p];
      if (OP == OP_ILU_FWD) {
        const double mat1 = a.dc[j] * __ldcg(a.rc + j);
        v = v - wt * mat1;
      } else if (OP == OP_GS) {
        v = v - wt * __ldcg(a.x + j);
      } else {
        v = v - wt * __ldcg(a.rc + j);
      }
    }
  }
  if (OP == OP_GS) {
    __stcg(a.x + i, v / r.own1);
  } else if (OP == OP_ILU_FWD) {
    __stcg(a.rc + i, v);
  } else {
    const double mat1 = r.own1 * v;
    __stcg(a.rc + i, mat1);
    a.x[i] = r.own2 + mat1;
  }
}

template <int OP, bool CLUSTER>
__global__ void __launch_bounds__(1024) k_sched_sell(SellArgs a) {
  unsigned int rank = 0, size = 1;
  if (CLUSTER) {
    asm("mov.u32 %0, %%cluster_ctarank;" : "=r"(rank));
    asm("mov.u32 %0, %%cluster_nctarank;" : "=r"(size));
  }
  const int tid = (int)rank * blockDim.x + threadIdx.x, nth = (int)size * blockDim.x;
  SellRow pre;
  {
    const int e = a.lstart[1];
    sell_load<OP>(pre, a, tid < e ? tid : -1);
  }
  for (int L = 0; L < a.nlev; ++L) {
    const int s = a.lstart[L], e = a.lstart[L + 1];
    if (s + tid < e) sell_finish<OP>(pre, a, s + tid);
    for (int p = s + tid + nth; p < e; p += nth) {
      SellRow r;
      sell_load<OP>(r, a, p);
      sell_finish<OP>(r, a, p);
    }
    if (L + 1 < a.nlev) {
      const int s2 = a.lstart[L + 1], e2 = a.lstart[L + 2];
      if (CLUSTER) {
        asm volatile("barrier.cluster.arrive.release;\n" ::: "memory");
        sell_load<OP>(pre, a, s2 + tid < e2 ? s2 + tid : -1);
        asm volatile("barrier.cluster.wait.acquire;\n" ::: "memory");
      } else {
        sell_load<OP>(pre, a, s2 + tid < e2 ? s2 + tid : -1);
        __syncthreads();
      }
    }
  }
}

template <int KIND>
static int sell_prepare_kind(LinCtx& c, Level& L) {
  const int n = L.n;
  const int* rows = (KIND == SELL_GS_FWD || KIND == SELL_ILU_FWD) ? L.fwdRows.p : L.bwdRows.p;
  if (!L.sell_valid[KIND]) {
    UFVM_CUDA(cudaMemsetAsync(c.iflag.p + 5, 0, sizeof(int), c.stream));
    k_sell_width<KIND><<<nblocks(n), kBlock, 0, c.stream>>>(n, rows, L.rowptr.p, L.col.p, L.lord.p, c.iflag.p + 5);
    UFVM_LAUNCH_CHECK();
    int W = 0;
    UFVM_CUDA(cudaMemcpyAsync(&W, c.iflag.p + 5, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    UFVM_CUDA(cudaStreamSynchronize(c.stream));
    const size_t cap = std::max<size_t>((size_t)W * n, 1);
    UFVM_CHECK(dalloc(L.sellCol[KIND], cap));
    UFVM_CHECK(dalloc(L.sellA[KIND], cap));
    L.sellW[KIND] = W;
    k_sell_fill<KIND, false><<<nblocks(n), kBlock, 0, c.stream>>>(n, W, rows, L.rowptr.p, L.col.p, L.lord.p, nullptr,
                                                                 L.sellCol[KIND].p, nullptr);
    UFVM_LAUNCH_CHECK();
    L.sell_valid[KIND] = true;
    L.sell_epoch[KIND] = 0;
  }
  // the copied coefficients follow the matrix: once per AMG solve, on every call outside one
  if (c.factor_epoch == 0 || L.sell_epoch[KIND] != c.factor_epoch) {
    k_sell_fill<KIND, true><<<nblocks(n), kBlock, 0, c.stream>>>(n, L.sellW[KIND], rows, L.rowptr.p, L.col.p,
                                                                L.lord.p, L.anb.p, nullptr, L.sellA[KIND].p);
    UFVM_LAUNCH_CHECK();
    L.sell_epoch[KIND] = c.factor_epoch;
  }
  return UFVM_OK;
}

// Rows a cluster sweep handles per thread and level before the wide (grid) form pays off.
constexpr int kClusterRowsPerThread = 4;

// 0: the wide grid form; 1: one CTA; 2, 4 or 8: one cluster of that many 1024-thread CTAs.
template <int OP>
static int sweep_shape(LinCtx& c, const Level& L) {
  const int w = std::max(L.maxw, 1);
  if (w <= 1024) return 1;
  if (w > 8 * 1024 * kClusterRowsPerThread) return 0;
  if (c.cluster_ok == 0) {
    // once per context: can a cluster of 8 such CTAs be resident?
    cudaLaunchConfig_t q = {};
    q.gridDim = dim3(8);
    q.blockDim = dim3(1024);
    q.stream = c.stream;
    cudaLaunchAttribute qa[1];
    qa[0].id = cudaLaunchAttributeClusterDimension;
    qa[0].val.clusterDim.x = 8;
    qa[0].val.clusterDim.y = 1;
    qa[0].val.clusterDim.z = 1;
    q.attrs = qa;
    q.numAttrs = 1;
    int ncl = 0;
    const cudaError_t e = cudaOccupancyMaxActiveClusters(&ncl, (const void*)k_sched_sell<OP_ILU_FWD, true>, &q);
    int ncl2 = 0;
    const cudaError_t e2 = cudaOccupancyMaxActiveClusters(&ncl2, (const void*)k_sched_sweep_cl<OP_ILU_FACT, true>, &q);
    if (e != cudaSuccess || e2 != cudaSuccess) (void)cudaGetLastError();
    c.cluster_ok = (e == cudaSuccess && e2 == cudaSuccess && ncl >= 1 && ncl2 >= 1) ? 1 : -1;
  }
  if (c.cluster_ok < 0) return 0;
  int cs = 2;
  while (cs < 8 && cs * 1024 < w) cs *= 2;
  return cs;
}

template <typename K, typename A>
static int launch_cluster(K kernel, int cs, cudaStream_t st, const A& args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(cs);
  cfg.blockDim = dim3(1024);
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cs;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  UFVM_CUDA(cudaLaunchKernelEx(&cfg, kernel, args));
  return UFVM_OK;
}

template <int OP>
static int launch_sweep(LinCtx& c, Level& L, bool fwd, int quirks) {
  const int shape = sweep_shape<OP>(c, L);
  const int w = std::max(L.maxw, 1);
  const int bs1 = std::min(1024, std::max(32, (w + 31) / 32 * 32));
  if (shape != 0 && OP != OP_ILU_FACT) {
    constexpr int kind = OP == OP_GS ? -1 : (OP == OP_ILU_FWD ? SELL_ILU_FWD : SELL_ILU_BWD);
    const int k = kind >= 0 ? kind : (fwd ? SELL_GS_FWD : SELL_GS_BWD);
    switch (k) {
      case SELL_GS_FWD: UFVM_CHECK(sell_prepare_kind<SELL_GS_FWD>(c, L)); break;
      case SELL_GS_BWD: UFVM_CHECK(sell_prepare_kind<SELL_GS_BWD>(c, L)); break;
      case SELL_ILU_FWD: UFVM_CHECK(sell_prepare_kind<SELL_ILU_FWD>(c, L)); break;
      default: UFVM_CHECK(sell_prepare_kind<SELL_ILU_BWD>(c, L)); break;
    }
    SellArgs s;
    s.n = L.n;
    s.nlev = fwd ? L.nfwd : L.nbwd;
    s.W = L.sellW[k];
    s.lstart = fwd ? L.fwdStart.p : L.bwdStart.p;
    s.rows = fwd ? L.fwdRows.p : L.bwdRows.p;
    s.scol = L.sellCol[k].p;
    s.sa = L.sellA[k].p;
    s.ac = L.ac.p; s.bc = L.bc.p; s.dc = L.dc.p;
    s.x = L.dphi.p; s.rc = L.rc.p;
    if (shape == 1) {
      k_sched_sell<OP, false><<<1, bs1, 0, c.stream>>>(s);
      UFVM_LAUNCH_CHECK();
      return UFVM_OK;
    }
    return launch_cluster(k_sched_sell<OP, true>, shape, c.stream, s);
  }
  SweepArgs a;
  a.n = L.n; a.quirks = quirks;
  a.nlev = fwd ? L.nfwd : L.nbwd;
  a.lstart = fwd ? L.fwdStart.p : L.bwdStart.p;
  a.rows = fwd ? L.fwdRows.p : L.bwdRows.p;
  a.rp = L.rowptr.p; a.col = L.col.p; a.tpos = L.tpos.p; a.lord = L.lord.p;
  a.ac = L.ac.p; a.anb = L.anb.p; a.bc = L.bc.p;
  a.x = L.dphi.p; a.dc = L.dc.p; a.rc = L.rc.p;
  if (shape == 1) {
    k_sched_sweep_cl<OP, false><<<1, bs1, 0, c.stream>>>(a);
    UFVM_LAUNCH_CHECK();
    return UFVM_OK;
  }
  if (shape > 1) return launch_cluster(k_sched_sweep_cl<OP, true>, shape, c.stream, a);
  GridBarrier gb{c.bar.p, c.bar.p + 1, c.berr.p};
  int maxb = 0;
  UFVM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&maxb, k_sched_sweep<OP>, kBlock, 0));
  const int coop = std::max(1, maxb * c.nsm);
  const int nb = std::max(1, std::min(coop, nblocks(L.maxw)));
  void* args[] = {(void*)&a, (void*)&gb};
  UFVM_CUDA(cudaLaunchCooperativeKernel((const void*)k_sched_sweep<OP>, dim3(nb), dim3(kBlock), args, 0, c.stream));
  return UFVM_OK;
}

int check_barrier(LinCtx& c) {
  int err = 0;
  UFVM_CUDA(cudaMemcpyAsync(&err, c.berr.p, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  UFVM_CUDA(cudaStreamSynchronize(c.stream));
  if (err) {
    UFVM_CUDA(cudaMemsetAsync(c.berr.p, 0, sizeof(int), c.stream));
    UFVM_CUDA(cudaMemsetAsync(c.bar.p, 0, 2 * sizeof(unsigned int), c.stream));
    set_error("grid barrier timed out in a level-scheduled sweep");
    return UFVM_E_TIMEOUT;
  }
  return UFVM_OK;
}

int gs_sweep(LinCtx& c, Level& L) {
  UFVM_CHECK(c.ensure(L.n));
  UFVM_CHECK(build_schedule(c, L));
  UFVM_CHECK(launch_sweep<OP_GS>(c, L, true, 0));
  UFVM_CHECK(launch_sweep<OP_GS>(c, L, false, 0));
  return UFVM_OK;
}

int ilu_factor(LinCtx& c, Level& L, int quirks) {
  UFVM_CHECK(c.ensure(L.n));
  UFVM_CHECK(build_schedule(c, L));
  // within one AMG solve the level's matrix is fixed: the factor already computed is the one
  // the reference recomputes on every smoother call (solve/cfdSolveAlgebraicSystem.m:29-33)
  if (c.factor_epoch != 0 && L.dc_epoch == c.factor_epoch && L.dc_quirks == quirks && L.dc.p) return UFVM_OK;
  UFVM_CHECK(dalloc(L.dc, L.n));
  UFVM_CHECK(launch_sweep<OP_ILU_FACT>(c, L, true, quirks));
  L.dc_epoch = c.factor_epoch;
  L.dc_quirks = quirks;
  return UFVM_OK;
}

int ilu_sweep(LinCtx& c, Level& L) {
  UFVM_CHECK(c.ensure(L.n));
  UFVM_CHECK(build_schedule(c, L));
  UFVM_CHECK(dalloc(L.rc, L.n));
  k_ilu_res<<<nblocks(L.n), kBlock, 0, c.stream>>>(L.n, L.rowptr.p, L.col.p, L.ac.p, L.anb.p, L.bc.p, L.dphi.p, L.rc.p);
  UFVM_LAUNCH_CHECK();
  UFVM_CHECK(launch_sweep<OP_ILU_FWD>(c, L, true, 0));
  UFVM_CHECK(launch_sweep<OP_ILU_BWD>(c, L, false, 0));
  return UFVM_OK;
}

// ---------------------------------------------------------------- colouring + MCGS
// Greedy first-fit colouring in natural order, computed in dependency rounds: a row takes
// the smallest colour unused by its lower-index neighbours once all of them are coloured.
// A row's colour depends only on its lower neighbours' final colours, so the result is the
// sequential greedy colouring whatever the round in which a row is reached.
__global__ void k_greedy_round(int n, const int* __restrict__ rp, const int* __restrict__ col, int* color,
                               int* remaining) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || __ldcg(color + i) >= 0) return;
  unsigned long long used = 0;
  bool big = false;
  for (int k = rp[i]; k < rp[i + 1]; ++k) {
    const int j = col[k];
    if (j >= i) continue;
    const int cj = __ldcg(color + j);
    if (cj < 0) { atomicAdd(remaining, 1); return; }
    if (cj < 64) used |= 1ull << cj;
    else big = true;
  }
  int c = ~used ? __ffsll(~used) - 1 : 64;
  if (c >= 64 || big) {
    for (c = 0;; ++c) {
      bool hit = false;
      for (int k = rp[i]; k < rp[i + 1] && !hit; ++k) hit = col[k] < i && __ldcg(color + col[k]) == c;
      if (!hit) break;
    }
  }
  __stcg(color + i, c);
}

__global__ void k_max_color(int n, const int* __restrict__ color, int* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) atomicMax(out, color[i] + 1);
}

int build_coloring(LinCtx& c, Level& L) {
  if (L.color_valid) return UFVM_OK;
  UFVM_CHECK(c.ensure(L.n));
  const int n = L.n;
  UFVM_CHECK(dalloc(L.color, n));
  UFVM_CUDA(cudaMemsetAsync(L.color.p, 0xff, n * sizeof(int), c.stream));
  for (int round = 0;; round += 8) {
    UFVM_CUDA(cudaMemsetAsync(c.iflag.p, 0, sizeof(int), c.stream));
    for (int k = 0; k < 8; ++k) {
      if (k == 7) UFVM_CUDA(cudaMemsetAsync(c.iflag.p, 0, sizeof(int), c.stream));
      k_greedy_round<<<nblocks(n), kBlock, 0, c.stream>>>(n, L.rowptr.p, L.col.p, L.color.p, c.iflag.p);
    }
    UFVM_LAUNCH_CHECK();
    int rem = 0;
    UFVM_CUDA(cudaMemcpyAsync(&rem, c.iflag.p, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    UFVM_CUDA(cudaStreamSynchronize(c.stream));
    if (rem == 0) break;
    if (round > n + 8) { set_error("colouring rounds did not terminate"); return UFVM_E_INVALID; }
  }
  UFVM_CUDA(cudaMemsetAsync(c.iflag.p + 2, 0, sizeof(int), c.stream));
  k_max_color<<<nblocks(n), kBlock, 0, c.stream>>>(n, L.color.p, c.iflag.p + 2);
  UFVM_LAUNCH_CHECK();
  int nc = 0;
  UFVM_CUDA(cudaMemcpyAsync(&nc, c.iflag.p + 2, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  UFVM_CUDA(cudaStreamSynchronize(c.stream));
  L.ncolor = nc;
  // rows grouped by colour
  DArr<int> cnt;
  UFVM_CHECK(dalloc(cnt, nc + 2));
  UFVM_CUDA(cudaMemsetAsync(cnt.p, 0, (nc + 2) * sizeof(int), c.stream));
  UFVM_CUDA(cudaMemsetAsync(c.iflag.p + 3, 0, sizeof(int), c.stream));
  k_level_hist<<<nblocks(n), kBlock, 0, c.stream>>>(n, L.color.p, cnt.p, c.iflag.p + 3);
  UFVM_CHECK(dalloc(L.colorStart, nc + 1));
  UFVM_CHECK(scan_exclusive(c, cnt.p, L.colorStart.p, nc, nullptr));
  UFVM_CUDA(cudaMemcpyAsync(cnt.p, L.colorStart.p, nc * sizeof(int), cudaMemcpyDeviceToDevice, c.stream));
  UFVM_CHECK(dalloc(L.colorRows, n));
  k_level_fill<<<nblocks(n), kBlock, 0, c.stream>>>(n, L.color.p, cnt.p, L.colorRows.p);
  UFVM_LAUNCH_CHECK();
  L.h_colorStart.resize(nc + 1);
  UFVM_CUDA(cudaMemcpyAsync(L.h_colorStart.data(), L.colorStart.p, (nc + 1) * sizeof(int), cudaMemcpyDeviceToHost,
                            c.stream));
  UFVM_CUDA(cudaStreamSynchronize(c.stream));
  dfree(cnt);
  L.color_valid = true;
  return UFVM_OK;
}

// The plain FP64 multicolour sweep reads a colour-major ELL copy of the matrix: position p
// holds row mcRow[p] (colours ascending, rows ascending inside a colour), entry k of position
// p sits at [k * n + p] (column -1 past the row's end), so a colour's rows are read with
// unit stride. x stays in natural order. Each row evaluates v = bc - sum anb * x in cconn
// order and x = v / ac, the operation order of the CSR sweep: the copy changes no bit.
__global__ void k_color_flag(int n, const int* __restrict__ color, int c, int* flag) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) flag[i] = color[i] == c;
}

__global__ void k_color_place(int n, const int* __restrict__ color, int c, int base, const int* __restrict__ pos,
                              int* mcRow) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && color[i] == c) mcRow[base + pos[i]] = i;
}

__global__ void k_row_len_max(int n, const int* __restrict__ rp, int* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) atomicMax(out, rp[i + 1] - rp[i]);
}

__global__ void k_mc_pattern(int n, int W, const int* __restrict__ mcRow, const int* __restrict__ rp,
                             const int* __restrict__ col, int* mcCol) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int i = mcRow[p], k0 = rp[i], len = rp[i + 1] - k0;
  for (int k = 0; k < W; ++k) mcCol[(size_t)k * n + p] = k < len ? col[k0 + k] : -1;
}

__global__ void k_mc_values(int n, int W, const int* __restrict__ mcRow, const int* __restrict__ rp,
                            const double* __restrict__ ac, const double* __restrict__ anb, double* mcAc,
                            double* mcAnb) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int i = mcRow[p], k0 = rp[i], len = rp[i + 1] - k0;
  mcAc[p] = ac[i];
  for (int k = 0; k < W; ++k) mcAnb[(size_t)k * n + p] = k < len ? anb[k0 + k] : 0.0;
}

__global__ void k_mc_bc(int n, const int* __restrict__ mcRow, const double* __restrict__ bc, double* mcBc) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n) mcBc[p] = bc[mcRow[p]];
}

// One colour's rows. The colour kernels of a sweep follow one another as programmatic
// dependent launches: a kernel starts while the previous colour is still running, loads what
// does not depend on x (its rows' positions, bc, ac and the first kMcPre entries, all
// coalesced), and only then waits (griddepcontrol.wait returns once the previous kernel has
// completed and its writes are visible) before it gathers the neighbour values.
constexpr int kMcPre = 4;

__global__ void __launch_bounds__(kBlock) k_mc_rows(int cnt, int p0, int n, int W, const int* __restrict__ mcRow,
                                                   const int* __restrict__ mcCol, const double* __restrict__ mcAnb,
                                                   const double* __restrict__ mcAc,
                                                   const double* __restrict__ mcBc, double* x) {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= cnt) return;
  const int p = p0 + t;
  const int i = mcRow[p];
  const double b = mcBc[p], a = mcAc[p];
  int j[kMcPre];
  double w[kMcPre];
#pragma unroll
  for (int k = 0; k < kMcPre; ++k) {
    j[k] = k < W ? mcCol[(size_t)k * n + p] : -1;
    w[k] = k < W ? mcAnb[(size_t)k * n + p] : 0.0;
  }
  asm volatile("griddepcontrol.wait;" ::: "memory");
  double xv[kMcPre];
#pragma unroll
  for (int k = 0; k < kMcPre; ++k) xv[k] = j[k] >= 0 ? x[j[k]] : 0.0;
  double v = b;
  bool end = false;
#pragma unroll
  for (int k = 0; k < kMcPre; ++k) {
    end |= j[k] < 0;
    if (!end) v = v - w[k] * xv[k];
  }
  if (!end) {
    for (int k = kMcPre; k < W; ++k) {
      const int jj = mcCol[(size_t)k * n + p];
      if (jj < 0) break;
      v = v - mcAnb[(size_t)k * n + p] * x[jj];
    }
  }
  x[i] = v / a;
}

static int build_mc_pattern(LinCtx& c, Level& L) {
  if (L.mc_valid) return UFVM_OK;
  UFVM_CHECK(build_coloring(c, L));
  const int n = L.n;
  UFVM_CHECK(dalloc(L.mcRow, n));
  DArr<int> flag, pos;
  UFVM_CHECK(dalloc(flag, n));
  UFVM_CHECK(dalloc(pos, n + 1));
  for (int q = 0; q < L.ncolor; ++q) {
    k_color_flag<<<nblocks(n), kBlock, 0, c.stream>>>(n, L.color.p, q, flag.p);
    UFVM_CHECK(scan_exclusive(c, flag.p, pos.p, n, nullptr));
    k_color_place<<<nblocks(n), kBlock, 0, c.stream>>>(n, L.color.p, q, L.h_colorStart[q], pos.p, L.mcRow.p);
  }
  UFVM_LAUNCH_CHECK();
  UFVM_CUDA(cudaMemsetAsync(c.iflag.p + 4, 0, sizeof(int), c.stream));
  k_row_len_max<<<nblocks(n), kBlock, 0, c.stream>>>(n, L.rowptr.p, c.iflag.p + 4);
  UFVM_LAUNCH_CHECK();
  int W = 0;
  UFVM_CUDA(cudaMemcpyAsync(&W, c.iflag.p + 4, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  UFVM_CUDA(cudaStreamSynchronize(c.stream));
  L.mcW = W;
  const size_t cap = std::max<size_t>((size_t)W * n, 1);
  UFVM_CHECK(dalloc(L.mcCol, cap));
  UFVM_CHECK(dalloc(L.mcAnb, cap));
  UFVM_CHECK(dalloc(L.mcAc, n));
  UFVM_CHECK(dalloc(L.mcBc, n));
  k_mc_pattern<<<nblocks(n), kBlock, 0, c.stream>>>(n, W, L.mcRow.p, L.rowptr.p, L.col.p, L.mcCol.p);
  UFVM_LAUNCH_CHECK();
  dfree(flag);
  dfree(pos);
  L.mc_valid = true;
  L.mc_epoch = 0;
  return UFVM_OK;
}

// Copies the matrix (once per AMG solve, or on every call outside one) and the right-hand
// side (every call) into the colour-major layout.
int mcgs_prepare(LinCtx& c, Level& L) {
  UFVM_CHECK(c.ensure(L.n));
  UFVM_CHECK(build_mc_pattern(c, L));
  if (c.factor_epoch == 0 || L.mc_epoch != c.factor_epoch) {
    k_mc_values<<<nblocks(L.n), kBlock, 0, c.stream>>>(L.n, L.mcW, L.mcRow.p, L.rowptr.p, L.ac.p, L.anb.p, L.mcAc.p,
                                                       L.mcAnb.p);
    L.mc_epoch = c.factor_epoch;
  }
  k_mc_bc<<<nblocks(L.n), kBlock, 0, c.stream>>>(L.n, L.mcRow.p, L.bc.p, L.mcBc.p);
  UFVM_LAUNCH_CHECK();
  return UFVM_OK;
}

int mcgs_sweep(LinCtx& c, Level& L) {
  if (!L.mc_valid) { set_error("mcgs_sweep: layout not prepared"); return UFVM_E_INVALID; }
  // the first colour kernel of the sweep waits for all earlier work the ordinary way; the
  // later ones are programmatic dependents of the colour before them
  int launched = 0;
  // the backward pass starts one colour in: its first colour would repeat the forward pass's
  // last update from the same neighbour values (same bits), so it is skipped
  for (int pass = 0; pass < 2; ++pass) {
    for (int q = pass; q < L.ncolor; ++q) {
      const int col_ = pass == 0 ? q : L.ncolor - 1 - q;
      const int s = L.h_colorStart[col_], cnt = L.h_colorStart[col_ + 1] - s;
      if (cnt <= 0) continue;
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(nblocks(cnt));
      cfg.blockDim = dim3(kBlock);
      cfg.stream = c.stream;
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
      attr[0].val.programmaticStreamSerializationAllowed = 1;
      cfg.attrs = attr;
      cfg.numAttrs = launched > 0 ? 1 : 0;
      UFVM_CUDA(cudaLaunchKernelEx(&cfg, k_mc_rows, cnt, s, L.n, L.mcW, (const int*)L.mcRow.p,
                                   (const int*)L.mcCol.p, (const double*)L.mcAnb.p, (const double*)L.mcAc.p,
                                   (const double*)L.mcBc.p, L.dphi.p));
      ++launched;
    }
  }
  return UFVM_OK;
}

// ---------------------------------------------------------------- smoother loop
int solve_algebraic_system(LinCtx& c, Level& L, int smoother, int n_iter, double rrf, int quirks, double* r0out,
                           double* r1out, int* iters) {
  UFVM_CHECK(c.ensure(L.n));
  double s0 = 0;
  UFVM_CHECK(sum_abs_residual(c, L, L.dphi.p, &s0));
  const double r0 = s0 / L.n;
  double r1 = r0;
  int it = 1;
  if (smoother == UFVM_SMOOTHER_ILU) {
    UFVM_CHECK(ilu_factor(c, L, quirks));
    while (it <= n_iter && r1 > rrf * r0) {
      UFVM_CHECK(ilu_sweep(c, L));
      double s = 0;
      UFVM_CHECK(sum_abs_residual(c, L, L.dphi.p, &s));
      UFVM_CHECK(check_barrier(c));
      r1 = s / L.n;
      ++it;
    }
  } else {
    if (smoother != UFVM_SMOOTHER_SOR) UFVM_CHECK(mcgs_prepare(c, L));
    while (it <= n_iter && r1 > rrf * r0) {
      if (smoother == UFVM_SMOOTHER_SOR) UFVM_CHECK(gs_sweep(c, L));
      else UFVM_CHECK(mcgs_sweep(c, L));
      double s = 0;
      UFVM_CHECK(sum_abs_residual(c, L, L.dphi.p, &s));
      if (smoother == UFVM_SMOOTHER_SOR) UFVM_CHECK(check_barrier(c));
      r1 = s / L.n;
      ++it;
    }
  }
  if (r0out) *r0out = r0;
  if (r1out) *r1out = r1;
  if (iters) *iters = it - 1;
  return UFVM_OK;
}

// ---------------------------------------------------------------- transfers
__global__ void k_restrict(int nc, const int* __restrict__ cs, const int* __restrict__ ch,
                           const double* __restrict__ r, double* bcC) {
  const int P = blockIdx.x * blockDim.x + threadIdx.x;
  if (P >= nc) return;
  double v = 0.0;
  for (int q = cs[P]; q < cs[P + 1]; ++q) v = v + r[ch[q]];
  bcC[P] = v;
}

__global__ void k_prolong(int n, const int* __restrict__ parents, const double* __restrict__ dC, double* dF) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dF[i] = dF[i] + dC[parents[i]];
}

int restrict_residual(LinCtx& c, Level& F, Level& C) {
  UFVM_CHECK(dalloc(F.r, F.n));
  UFVM_CHECK(residual(c, F, F.dphi.p, F.r.p));
  k_restrict<<<nblocks(C.n), kBlock, 0, c.stream>>>(C.n, F.childStart.p, F.child.p, F.r.p, C.bc.p);
  UFVM_LAUNCH_CHECK();
  return UFVM_OK;
}

int prolong(LinCtx& c, Level& F, const Level& C) {
  k_prolong<<<nblocks(F.n), kBlock, 0, c.stream>>>(F.n, F.parents.p, C.dphi.p, F.dphi.p);
  UFVM_LAUNCH_CHECK();
  return UFVM_OK;
}

}  // namespace ufvm
