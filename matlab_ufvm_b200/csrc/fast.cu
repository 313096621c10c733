// fast.cu -- the batched steady-case service (many cases, one launch per stage).
//
// Linear solves (declared deviations from the reference's sequential smoothers; the SIMPLE
// stages themselves are the reference's, shared with the plain path):
//   U : multicolour symmetric Gauss-Seidel in FP64 with the reference's stopping rule
//       (solve/cfdSolveAlgebraicSystem.m:38-46: at most u_n_iter sweeps, stop once
//       sum|r|/N <= rrf * initial), evaluated per case on the device.
//   p : FP64 flexible CG preconditioned by one FP32 agglomeration-AMG V-cycle (multicolour GS
//       smoothing, FP32 restriction / prolongation by the agglomeration maps, FP64 coarsest
//       solution operator); the residual, search directions and the update stay FP64, and
//       iterations stop per case on the reference's rule (cfdApplyAMG.m:27-52: at most
//       p_max_cycles, stop once sum|r| <= termination * initial). p_krylov 0 gives plain FP64
//       iterative refinement (x += V(r)) instead.
// The agglomeration maps are the reference's (exact seed agglomeration of the assembled p
// matrix) built on a case's first p solve and reused; the Galerkin coarse operators are
// recomputed in FP64 from the current matrix at every p solve. Level 0 of the V-cycle is
// stored colour-permuted in ELL form; levels up to cta_rows rows run one CTA per case.
// A step without hierarchy builds is captured once and replayed as a CUDA graph whose solve
// loops are conditional WHILE nodes ended on the device.
#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <thread>
#include <utility>

#include "fast.cuh"

namespace ufvm {

#define LEV(l, s) levTab[(size_t)(l) * ns + (s)]

// rows of ELL matrices with at most this many entries issue all their column and coefficient
// loads before the first neighbour gather
constexpr int kEllUnroll = 8;

// ---------------------------------------------------------------- FP64 fine-level kernels
// ---- the FP64 U solve. A case whose level 0 has the colour-permuted ELL layout (pmode 1)
// smooths an ELL copy of its momentum matrix (uAc, uBc, uAnb at [k * n + p], uX), made after
// each assembly and scattered back into dphi after the solve; a case without it (its first
// step, before its hierarchy exists) smooths the natural CSR matrix through the colour rows.
// Either way each row is v = bc - sum anb x in cconn order, x = v / ac.
__device__ __forceinline__ double urow_sum(const LevDesc& A, int p, double v) {
  const int W = A.ellW;
  const size_t n = (size_t)A.n;
  if (W <= kEllUnroll) {
    int c[kEllUnroll];
    double a[kEllUnroll];
#pragma unroll
    for (int k = 0; k < kEllUnroll; ++k) {
      c[k] = k < W ? A.ellCol[k * n + p] : -1;
      a[k] = k < W ? A.uAnb[k * n + p] : 0.0;
    }
    double xv[kEllUnroll];
#pragma unroll
    for (int k = 0; k < kEllUnroll; ++k) xv[k] = c[k] >= 0 ? A.uX[c[k]] : 0.0;
#pragma unroll
    for (int k = 0; k < kEllUnroll; ++k)
      if (c[k] >= 0) v = v - a[k] * xv[k];
    return v;
  }
  for (int k = 0; k < W; ++k) {
    const int c = A.ellCol[k * n + p];
    if (c < 0) break;
    v = v - A.uAnb[k * n + p] * A.uX[c];
  }
  return v;
}

__global__ void k_res64_abs(const SlotDesc* __restrict__ slots, const LevDesc* __restrict__ levTab, int ns,
                            const int2* __restrict__ work, const SolveCtl* __restrict__ ctl, double* part) {
  pdl_trigger();  // a chained launch of the solve loops (see launch_k): start early, then
  pdl_wait();     // wait for the kernel before it
  __shared__ double sh[32];
  const int2 w = work[blockIdx.x];
  const SlotDesc& S = slots[w.x];
  const LevDesc& A = LEV(0, w.x);
  const int i = w.y * blockDim.x + threadIdx.x;
  double v = 0.0;
  if (i < S.m.Nc && ctl[w.x].active) {
    if (A.pmode) {
      v = fabs(urow_sum(A, i, A.uBc[i] - A.uAc[i] * A.uX[i]));
    } else {
      const int* rp = S.m.rowptr;
      double r = S.bc[i] - S.ac[i] * S.dphi[i];
      for (int k = rp[i]; k < rp[i + 1]; ++k) r = r - S.anb[k] * S.dphi[S.m.col[k]];
      v = fabs(r);
    }
  }
  v = block_reduce<0>(v, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = v;
}

// ELL copy of the just-assembled momentum matrix (pmode cases)
__global__ void k_u_to_ell(const SlotDesc* __restrict__ slots, const LevDesc* __restrict__ levTab, int ns,
                           const int2* __restrict__ work) {
  const int2 w = work[blockIdx.x];
  const LevDesc& A = LEV(0, w.x);
  if (!A.pmode) return;
  const SlotDesc& S = slots[w.x];
  const int p = w.y * blockDim.x + threadIdx.x;
  if (p >= A.n) return;
  const int i = A.perm[p], k0 = S.m.rowptr[i], deg = S.m.rowptr[i + 1] - k0;
  A.uAc[p] = S.ac[i];
  A.uBc[p] = S.bc[i];
  A.uX[p] = S.dphi[i];
  for (int k = 0; k < A.ellW; ++k) A.uAnb[(size_t)k * A.n + p] = k < deg ? S.anb[k0 + k] : 0.0;
}

__global__ void k_u_from_ell(const SlotDesc* __restrict__ slots, const LevDesc* __restrict__ levTab, int ns,
                             const int2* __restrict__ work) {
  const int2 w = work[blockIdx.x];
  const LevDesc& A = LEV(0, w.x);
  if (!A.pmode) return;
  const SlotDesc& S = slots[w.x];
  const int p = w.y * blockDim.x + threadIdx.x;
  if (p < A.n) S.dphi[A.perm[p]] = A.uX[p];
}

// r = b - A x (FP64) -> FP32 right-hand side of the correction; e = 0
__global__ void k_res64_rhs(const SlotDesc* __restrict__ slots, const LevDesc* __restrict__ levTab, int ns,
                            const int2* __restrict__ work, const SolveCtl* __restrict__ ctl, double* part) {
  pdl_trigger();  // a chained launch of the solve loops (see launch_k): start early, then
  pdl_wait();     // wait for the kernel before it
  __shared__ double sh[32];
  const int2 w = work[blockIdx.x];
  const SlotDesc& S = slots[w.x];
  const LevDesc& A = LEV(0, w.x);
  const int i = w.y * blockDim.x + threadIdx.x;
  double v = 0.0;
  if (i < S.m.Nc && ctl[w.x].active) {
    const int* rp = S.m.rowptr;
    double r = S.bc[i] - S.ac[i] * S.dphi[i];
    for (int k = rp[i]; k < rp[i + 1]; ++k) r = r - S.anb[k] * S.dphi[S.m.col[k]];
    v = fabs(r);
    if (A.fr) A.fr[i] = r;
    const int j = A.pmode ? A.inv[i] : i;
    A.bc[j] = (float)r;
    A.x[j] = 0.0f;
  }
  v = block_reduce<0>(v, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = v;
}

__global__ void k_update64(const SlotDesc* __restrict__ slots, const LevDesc* __restrict__ levTab, int ns,
                           const int2* __restrict__ work, const SolveCtl* __restrict__ ctl) {
  pdl_trigger();  // a chained launch of the solve loops (see launch_k): start early, then
  pdl_wait();     // wait for the kernel before it
  const int2 w = work[blockIdx.x];
  if (!ctl[w.x].active) return;
  const SlotDesc& S = slots[w.x];
  const int i = w.y * blockDim.x + threadIdx.x;
  const LevDesc& A = LEV(0, w.x);
  if (i < S.m.Nc) S.dphi[i] = S.dphi[i] + (double)A.x[A.pmode ? A.inv[i] : i];
}

// ---------------------------------------------------------------- flexible CG on level 0
// FCG(1) (Notay, SIAM J. Sci. Comput. 22 (2000) 1444) on the FP64 correction equation, with one
// FP32 V-cycle z = V(r) as the (slightly non-symmetric, non-stationary) preconditioner:
//   beta = (z, q_old) / (p_old, q_old),  p = z - beta p_old,  q = A p,
//   alpha = (p, r) / (p, q),  x += alpha p,  r -= alpha q.
// The p-correction matrix is symmetric positive semi-definite (face coefficients enter the
// owner and neighbour rows alike), which is what CG needs; the stopping rule stays the
// reference's (sum|r| against the initial sum). Dot products are per (slot, block) partials
// summed per slot in a fixed order.
__global__ void k_fcg_zq(const SlotDesc* __restrict__ slots, const LevDesc* __restrict__ levTab, int ns,
                         const int2* __restrict__ work, const SolveCtl* __restrict__ ctl, double* part) {
  pdl_trigger();  // a chained launch of the solve loops (see launch_k): start early, then
  pdl_wait();     // wait for the kernel before it
  __shared__ double sh[32];
  const int2 w = work[blockIdx.x];
  const SlotDesc& S = slots[w.x];
  const LevDesc& A = LEV(0, w.x);
  const int i = w.y * blockDim.x + threadIdx.x;
  double v = 0.0;
  if (i < S.m.Nc && ctl[w.x].active && ctl[w.x].iters > 0) v = (double)A.x[A.pmode ? A.inv[i] : i] * A.fq[i];
  v = block_reduce<0>(v, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = v;
}

__global__ void k_fcg_p(const SlotDesc* __restrict__ slots, const LevDesc* __restrict__ levTab, int ns,
                        const int2* __restrict__ work, const SolveCtl* __restrict__ ctl,
                        const double* __restrict__ zq, const double2* __restrict__ pqr) {
  pdl_trigger();  // a chained launch of the solve loops (see launch_k): start early, then
  pdl_wait();     // wait for the kernel before it
  const int2 w = work[blockIdx.x];
  const SolveCtl c = ctl[w.x];
  if (!c.active) return;
  const SlotDesc& S = slots[w.x];
  const LevDesc& A = LEV(0, w.x);
  const int i = w.y * blockDim.x + threadIdx.x;
  if (i >= S.m.Nc) return;
  const double z = (double)A.x[A.pmode ? A.inv[i] : i];
  if (c.iters == 0) {
    A.fp[i] = z;
  } else {
    const double pq = pqr[w.x].x;
    const double beta = pq > 0.0 ? zq[w.x] / pq : 0.0;
    A.fp[i] = z - beta * A.fp[i];
  }
}

__global__ void k_fcg_q(const SlotDesc* __restrict__ slots, const LevDesc* __restrict__ levTab, int ns,
                        const int2* __restrict__ work, const SolveCtl* __restrict__ ctl, double2* part) {
  pdl_trigger();  // a chained launch of the solve loops (see launch_k): start early, then
  pdl_wait();     // wait for the kernel before it
  __shared__ double sh[32];
  const int2 w = work[blockIdx.x];
  const SlotDesc& S = slots[w.x];
  const LevDesc& A = LEV(0, w.x);
  const int i = w.y * blockDim.x + threadIdx.x;
  double pq = 0.0, pr = 0.0;
  if (i < S.m.Nc && ctl[w.x].active) {
    const int* rp = S.m.rowptr;
    const double pi = A.fp[i];
    double q = S.ac[i] * pi;
    for (int k = rp[i]; k < rp[i + 1]; ++k) q = q + S.anb[k] * A.fp[S.m.col[k]];
    A.fq[i] = q;
    pq = pi * q;
    pr = pi * A.fr[i];
  }
  pq = block_reduce<0>(pq, sh);
  pr = block_reduce<0>(pr, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = make_double2(pq, pr);
}

__global__ void k_fcg_update(const SlotDesc* __restrict__ slots, const LevDesc* __restrict__ levTab, int ns,
                             const int2* __restrict__ work, const SolveCtl* __restrict__ ctl,
                             const double2* __restrict__ pqr, double* part) {
  pdl_trigger();  // a chained launch of the solve loops (see launch_k): start early, then
  pdl_wait();     // wait for the kernel before it
  __shared__ double sh[32];
  const int2 w = work[blockIdx.x];
  const SlotDesc& S = slots[w.x];
  const LevDesc& A = LEV(0, w.x);
  const int i = w.y * blockDim.x + threadIdx.x;
  double v = 0.0;
  if (i < S.m.Nc && ctl[w.x].active) {
    const double2 d = pqr[w.x];
    const double alpha = d.x > 0.0 ? d.y / d.x : 0.0;
    S.dphi[i] = S.dphi[i] + alpha * A.fp[i];
    const double r = A.fr[i] - alpha * A.fq[i];
    A.fr[i] = r;
    const int j = A.pmode ? A.inv[i] : i;
    A.bc[j] = (float)r;
    A.x[j] = 0.0f;
    v = fabs(r);
  }
  v = block_reduce<0>(v, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = v;
}

// FP64 multicolour GS row update on level 0 (rows of one colour)
__global__ void k_mc64(const SlotDesc* __restrict__ slots, const LevDesc* __restrict__ levTab, int ns,
                       const int2* __restrict__ work, int color, const SolveCtl* __restrict__ ctl) {
  const int2 w = work[blockIdx.x];
  if (!ctl[w.x].active) return;
  const SlotDesc& S = slots[w.x];
  const LevDesc& A = LEV(0, w.x);
  if (color >= A.ncolor) return;
  const int s0 = A.colorStart[color], cnt = A.colorStart[color + 1] - s0;
  const int t = w.y * blockDim.x + threadIdx.x;
  if (t >= cnt) return;
  if (A.pmode) {
    const int p = s0 + t;
    A.uX[p] = urow_sum(A, p, A.uBc[p]) / A.uAc[p];
    return;
  }
  const int i = A.colorRows[s0 + t];
  const int* rp = S.m.rowptr;
  double v = S.bc[i];
  for (int k = rp[i]; k < rp[i + 1]; ++k) v = v - S.anb[k] * S.dphi[S.m.col[k]];
  S.dphi[i] = v / S.ac[i];
}

// One colour of the FP64 U Gauss-Seidel from self-contained work items (the ELL copy of the
// momentum matrix; same row arithmetic as k_mc64).
// The colour kernels of a sweep are chained as programmatic dependent launches (every colour
// launch but a sweep's first, see `launch_colour`): a kernel may start while the colour before it
// runs. It loads what no colour kernel writes (its item, the active flag, the row's entries, bc
// and ac) and then waits (griddepcontrol.wait: the previous kernel has completed and its writes
// are visible) before it gathers x. Every thread waits, also one with no row, so that no colour
// kernel completes before the one it follows; the kernel after a sweep is launched the ordinary
// way and so starts after all of them. A launch without the attribute passes the wait at once;
// the two give the same bits.

__global__ void k_mc64_items(const U0Item* __restrict__ items, const SolveCtl* __restrict__ ctl) {
  pdl_trigger();
  const U0Item& it = items[blockIdx.x];
  const int t = threadIdx.x;
  if (t >= it.cnt || !ctl[it.slot].active) return pdl_wait();
  const int p = it.p0 + t;
  const size_t n = (size_t)it.n;
  const int W = it.W;
  int c[kEllUnroll];
  double a[kEllUnroll];
#pragma unroll
  for (int k = 0; k < kEllUnroll; ++k) {
    c[k] = k < W ? it.ellCol[k * n + p] : -1;
    a[k] = k < W ? it.anb[k * n + p] : 0.0;
  }
  double v = it.bc[p];
  const double d = it.ac[p];
  pdl_wait();
  double xv[kEllUnroll];
#pragma unroll
  for (int k = 0; k < kEllUnroll; ++k) xv[k] = c[k] >= 0 ? it.x[c[k]] : 0.0;
#pragma unroll
  for (int k = 0; k < kEllUnroll; ++k)
    if (c[k] >= 0) v = v - a[k] * xv[k];
  it.x[p] = v / d;
}

// sum |r| block partials of the U system from self-contained items (wc order; the same row
// values and block sums as k_res64_abs on the ELL copy)
__global__ void k_res64_items(const U0Item* __restrict__ items, const SolveCtl* __restrict__ ctl, double* part) {
  pdl_trigger();  // a chained launch of the solve loops (see launch_k): start early, then
  pdl_wait();     // wait for the kernel before it
  __shared__ double sh[32];
  const U0Item& it = items[blockIdx.x];
  const int t = threadIdx.x;
  double v = 0.0;
  if (t < it.cnt && ctl[it.slot].active) {
    const int p = it.p0 + t;
    const size_t n = (size_t)it.n;
    const int W = it.W;
    int c[kEllUnroll];
    double a[kEllUnroll];
#pragma unroll
    for (int k = 0; k < kEllUnroll; ++k) {
      c[k] = k < W ? it.ellCol[k * n + p] : -1;
      a[k] = k < W ? it.anb[k * n + p] : 0.0;
    }
    double r = it.bc[p] - it.ac[p] * it.x[p];
    double xv[kEllUnroll];
#pragma unroll
    for (int k = 0; k < kEllUnroll; ++k) xv[k] = c[k] >= 0 ? it.x[c[k]] : 0.0;
#pragma unroll
    for (int k = 0; k < kEllUnroll; ++k)
      if (c[k] >= 0) r = r - a[k] * xv[k];
    v = fabs(r);
  }
  v = block_reduce<0>(v, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = v;
}

// per-slot sums of block partials (fixed order)
__global__ void k_slot_sum(const int* __restrict__ ws, const int* __restrict__ we, const double* __restrict__ part,
                           double* out) {
  pdl_trigger();  // a chained launch of the solve loops (see launch_k): start early, then
  pdl_wait();     // wait for the kernel before it
  __shared__ double sh[32];
  const int s = blockIdx.x;
  double v = 0.0;
  for (int k = ws[s] + (int)threadIdx.x; k < we[s]; k += blockDim.x) v = v + part[k];
  v = block_reduce<0>(v, sh);
  if (threadIdx.x == 0) out[s] = v;
}

__global__ void k_slot_sum2(const int* __restrict__ ws, const int* __restrict__ we,
                            const double2* __restrict__ part, double2* out) {
  pdl_trigger();  // a chained launch of the solve loops (see launch_k): start early, then
  pdl_wait();     // wait for the kernel before it
  __shared__ double sh[32];
  const int s = blockIdx.x;
  double a = 0.0, b = 0.0;
  for (int k = ws[s] + (int)threadIdx.x; k < we[s]; k += blockDim.x) { a = a + part[k].x; b = b + part[k].y; }
  a = block_reduce<0>(a, sh);
  b = block_reduce<0>(b, sh);
  if (threadIdx.x == 0) out[s] = make_double2(a, b);
}

// stopping rule of cfdSolveAlgebraicSystem / cfdApplyAMG, per slot
// In a captured tick the same kernel also sets the condition of the solve's while node, so
// the loop ends on the device once no slot is active.
__global__ void k_ctrl(const SlotDesc* __restrict__ slots, int ns, const double* __restrict__ sums, SolveCtl* ctl,
                       int first, int max_iter, double rrf, int divide_n, int r0_slot, int r1_slot, int* any,
                       int set_cond, cudaGraphConditionalHandle cond, unsigned long long* loops, int which) {
  pdl_trigger();  // a chained launch of the solve loops (see launch_k): start early, then
  pdl_wait();     // wait for the kernel before it
  __shared__ int sany;
  if (threadIdx.x == 0) sany = 0;
  __syncthreads();
  for (int s = threadIdx.x; s < ns; s += blockDim.x) {
    const double v = divide_n ? sums[s] / slots[s].m.Nc : sums[s];
    SolveCtl c = ctl[s];
    if (first) {
      c.r0 = v; c.r1 = v; c.iters = 0;
      c.active = (0 < max_iter && v > rrf * v) ? 1 : 0;
    } else if (c.active) {
      c.r1 = v;
      c.iters += 1;
      c.active = (c.iters < max_iter && v > rrf * c.r0) ? 1 : 0;
    }
    ctl[s] = c;
    slots[s].scal[r0_slot] = c.r0;
    slots[s].scal[r1_slot] = c.r1;
    if (r1_slot == SCAL_P_R1) slots[s].scal[SCAL_CYC] = c.iters;
    if (c.active) atomicOr(&sany, 1);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    *any = sany;
    if (!first) loops[which] += 1ull;
    if (set_cond) cudaGraphSetConditional(cond, sany ? 1u : 0u);
  }
}

__global__ void k_copy_scal(const SlotDesc* __restrict__ slots, int ns, int from, int to) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < ns) slots[s].scal[to] = slots[s].scal[from];
}

__global__ void k_set_active(SolveCtl* ctl, int ns) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < ns) ctl[s].active = 1;
}

// ---------------------------------------------------------------- FP32 AMG kernels
// Galerkin by summation from level l into level l+1 (assembleAgglomeratedLHS.m:16-30 order).
// One thread per coarse row. A row of at most kGalW entries is accumulated in shared memory
// (thread t's entry k at [k * kBlock + t]) and written once at the end; a wider row is
// accumulated in place in global memory. Either way each coarse entry starts at 0.0 and takes
// its fine entries in the same order: same bits.
constexpr int kGalW = 16;
__global__ void __launch_bounds__(kBlock) k_galerkin_b(const LevDesc* __restrict__ levTab, int ns, int l,
                                                       const int2* __restrict__ work,
                                                       const SolveCtl* __restrict__ ctl) {
  __shared__ double acc[kGalW * kBlock];
  const int2 w = work[blockIdx.x];
  if (!ctl[w.x].active) return;
  const LevDesc& F = LEV(l, w.x);
  const LevDesc& C = LEV(l + 1, w.x);
  const int P = w.y * blockDim.x + threadIdx.x;
  if (P >= C.n) return;
  const int c0 = C.rowptr[P], c1 = C.rowptr[P + 1];
  if (c1 - c0 <= kGalW && F.gpos) {
    double* a = acc + threadIdx.x;
    for (int t = 0; t < c1 - c0; ++t) a[t * kBlock] = 0.0;
    double AC = 0.0;
    for (int q = F.childStart[P]; q < F.childStart[P + 1]; ++q) {
      const int c = F.child[q];
      AC = AC + F.ac64[c];
      for (int k = F.rowptr[c]; k < F.rowptr[c + 1]; ++k) {
        const int pos = F.gpos[k];  // -1 inside the aggregate, else the coarse entry
        const double v = F.anb64[k];
        if (pos == -1) AC = AC + v;
        else if (pos >= 0) a[(pos - c0) * kBlock] = a[(pos - c0) * kBlock] + v;
      }
    }
    for (int t = 0; t < c1 - c0; ++t) C.anb64[c0 + t] = a[t * kBlock];
    C.ac64[P] = AC;
    return;
  }
  for (int t = c0; t < c1; ++t) C.anb64[t] = 0.0;
  double AC = 0.0;
  for (int q = F.childStart[P]; q < F.childStart[P + 1]; ++q) {
    const int c = F.child[q];
    AC = AC + F.ac64[c];
    for (int k = F.rowptr[c]; k < F.rowptr[c + 1]; ++k) {
      int pos;
      if (F.gpos) {
        pos = F.gpos[k];  // precomputed: -1 inside the aggregate, else the coarse entry
      } else {
        const int Q = F.parents[F.col[k]];
        pos = -1;
        if (Q != P) {
          pos = c0;
          while (pos < c1 && C.col[pos] != Q) ++pos;
          if (pos == c1) pos = -2;
        }
      }
      if (pos == -1) AC = AC + F.anb64[k];
      else if (pos >= 0) C.anb64[pos] = C.anb64[pos] + F.anb64[k];
    }
  }
  C.ac64[P] = AC;
}

// ---- FP32 levels of the V-cycle. Every level except a case's coarsest is stored colour-
// permuted in ELL form (pmode 1): position p holds row perm[p], rows of one colour are
// contiguous, entry k of position p sits at [k * n + p] with its column as a position. The row
// arrays are then read with unit stride, every entry's column and coefficient are coalesced
// across the warp, and the only dependent load is the neighbour x. Each row keeps the CSR
// (cconn) order of its entries. A level in natural CSR form (pmode 0) is the coarsest level,
// or level 0 of a case without a hierarchy.

// FP32 copy of a level's FP64 matrix in its storage form (every p solve)
__global__ void k_lev_to32(const LevDesc* __restrict__ levTab, int ns, int l, const int2* __restrict__ work,
                           const SolveCtl* __restrict__ ctl) {
  const int2 w = work[blockIdx.x];
  if (!ctl[w.x].active) return;
  const LevDesc& A = LEV(l, w.x);
  const int p = w.y * blockDim.x + threadIdx.x;
  if (p >= A.n) return;
  if (!A.pmode) {
    A.ac[p] = (float)A.ac64[p];
    for (int k = A.rowptr[p]; k < A.rowptr[p + 1]; ++k) A.anb[k] = (float)A.anb64[k];
    return;
  }
  const int i = A.perm[p], k0 = A.rowptr[i], deg = A.rowptr[i + 1] - k0;
  A.ac[p] = (float)A.ac64[i];
  for (int k = 0; k < A.ellW; ++k) A.ellAnb[(size_t)k * A.n + p] = k < deg ? (float)A.anb64[k0 + k] : 0.0f;
}

// v - sum_k anb_k x_k over the row's entries in order. In ELL form and up to kEllUnroll
// entries, the column and coefficient loads are all issued before the first neighbour gather.
__device__ __forceinline__ float row_sum32(const LevDesc& A, int p, float v) {
  if (!A.pmode) {
    for (int k = A.rowptr[p]; k < A.rowptr[p + 1]; ++k) v = v - A.anb[k] * A.x[A.col[k]];
    return v;
  }
  const int W = A.ellW;
  const size_t n = (size_t)A.n;
  if (W <= kEllUnroll) {
    int c[kEllUnroll];
    float a[kEllUnroll];
#pragma unroll
    for (int k = 0; k < kEllUnroll; ++k) {
      c[k] = k < W ? A.ellCol[k * n + p] : -1;
      a[k] = k < W ? A.ellAnb[k * n + p] : 0.0f;
    }
    float xv[kEllUnroll];
#pragma unroll
    for (int k = 0; k < kEllUnroll; ++k) xv[k] = c[k] >= 0 ? A.x[c[k]] : 0.0f;
#pragma unroll
    for (int k = 0; k < kEllUnroll; ++k)
      if (c[k] >= 0) v = v - a[k] * xv[k];
    return v;
  }
  for (int k = 0; k < W; ++k) {
    const int c = A.ellCol[k * n + p];
    if (c < 0) break;
    v = v - A.ellAnb[k * n + p] * A.x[c];
  }
  return v;
}

// storage index of the t-th row of colour c
__device__ __forceinline__ int color_row(const LevDesc& A, int c, int t) {
  const int q = A.colorStart[c] + t;
  return A.pmode ? q : A.colorRows[q];
}

// one Gauss-Seidel update of row (storage index) p
__device__ __forceinline__ void gs_row32(const LevDesc& A, int p) {
  A.x[p] = row_sum32(A, p, A.bc[p]) / A.ac[p];
}

__device__ __forceinline__ void res_row32(const LevDesc& A, int p) {
  A.r[p] = row_sum32(A, p, A.bc[p] - A.ac[p] * A.x[p]);
}

// restriction into coarse storage index P of the next level (children in their original order)
__device__ __forceinline__ void restrict_row32(const LevDesc& F, const LevDesc& C, int P) {
  float v = 0.0f;
  if (F.pmode) {
    for (int q = F.childStartP[P]; q < F.childStartP[P + 1]; ++q) v = v + F.r[F.childP[q]];
  } else {
    for (int q = F.childStart[P]; q < F.childStart[P + 1]; ++q) v = v + F.r[F.child[q]];
  }
  C.bc[P] = v;
  C.x[P] = 0.0f;
}

// The same restriction with each child's residual formed in place (the same operations as
// res_row32, so the same values) instead of read back from F.r: used where nothing else reads
// F.r, it saves a pass over the level and the barrier between the two.
__device__ __forceinline__ void restrict_res_row32(const LevDesc& F, const LevDesc& C, int P) {
  float v = 0.0f;
  if (F.pmode) {
    for (int q = F.childStartP[P]; q < F.childStartP[P + 1]; ++q) {
      const int p = F.childP[q];
      v = v + row_sum32(F, p, F.bc[p] - F.ac[p] * F.x[p]);
    }
  } else {
    for (int q = F.childStart[P]; q < F.childStart[P + 1]; ++q) {
      const int p = F.child[q];
      v = v + row_sum32(F, p, F.bc[p] - F.ac[p] * F.x[p]);
    }
  }
  C.bc[P] = v;
  C.x[P] = 0.0f;
}

__device__ __forceinline__ void prolong_row32(const LevDesc& F, const LevDesc& C, int p) {
  F.x[p] = F.x[p] + F.pw * C.x[F.pmode ? F.parentsP[p] : F.parents[p]];
}

// One colour of a level-0 Gauss-Seidel sweep from self-contained work items: the item carries
// the row range and the level's array pointers, so the only loads before the row data are the
// item and the case's active flag (issued together).
__global__ void k_mc32_l0(const L0Item* __restrict__ items, const SolveCtl* __restrict__ ctl) {
  pdl_trigger();
  const L0Item& it = items[blockIdx.x];
  const int t = threadIdx.x;
  if (t >= it.cnt || !ctl[it.slot].active) return pdl_wait();
  const int p = it.p0 + t;
  const size_t n = (size_t)it.n;
  const int W = it.W;
  int c[kEllUnroll];
  float a[kEllUnroll];
#pragma unroll
  for (int k = 0; k < kEllUnroll; ++k) {
    c[k] = k < W ? it.ellCol[k * n + p] : -1;
    a[k] = k < W ? it.ellAnb[k * n + p] : 0.0f;
  }
  float v = it.bc[p];
  const float d = it.ac[p];
  pdl_wait();
  float xv[kEllUnroll];
#pragma unroll
  for (int k = 0; k < kEllUnroll; ++k) xv[k] = c[k] >= 0 ? it.x[c[k]] : 0.0f;
#pragma unroll
  for (int k = 0; k < kEllUnroll; ++k)
    if (c[k] >= 0) v = v - a[k] * xv[k];
  it.x[p] = v / d;
}

// One colour of a Gauss-Seidel sweep (a grid level), chained like k_mc32_l0.
__global__ void k_mc32(const LevDesc* __restrict__ levTab, int ns, int l, const int2* __restrict__ work, int color,
                       const SolveCtl* __restrict__ ctl) {
  pdl_trigger();
  const int2 w = work[blockIdx.x];
  if (!ctl[w.x].active) return pdl_wait();
  const LevDesc& A = LEV(l, w.x);
  if (color >= A.ncolor) return pdl_wait();
  const int t = w.y * blockDim.x + threadIdx.x;
  if (t >= A.colorStart[color + 1] - A.colorStart[color]) return pdl_wait();
  const int p = color_row(A, color, t);
  if (!A.pmode || A.ellW > kEllUnroll) {
    pdl_wait();
    gs_row32(A, p);
    return;
  }
  // gs_row32 / row_sum32 on an ELL row of at most kEllUnroll entries, with the loads that do not
  // read x before the wait: the same operations in the same order
  const int W = A.ellW;
  const size_t n = (size_t)A.n;
  int c[kEllUnroll];
  float a[kEllUnroll];
#pragma unroll
  for (int k = 0; k < kEllUnroll; ++k) {
    c[k] = k < W ? A.ellCol[k * n + p] : -1;
    a[k] = k < W ? A.ellAnb[k * n + p] : 0.0f;
  }
  float v = A.bc[p];
  const float d = A.ac[p];
  pdl_wait();
  float xv[kEllUnroll];
#pragma unroll
  for (int k = 0; k < kEllUnroll; ++k) xv[k] = c[k] >= 0 ? A.x[c[k]] : 0.0f;
#pragma unroll
  for (int k = 0; k < kEllUnroll; ++k)
    if (c[k] >= 0) v = v - a[k] * xv[k];
  A.x[p] = v / d;
}

__global__ void k_res32(const LevDesc* __restrict__ levTab, int ns, int l, const int2* __restrict__ work,
                        const SolveCtl* __restrict__ ctl) {
  pdl_trigger();  // a chained launch of the solve loops (see launch_k): start early, then
  pdl_wait();     // wait for the kernel before it
  const int2 w = work[blockIdx.x];
  if (!ctl[w.x].active) return;
  const LevDesc& A = LEV(l, w.x);
  const int p = w.y * blockDim.x + threadIdx.x;
  if (p < A.n) res_row32(A, p);
}

__global__ void k_restrict32(const LevDesc* __restrict__ levTab, int ns, int l, const int2* __restrict__ work,
                             const SolveCtl* __restrict__ ctl) {
  pdl_trigger();  // a chained launch of the solve loops (see launch_k): start early, then
  pdl_wait();     // wait for the kernel before it
  const int2 w = work[blockIdx.x];
  if (!ctl[w.x].active) return;
  const LevDesc& F = LEV(l, w.x);
  const LevDesc& C = LEV(l + 1, w.x);
  const int P = w.y * blockDim.x + threadIdx.x;
  if (P < C.n) restrict_row32(F, C, P);
}

__global__ void k_prolong32(const LevDesc* __restrict__ levTab, int ns, int l, const int2* __restrict__ work,
                            const SolveCtl* __restrict__ ctl) {
  pdl_trigger();  // a chained launch of the solve loops (see launch_k): start early, then
  pdl_wait();     // wait for the kernel before it
  const int2 w = work[blockIdx.x];
  if (!ctl[w.x].active) return;
  const LevDesc& F = LEV(l, w.x);
  const LevDesc& C = LEV(l + 1, w.x);
  const int p = w.y * blockDim.x + threadIdx.x;
  if (p < F.n) prolong_row32(F, C, p);
}

// Coarsest level of each slot (at most kDense rows): its FP64 solution operator X, with
// x = X b, is formed once per p solve by Gauss-Jordan elimination with partial pivoting of
// [M | I]; a pivot that vanishes (the pure-Neumann pressure operator is singular) pins that
// unknown to zero, so X is the linear map of the pinned elimination. Every V-cycle then
// applies X with one dense product. Coarsest levels above kDense rows (reached only when
// max_coarse_levels stops the hierarchy early) get 40 FP64 Gauss-Seidel sweeps instead.
constexpr int kDense = 64;
constexpr int kDenseLd = kDense + 1;
struct DenseFactorSmem {
  double M[kDense][kDenseLd];
  double X[kDense][kDenseLd];
  double f[kDense];
  double red[32];
  int pinned[kDense];
  int piv_row;
};

__global__ void __launch_bounds__(1024) k_coarse_factor(const LevDesc* __restrict__ levTab, int ns,
                                                        const int* __restrict__ coarsest, double* cinv) {
  extern __shared__ __align__(16) unsigned char dsm_raw[];
  DenseFactorSmem& sm = *reinterpret_cast<DenseFactorSmem*>(dsm_raw);
  const int s = blockIdx.x;
  const LevDesc& A = LEV(coarsest[s], s);
  const int n = A.n;
  if (n > kDense) return;
  for (int t = threadIdx.x; t < kDense * kDense; t += blockDim.x) {
    const int i = t / kDense, j = t % kDense;
    sm.M[i][j] = 0.0;
    sm.X[i][j] = i == j ? 1.0 : 0.0;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    sm.M[i][i] = A.ac64[i];
    for (int k = A.rowptr[i]; k < A.rowptr[i + 1]; ++k) sm.M[i][A.col[k]] = A.anb64[k];
    sm.pinned[i] = 0;
  }
  __syncthreads();
  double mx = 0.0;
  for (int t = threadIdx.x; t < n * n; t += blockDim.x) mx = fmax(mx, fabs(sm.M[t / n][t % n]));
  const double scale = block_reduce<1>(mx, sm.red);
  __shared__ double s_scale;
  if (threadIdx.x == 0) s_scale = scale;
  __syncthreads();
  for (int k = 0; k < n; ++k) {
    if (threadIdx.x < 32) {
      // partial pivoting: the first row of the largest |M[i][k]|, i >= k (each lane takes rows
      // k + lane, k + lane + 32, ... in order, then the lanes' bests are merged preferring the
      // lower row on equal values: the row a sequential search would pick)
      const int lane = threadIdx.x;
      int p = -1;
      double best = 0.0;
      for (int i = k + lane; i < n; i += 32) {
        const double v = fabs(sm.M[i][k]);
        if (p < 0 || v > best) { best = v; p = i; }
      }
      for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_down_sync(0xffffffffu, best, o);
        const int op = __shfl_down_sync(0xffffffffu, p, o);
        if (op >= 0 && (p < 0 || ob > best || (ob == best && op < p))) { best = ob; p = op; }
      }
      if (lane == 0) {
        sm.piv_row = p;
        if (best <= 1e-9 * s_scale) sm.pinned[k] = 1;
      }
    }
    __syncthreads();
    if (sm.pinned[k]) continue;  // uniform across the block
    const int p = sm.piv_row;
    if (p != k)
      for (int j = threadIdx.x; j < 2 * n; j += blockDim.x) {
        double* rk = j < n ? &sm.M[k][j] : &sm.X[k][j - n];
        double* rp = j < n ? &sm.M[p][j] : &sm.X[p][j - n];
        const double t = *rk; *rk = *rp; *rp = t;
      }
    __syncthreads();
    for (int i = k + 1 + threadIdx.x; i < n; i += blockDim.x) sm.f[i] = sm.M[i][k] / sm.M[k][k];
    __syncthreads();
    const int rows = n - k - 1;
    for (int t = threadIdx.x; t < rows * 2 * n; t += blockDim.x) {
      const int i = k + 1 + t / (2 * n), j = t % (2 * n);
      if (j < n) {
        if (j >= k) sm.M[i][j] -= sm.f[i] * sm.M[k][j];
      } else {
        sm.X[i][j - n] -= sm.f[i] * sm.X[k][j - n];
      }
    }
    __syncthreads();
  }
  // back substitution of every column of X
  for (int k = n - 1; k >= 0; --k) {
    for (int c = threadIdx.x; c < n; c += blockDim.x) {
      double v = 0.0;
      if (!sm.pinned[k]) {
        v = sm.X[k][c];
        for (int j = k + 1; j < n; ++j) v -= sm.M[k][j] * sm.X[j][c];
        v /= sm.M[k][k];
      }
      sm.X[k][c] = v;
    }
    __syncthreads();
  }
  double* out = cinv + (size_t)s * kDense * kDense;
  for (int t = threadIdx.x; t < n * n; t += blockDim.x) out[t] = sm.X[t / n][t % n];
}

// Synchronisation domains of the coarse V-cycle: one CTA, or one thread group of a CTA with
// its own named barrier. tid / nth: this thread's index and the domain's thread count.
struct CtaDomain {
  int tid, nth;
  __device__ void sync() const { __syncthreads(); }
};
// a 256-thread group of a CTA with its own named barrier (ids 1..4; 0 is __syncthreads)
struct GroupDomain {
  int tid, nth, bar;
  __device__ void sync() const { asm volatile("bar.sync %0, %1;" ::"r"(bar), "r"(nth) : "memory"); }
};

template <class D>
__device__ void coarse_apply(const LevDesc& A, const double* __restrict__ X, const D& d) {
  const int n = A.n;
  if (n > kDense) {
    if (d.tid == 0) {
      for (int sweep = 0; sweep < 40; ++sweep)
        for (int pass = 0; pass < 2; ++pass)
          for (int q = 0; q < n; ++q) {
            const int i = pass == 0 ? q : n - 1 - q;
            double v = A.bc[i];
            for (int k = A.rowptr[i]; k < A.rowptr[i + 1]; ++k) v -= A.anb64[k] * (double)A.x[A.col[k]];
            A.x[i] = (float)(v / A.ac64[i]);
          }
    }
    d.sync();
    return;
  }
  // b is read in full before any x is written (A.bc and A.x are distinct arrays)
  for (int i = d.tid; i < n; i += d.nth) {
    double v = 0.0;
    for (int j = 0; j < n; ++j) v += X[(size_t)i * n + j] * (double)A.bc[j];
    A.x[i] = (float)v;
  }
  d.sync();
}

// A symmetric multicolour sweep runs the colours forward and then backward. The backward pass
// starts at colour C-1, which the forward pass has just updated from the same neighbour values
// (rows of one colour are not coupled, and a row's update x = (b - sum anb x_nb) / a does not
// read its own x), so that update would write the same bits again: every sweep below skips it.
// Before the barrier that ends a colour, each thread asks L1 for what its first row of the next
// colour reads apart from x (the ELL entries, bc, ac: none of them changes while the level is
// smoothed), so that after the barrier only the neighbour gathers wait on memory.
__device__ __forceinline__ void prefetch_l1(const void* p) {
  asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}
__device__ __forceinline__ void prefetch_row32(const LevDesc& A, int c, int t) {
  if (!A.pmode || t >= A.colorStart[c + 1] - A.colorStart[c]) return;
  const int p = A.colorStart[c] + t;
  const size_t n = (size_t)A.n;
  for (int k = 0; k < A.ellW; ++k) {
    prefetch_l1(A.ellCol + k * n + p);
    prefetch_l1(A.ellAnb + k * n + p);
  }
  prefetch_l1(A.bc + p);
  prefetch_l1(A.ac + p);
}

template <class D>
__device__ void smooth_dom(const LevDesc& A, int sweeps, const D& d) {
  for (int sw = 0; sw < sweeps; ++sw)
    for (int pass = 0; pass < 2; ++pass)
      for (int q = pass; q < A.ncolor; ++q) {
        const int c = pass == 0 ? q : A.ncolor - 1 - q;
        const int cnt = A.colorStart[c + 1] - A.colorStart[c];
        for (int t = d.tid; t < cnt; t += d.nth) gs_row32(A, color_row(A, c, t));
        // the colour after this one: the next in this pass, or the first of the next pass
        int cn = -1;
        if (pass == 0) cn = q + 1 < A.ncolor ? q + 1 : (A.ncolor >= 2 ? A.ncolor - 2 : -1);
        else if (q + 1 < A.ncolor) cn = A.ncolor - 2 - q;
        else if (sw + 1 < sweeps) cn = 0;
        if (cn >= 0) prefetch_row32(A, cn, d.tid);
        d.sync();
      }
}

// Levels g .. coarsest of slot s: descend with pre-smoothing, residual and restriction; apply
// the coarsest operator; ascend with prolongation and post-smoothing. Every thread of the
// domain takes the same path (the loops depend on the slot only), so the barriers match.
template <class D>
__device__ void vcycle_levels(const LevDesc* __restrict__ levTab, int ns, int s, int L, int g,
                              const double* __restrict__ cinv, int pre, int post, const D& d) {
  for (int l = g; l < L; ++l) {
    const LevDesc& A = LEV(l, s);
    const LevDesc& C = LEV(l + 1, s);
    smooth_dom(A, pre, d);
    for (int P = d.tid; P < C.n; P += d.nth) restrict_res_row32(A, C, P);
    d.sync();
  }
  coarse_apply(LEV(L, s), cinv + (size_t)s * kDense * kDense, d);
  for (int l = L - 1; l >= g; --l) {
    const LevDesc& A = LEV(l, s);
    const LevDesc& C = LEV(l + 1, s);
    for (int p = d.tid; p < A.n; p += d.nth) prolong_row32(A, C, p);
    d.sync();
    smooth_dom(A, post, d);
  }
}

// The small-level part of the V-cycle, one CTA per slot (levels g .. coarsest, where g is the
// first level of the slot small enough for this kernel; larger levels run as grid-wide
// launches). A slot whose coarsest level is 0 gets its direct solve on level 0 here.
__global__ void __launch_bounds__(1024, 2) k_coarse_vcycle(const LevDesc* __restrict__ levTab, int ns,
                                                        const int* __restrict__ coarsest,
                                                        const int* __restrict__ gstart, const double* __restrict__ cinv,
                                                        int pre, int post, const SolveCtl* __restrict__ ctl,
                                                        const int* __restrict__ order) {
  pdl_trigger();  // a chained launch of the solve loops (see launch_k): start early, then
  pdl_wait();     // wait for the kernel before it
  const int s = order[blockIdx.x];
  if (!ctl[s].active) return;
  vcycle_levels(levTab, ns, s, coarsest[s], gstart[s], cinv, pre, post,
                       CtaDomain{(int)threadIdx.x, (int)blockDim.x});
}

// The same with packed CTAs: a task either gives one large slot the whole CTA, or gives each of
// its kPackGroups groups of kBlockPack / kPackGroups threads its own small slot (each group
// synchronises on its own named barrier), so that many small cases share one CTA.
__global__ void __launch_bounds__(kBlockPack, 1) k_coarse_vcycle_pk(const LevDesc* __restrict__ levTab, int ns,
                                                                   const int* __restrict__ coarsest,
                                                                   const int* __restrict__ gstart,
                                                                   const double* __restrict__ cinv, int pre, int post,
                                                                   const SolveCtl* __restrict__ ctl,
                                                                   const PackTask* __restrict__ tasks) {
  pdl_trigger();  // a chained launch of the solve loops (see launch_k): start early, then
  pdl_wait();     // wait for the kernel before it
  const PackTask& T = tasks[blockIdx.x];
  // one code path for both: a large slot is one group of the whole CTA on barrier 1
  const int gsize = T.big ? kBlockPack : kBlockPack / kPackGroups;
  const int grp = threadIdx.x / gsize;
  const int s = T.slot[grp];
  if (s < 0 || !ctl[s].active) return;  // the same decision in every thread of the group
  vcycle_levels(levTab, ns, s, coarsest[s], gstart[s], cinv, pre, post,
                       GroupDomain{(int)threadIdx.x % gsize, gsize, 1 + grp});
}

// ---------------------------------------------------------------- host side
static int upload_work(DArr<int2>& d, const std::vector<int2>& h, cudaStream_t st) {
  UFVM_CHECK(dalloc(d, std::max<size_t>(h.size(), 1)));
  if (!h.empty()) UFVM_CUDA(cudaMemcpyAsync(d.p, h.data(), h.size() * sizeof(int2), cudaMemcpyHostToDevice, st));
  return UFVM_OK;
}

template <typename T>
static int upload_vec(DArr<T>& d, const std::vector<T>& h, cudaStream_t st) {
  UFVM_CHECK(dalloc(d, std::max<size_t>(h.size(), 1)));
  if (!h.empty()) UFVM_CUDA(cudaMemcpyAsync(d.p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, st));
  return UFVM_OK;
}

// Launches inside the solve loops' bodies. A chained launch is a programmatic dependent of the
// kernel before it: it may start while that kernel runs and waits on the device (pdl_wait)
// before it touches what earlier kernels wrote. The kernels launched this way wait at their top,
// except the colour kernels (k_mc32, k_mc32_l0, k_mc64_items), which first load what no colour
// kernel writes; so a sweep's first colour is never chained (its right-hand side may come from
// the kernel just before it), and a body's first launch is never chained (it has no kernel
// before it in the body's graph).
template <typename... Exp, typename... Act>
static int launch_k(bool chained, void (*kernel)(Exp...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                    Act&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = chained ? 1 : 0;
  UFVM_CUDA(cudaLaunchKernelEx(&cfg, kernel, std::forward<Act>(args)...));
  return UFVM_OK;
}
template <typename... Exp, typename... Act>
static int launch_colour(bool chained, void (*kernel)(Exp...), int grid, cudaStream_t st, Act&&... args) {
  return launch_k(chained, kernel, dim3(grid), dim3(kBlock), 0, st, std::forward<Act>(args)...);
}

// blocks of n items for every slot passing `use`, with per-slot entry ranges
template <typename F>
static void build_list(int ns, F count, std::vector<int2>& out, std::vector<int>* st, std::vector<int>* en) {
  out.clear();
  if (st) { st->assign(ns, 0); en->assign(ns, 0); }
  for (int s = 0; s < ns; ++s) {
    const int n = count(s);
    if (st) (*st)[s] = (int)out.size();
    for (int b = 0; b < nblocks(n); ++b) out.push_back(make_int2(s, b));
    if (st) (*en)[s] = (int)out.size();
  }
}

int Service::rebuild_tables() {
  const int ns = (int)cases.size();
  if (ns == 0) { tables_dirty = false; return UFVM_OK; }
  UFVM_CHECK(dalloc(scal, (size_t)ns * SCAL_SLOT_N));
  UFVM_CHECK(dalloc(flags, (size_t)ns * FLAG_N));
  UFVM_CHECK(dalloc(uctl, ns));
  UFVM_CHECK(dalloc(pctl, ns));
  UFVM_CHECK(dalloc(anyflag, 4));
  if (!loopcnt.p) {
    UFVM_CHECK(dalloc(loopcnt, 2));
    UFVM_CUDA(cudaMemsetAsync(loopcnt.p, 0, 2 * sizeof(unsigned long long), stream));
  }
  std::vector<SlotDesc> h(ns);
  for (int s = 0; s < ns; ++s) {
    h[s] = cases[s]->desc();
    h[s].rowsU = cases[s]->rowsU;
    h[s].scal = scal.p + (size_t)s * SCAL_SLOT_N;
    h[s].flags = flags.p + (size_t)s * FLAG_N;
  }
  UFVM_CHECK(upload_vec(slotTab, h, stream));
  std::vector<int2> v;
  std::vector<int> a, b;
  build_list(ns, [&](int s) { return cases[s]->M.Nc; }, v, &a, &b);
  nwc = (int)v.size();
  UFVM_CHECK(upload_work(wc, v, stream));
  UFVM_CHECK(upload_vec(cstart, a, stream));
  UFVM_CHECK(upload_vec(cend, b, stream));
  build_list(ns, [&](int s) { return cases[s]->M.F; }, v, nullptr, nullptr);
  nwf = (int)v.size();
  UFVM_CHECK(upload_work(wf, v, stream));
  build_list(ns, [&](int s) { return cases[s]->M.Fb; }, v, nullptr, nullptr);
  nwb = (int)v.size();
  UFVM_CHECK(upload_work(wb, v, stream));
  build_list(ns, [&](int s) { return cases[s]->rowsU; }, v, &a, &b);
  nwu = (int)v.size();
  UFVM_CHECK(upload_work(wu, v, stream));
  UFVM_CHECK(upload_vec(ustart, a, stream));
  UFVM_CHECK(upload_vec(uend, b, stream));
  UFVM_CHECK(dalloc(part, 2 * (size_t)std::max(nwc, nwu) + 16));
  UFVM_CHECK(dalloc(fcg, 4 * (size_t)nwc + 4 * (size_t)ns + 16));
  // AMG tables (cases without a hierarchy yet count as one level)
  Lmax = 1;
  for (auto* c : cases) Lmax = std::max(Lmax, c->hierarchy_valid ? c->n_levels : 1);
  std::vector<LevDesc> lt((size_t)Lmax * ns);
  for (int l = 0; l < Lmax; ++l)
    for (int s = 0; s < ns; ++s) {
      LevDesc d{};
      Case& c = *cases[s];
      const int nl = c.hierarchy_valid ? c.n_levels : 1;
      if (l < nl) {
        Level& L = c.lev[l];
        d.n = L.n; d.nnz = L.nnz; d.ncolor = L.color_valid ? L.ncolor : 0; d.coarsest = (l == nl - 1);
        d.rowptr = L.rowptr.p; d.col = L.col.p; d.ac64 = L.ac.p; d.anb64 = L.anb.p;
        d.ac = L.ac32.p; d.anb = L.anb32.p; d.bc = L.bc32.p; d.x = L.dphi32.p; d.r = L.r32.p;
        d.parents = l + 1 < nl ? L.parents.p : nullptr;
        d.childStart = l + 1 < nl ? L.childStart.p : nullptr;
        d.child = l + 1 < nl ? L.child.p : nullptr;
        d.colorRows = L.colorRows.p; d.colorStart = L.colorStart.p;
        if (l == 0) { d.fr = L.fr.p; d.fp = L.fp.p; d.fq = L.fq.p; }
        d.pw = (S.p_coarse_weight > 0.0) ? (float)S.p_coarse_weight : 1.0f;
        d.pmode = (l + 1 < nl && L.ell_valid) ? 1 : 0;
        if (d.pmode) {
          d.ellW = L.ellW;
          d.perm = L.perm.p; d.inv = L.inv.p; d.ellCol = L.ellCol.p; d.ellAnb = L.ellAnb.p;
          d.parentsP = L.parentsP.p; d.childP = L.childP.p; d.childStartP = L.childStartP.p;
          if (l == 0) { d.uAnb = L.uAnb.p; d.uAc = L.uAc.p; d.uBc = L.uBc.p; d.uX = L.uX.p; }
          d.gpos = L.gpos.p;
        }
      }
      lt[(size_t)l * ns + s] = d;
    }
  UFVM_CHECK(upload_vec(levTab, lt, stream));
  wrows.resize(Lmax); nwrows.assign(Lmax, 0); wsm.resize(Lmax); nwsm.assign(Lmax, 0);
  wnc.resize(Lmax); nwnc.assign(Lmax, 0); wrc.resize(Lmax); nwrc.assign(Lmax, 0);
  maxcol.assign(Lmax, 0); smoff.assign(Lmax, {}); smcnt.assign(Lmax, {});
  auto nlev = [&](int q) { return cases[q]->hierarchy_valid ? cases[q]->n_levels : 1; };
  std::vector<int> hco(ns), hg(ns);
  maxg = 0;
  for (int q = 0; q < ns; ++q) {
    const int L = nlev(q) - 1;
    int g = 0;
    if (L > 0) {
      g = 1;
      while (g < L && cases[q]->lev[g].n > cta_rows) ++g;
    }
    hco[q] = L;
    hg[q] = g;
    maxg = std::max(maxg, g);
  }
  UFVM_CHECK(upload_vec(dcoarsest, hco, stream));
  UFVM_CHECK(upload_vec(dgstart, hg, stream));
  h_coarsest = hco;
  h_gstart = hg;
  {  // CTA order of the coarse V-cycle: the cases with the most rows below the grid levels first
    std::vector<long long> work_rows(ns, 0);
    for (int q = 0; q < ns; ++q)
      for (int l = hg[q]; l <= hco[q]; ++l) work_rows[q] += cases[q]->lev[l].n;
    std::vector<int> order(ns);
    for (int q = 0; q < ns; ++q) order[q] = q;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return work_rows[a] > work_rows[b]; });
    UFVM_CHECK(upload_vec(dcta_order, order, stream));
    // packed tasks: a slot with more than pk_rows rows below its grid levels gets a whole CTA,
    // the others are packed kPackGroups to a CTA (largest first)
    std::vector<PackTask> tasks;
    PackTask cur{};
    int fill = 0;
    for (int q : order) {
      if (work_rows[q] > pk_rows) {
        PackTask t{};
        t.big = 1;
        for (int k = 0; k < kPackGroups; ++k) t.slot[k] = -1;
        t.slot[0] = q;
        tasks.push_back(t);
        continue;
      }
      if (fill == 0) {
        cur = PackTask{};
        cur.big = 0;
        for (int k = 0; k < kPackGroups; ++k) cur.slot[k] = -1;
      }
      cur.slot[fill++] = q;
      if (fill == kPackGroups) { tasks.push_back(cur); fill = 0; }
    }
    if (fill) tasks.push_back(cur);
    npk_tasks = (int)tasks.size();
    UFVM_CHECK(upload_vec(dpk_tasks, tasks, stream));
  }
  UFVM_CHECK(dalloc(cinv, (size_t)ns * kDense * kDense));
  for (int l = 0; l < Lmax; ++l) {
    build_list(ns, [&](int q) { return l < nlev(q) ? cases[q]->lev[l].n : 0; }, v, nullptr, nullptr);
    nwrows[l] = (int)v.size();
    UFVM_CHECK(upload_work(wrows[l], v, stream));
    build_list(ns, [&](int q) { return l < hg[q] ? cases[q]->lev[l].n : 0; }, v, nullptr, nullptr);
    nwnc[l] = (int)v.size();
    UFVM_CHECK(upload_work(wnc[l], v, stream));
    build_list(ns, [&](int q) { return l < hg[q] ? cases[q]->lev[l + 1].n : 0; }, v, nullptr, nullptr);
    nwrc[l] = (int)v.size();
    UFVM_CHECK(upload_work(wrc[l], v, stream));
    // smoothing lists: rows of each colour for slots with l < g
    int mc = 0;
    for (int q = 0; q < ns; ++q)
      if (l < hg[q] && cases[q]->lev[l].color_valid) mc = std::max(mc, cases[q]->lev[l].ncolor);
    maxcol[l] = mc;
    std::vector<int2> sm;
    std::vector<L0Item> sm0;
    smoff[l].assign(mc, 0); smcnt[l].assign(mc, 0);
    for (int c = 0; c < mc; ++c) {
      smoff[l][c] = (int)sm.size();
      for (int q = 0; q < ns; ++q) {
        Level& L = cases[q]->lev[l];
        if (!(l < hg[q]) || !L.color_valid || c >= L.ncolor) continue;
        const int cnt = L.h_colorStart[c + 1] - L.h_colorStart[c];
        for (int bb = 0; bb < nblocks(cnt); ++bb) {
          sm.push_back(make_int2(q, bb));
          if (l == 0 && L.ell_valid && L.ellW <= kEllUnroll) {  // self-contained level-0 item
            L0Item it{};
            it.slot = q;
            it.p0 = L.h_colorStart[c] + bb * kBlock;
            it.cnt = std::min(kBlock, cnt - bb * kBlock);
            it.n = L.n;
            it.W = L.ellW;
            it.x = L.dphi32.p; it.bc = L.bc32.p; it.ac = L.ac32.p;
            it.ellCol = L.ellCol.p; it.ellAnb = L.ellAnb.p;
            sm0.push_back(it);
          }
        }
      }
      smcnt[l][c] = (int)sm.size() - smoff[l][c];
    }
    nwsm[l] = (int)sm.size();
    UFVM_CHECK(upload_work(wsm[l], sm, stream));
    if (l == 0) {
      // the self-contained items replace the (slot, block) list only when every item has one
      l0_items = (int)sm0.size() == nwsm[0] && nwsm[0] > 0;
      if (l0_items) UFVM_CHECK(upload_vec(wsm0, sm0, stream));
    }
  }
  // level-0 colour rows of every slot (FP64 U smoother)
  ucolors = 0;
  for (auto* c : cases) ucolors = std::max(ucolors, c->lev[0].color_valid ? c->lev[0].ncolor : 0);
  std::vector<int2> uc;
  std::vector<U0Item> uci;
  ucol_off.assign(ucolors, 0); ucol_cnt.assign(ucolors, 0);
  for (int c = 0; c < ucolors; ++c) {
    ucol_off[c] = (int)uc.size();
    for (int s = 0; s < ns; ++s) {
      Case& cs = *cases[s];
      Level& L = cs.lev[0];
      if (!L.color_valid || c >= L.ncolor) continue;
      const int cnt = L.h_colorStart[c + 1] - L.h_colorStart[c];
      const bool ell = cs.hierarchy_valid && cs.n_levels > 1 && L.ell_valid && L.ellW <= kEllUnroll;
      for (int bb = 0; bb < nblocks(cnt); ++bb) {
        uc.push_back(make_int2(s, bb));
        if (ell) {
          U0Item it{};
          it.slot = s;
          it.p0 = L.h_colorStart[c] + bb * kBlock;
          it.cnt = std::min(kBlock, cnt - bb * kBlock);
          it.n = L.n;
          it.W = L.ellW;
          it.x = L.uX.p; it.bc = L.uBc.p; it.ac = L.uAc.p; it.anb = L.uAnb.p; it.ellCol = L.ellCol.p;
          uci.push_back(it);
        }
      }
    }
    ucol_cnt[c] = (int)uc.size() - ucol_off[c];
  }
  UFVM_CHECK(upload_work(wu_col, uc, stream));
  u_items = (int)uci.size() == (int)uc.size() && !uc.empty();
  if (u_items) UFVM_CHECK(upload_vec(wu_items, uci, stream));
  {  // U residual items over every slot's rows, in the order of the wc list
    std::vector<U0Item> ri;
    bool all = true;
    for (int s = 0; s < ns && all; ++s) {
      Case& cs = *cases[s];
      Level& L = cs.lev[0];
      if (!(cs.hierarchy_valid && cs.n_levels > 1 && L.ell_valid && L.ellW <= kEllUnroll)) { all = false; break; }
      for (int bb = 0; bb < nblocks(cs.M.Nc); ++bb) {
        U0Item it{};
        it.slot = s;
        it.p0 = bb * kBlock;
        it.cnt = std::min(kBlock, cs.M.Nc - bb * kBlock);
        it.n = L.n;
        it.W = L.ellW;
        it.x = L.uX.p; it.bc = L.uBc.p; it.ac = L.uAc.p; it.anb = L.uAnb.p; it.ellCol = L.ellCol.p;
        ri.push_back(it);
      }
    }
    ures_items = all && (int)ri.size() == nwc;
    if (ures_items) UFVM_CHECK(upload_vec(wures_items, ri, stream));
  }
  // boundary-velocity correction modes with work (k_vel_patch): 1 symmetry / empty / slip
  // wall, 2 and 3 an outlet with fixed p
  {
    int maxp = 0;
    for (auto* c : cases) maxp = std::max(maxp, c->P.n);
    vel_mask.assign(3 * (size_t)maxp, 0);
    for (auto* c : cases)
      for (int ip = 0; ip < c->P.n; ++ip) {
        const int ty = c->P.type[ip], tp = c->P.bcP[ip];
        if (ty == UFVM_PATCH_SYMMETRY || ty == UFVM_PATCH_EMPTY || (ty == UFVM_PATCH_WALL && tp == UFVM_BC_SLIP))
          vel_mask[3 * ip + 0] = 1;
        if (ty == UFVM_PATCH_OUTLET && tp == UFVM_BC_FIXED_VALUE) vel_mask[3 * ip + 1] = vel_mask[3 * ip + 2] = 1;
      }
  }
  tables_dirty = false;
  graph_valid = false;
  UFVM_CUDA(cudaFuncSetAttribute(k_coarse_factor, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)sizeof(DenseFactorSmem)));
  return UFVM_OK;
}

BatchLaunch Service::batch() {
  BatchLaunch b{slotTab.p, wc.p, nwc, wf.p, nwf, wb.p, nwb, wu.p, nwu, cstart.p, cend.p, ustart.p, uend.p,
                (int)cases.size(), part.p, stream};
  b.vel_mask = vel_mask.empty() ? nullptr : vel_mask.data();
  return b;
}

// The reference's agglomeration of the assembled p matrix, FP32 arrays and colourings.
int Service::ensure_hierarchy(Case& c, cudaStream_t st, double* ms) {
  const long long b0 = t_dev_bytes;
  const double a0 = t_alloc_ms;
  cudaStream_t own = c.lin.stream;
  c.lin.stream = st;  // the case's scratch and solver work run on `st` for the build
  const int rc = ensure_hierarchy_(c, st, ms);
  c.lin.stream = own;
  c.dev_bytes += t_dev_bytes - b0;
  ms[3] += t_alloc_ms - a0;
  return rc;
}

// Hierarchy builds of several newly admitted cases: each case's build is a chain of small
// launches and host waits (agglomeration rounds, colourings, the host-side ELL permutation), and
// the cases are independent, so they run on up to kBuildThreads host threads, each with its own
// stream, after the assembly that produced their matrices; the service stream then waits for all
// of them. A build's result does not depend on which thread or stream ran it.
int Service::build_hierarchies(std::vector<Case*>& need) {
  if (need.empty()) return UFVM_OK;
  const double w0 = host_ms_now();
  const int nt = (int)std::min<size_t>(need.size(), kBuildThreads);
  std::vector<std::array<double, 4>> ms(std::max(nt, 1), std::array<double, 4>{0.0, 0.0, 0.0, 0.0});
  auto account = [&]() {
    for (const auto& m : ms)
      for (int k = 0; k < 4; ++k) build_ms[k] += m[k];
    build_wall_ms += host_ms_now() - w0;
  };
  if (nt <= 1) {
    for (Case* c : need) {
      const int r = ensure_hierarchy(*c, stream, ms[0].data());
      if (r != UFVM_OK) return r;
    }
    account();
    return UFVM_OK;
  }
  int dev = 0;
  UFVM_CUDA(cudaGetDevice(&dev));
  while ((int)build_streams.size() < nt) {
    cudaStream_t s2 = nullptr;
    UFVM_CUDA(cudaStreamCreateWithFlags(&s2, cudaStreamNonBlocking));
    build_streams.push_back(s2);
  }
  if (!build_event) UFVM_CUDA(cudaEventCreateWithFlags(&build_event, cudaEventDisableTiming));
  UFVM_CUDA(cudaEventRecord(build_event, stream));
  std::atomic<size_t> next{0};
  std::vector<int> rc(nt, UFVM_OK);
  std::vector<std::string> msg(nt);
  auto worker = [&](int w) {
    if (cudaSetDevice(dev) != cudaSuccess || cudaStreamWaitEvent(build_streams[w], build_event, 0) != cudaSuccess) {
      rc[w] = UFVM_E_CUDA;
      msg[w] = "a hierarchy build thread could not join the service's device or stream";
      return;
    }
    AllocStreamScope scope(build_streams[w]);  // this thread's allocations are ordered on its stream
    for (size_t k = next++; k < need.size(); k = next++) {
      const int r = ensure_hierarchy(*need[k], build_streams[w], ms[w].data());
      if (r != UFVM_OK) {
        rc[w] = r;
        msg[w] = get_error();
        return;
      }
    }
    if (cudaStreamSynchronize(build_streams[w]) != cudaSuccess) {
      rc[w] = UFVM_E_CUDA;
      msg[w] = "hierarchy build stream failed";
    }
  };
  std::vector<std::thread> th;
  for (int w = 1; w < nt; ++w) th.emplace_back(worker, w);
  worker(0);
  for (auto& t : th) t.join();
  for (int w = 0; w < nt; ++w)
    if (rc[w] != UFVM_OK) {
      set_error(msg[w]);
      return rc[w];
    }
  account();
  return UFVM_OK;
}

int Service::ensure_hierarchy_(Case& c, cudaStream_t st, double* ms) {
  c.amg->smoother = UFVM_SMOOTHER_MCGS; c.amg->quirks = c.S.quirks;
  double t0 = host_ms_now();
  UFVM_CHECK(c.amg->build(c.lev, c.S.p_max_coarse_levels, c.S.quirks, &c.n_levels));
  double t1 = host_ms_now();
  ms[0] += t1 - t0;
  for (int l = 0; l < c.n_levels; ++l) {
    Level& L = c.lev[l];
    UFVM_CHECK(dalloc(L.ac32, L.n));
    UFVM_CHECK(dalloc(L.anb32, std::max(L.nnz, 1)));
    UFVM_CHECK(dalloc(L.bc32, L.n));
    UFVM_CHECK(dalloc(L.dphi32, L.n));
    UFVM_CHECK(dalloc(L.r32, L.n));
    if (l + 1 < c.n_levels) UFVM_CHECK(build_coloring(c.lin, L));
    if (l == 0) {
      UFVM_CHECK(dalloc(L.fr, L.n));
      UFVM_CHECK(dalloc(L.fp, L.n));
      UFVM_CHECK(dalloc(L.fq, L.n));
    }
  }
  t0 = host_ms_now();
  ms[1] += t0 - t1;
  if (c.n_levels > 1) UFVM_CHECK(build_ell(c, st));
  ms[2] += host_ms_now() - t0;
  c.hierarchy_valid = true;
  return UFVM_OK;
}

// ---------------------------------------------------------------- graph capture helpers
// A captured tick is one CUDA graph, stream-captured on `stream`. Every convergence-controlled
// solve loop becomes a conditional WHILE node added to the graph being captured; its body is
// captured on a second stream into the node's body graph, and k_ctrl in the body sets the
// node's condition on the device. The node starts from its default condition 1 at every launch.
int Service::loop_begin(int kind, cudaGraphConditionalHandle* h) {
  cudaStreamCaptureStatus cs;
  cudaGraph_t cg = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  UFVM_CUDA(cudaStreamGetCaptureInfo(stream, &cs, nullptr, &cg, &deps, &nd));
  if (cs != cudaStreamCaptureStatusActive || !cg) { set_error("loop_begin outside a capture"); return UFVM_E_CUDA; }
  std::vector<cudaGraphNode_t> dv(deps, deps + nd);
  UFVM_CUDA(cudaGraphConditionalHandleCreate(h, cg, 1, cudaGraphCondAssignDefault));
  cudaGraphNodeParams np = {};
  np.type = cudaGraphNodeTypeConditional;
  np.conditional.handle = *h;
  np.conditional.type = cudaGraphCondTypeWhile;
  np.conditional.size = 1;
  cudaGraphNode_t node;
  UFVM_CUDA(cudaGraphAddNode(&node, cg, dv.empty() ? nullptr : dv.data(), dv.size(), &np));
  UFVM_CUDA(cudaStreamUpdateCaptureDependencies(stream, &node, 1, cudaStreamSetCaptureDependencies));
  cudaGraph_t body = np.conditional.phGraph_out[0];
  bodies.push_back({kind, body});
  if (!bstream) UFVM_CUDA(cudaStreamCreateWithFlags(&bstream, cudaStreamNonBlocking));
  UFVM_CUDA(cudaStreamBeginCaptureToGraph(bstream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  main_stream = stream;
  stream = bstream;  // the body's kernels are launched on the body stream
  return UFVM_OK;
}

int Service::loop_end() {
  stream = main_stream;
  cudaGraph_t g = nullptr;
  UFVM_CUDA(cudaStreamEndCapture(bstream, &g));
  return UFVM_OK;
}

// Every level but the coarsest of the FP32 V-cycle in colour-permuted ELL form (built once
// per hierarchy): rows sorted by colour, natural order inside a colour (a stable counting
// sort on the host).
int Service::build_ell(Case& c, cudaStream_t st) {
  const int nl = c.n_levels;
  if (nl < 2) return UFVM_OK;
  std::vector<std::vector<int>> perm(nl), inv(nl);
  for (int l = 0; l + 1 < nl; ++l) {
    Level& L = c.lev[l];
    L.ell_valid = false;
    if (!L.color_valid) { set_error("build_ell: level without a colouring"); return UFVM_E_INVALID; }
    const int n = L.n;
    std::vector<int> color(n);
    UFVM_CUDA(cudaMemcpyAsync(color.data(), L.color.p, n * sizeof(int), cudaMemcpyDeviceToHost, st));
    UFVM_CUDA(cudaStreamSynchronize(st));
    std::vector<int> start(L.ncolor + 1, 0);
    for (int i = 0; i < n; ++i) {
      if (color[i] < 0 || color[i] >= L.ncolor) { set_error("build_ell: row without a colour"); return UFVM_E_INVALID; }
      start[color[i] + 1]++;
    }
    for (int k = 0; k < L.ncolor; ++k) start[k + 1] += start[k];
    for (int k = 0; k <= L.ncolor; ++k)
      if (start[k] != L.h_colorStart[k]) { set_error("build_ell: colour ranges disagree"); return UFVM_E_INVALID; }
    perm[l].resize(n);
    inv[l].resize(n);
    std::vector<int> cur(start.begin(), start.end() - 1);
    for (int i = 0; i < n; ++i) perm[l][cur[color[i]]++] = i;
    for (int q = 0; q < n; ++q) inv[l][perm[l][q]] = q;
  }
  for (int l = 0; l + 1 < nl; ++l) {
    Level& L = c.lev[l];
    const Level& C = c.lev[l + 1];
    const bool cperm = l + 2 < nl;  // the next level is permuted too (it is not the coarsest)
    const int n = L.n, nnz = L.nnz, nc = C.n;
    std::vector<int> rp(n + 1), col(std::max(nnz, 1)), parents(n), cs(nc + 1), child(n);
    UFVM_CUDA(cudaMemcpyAsync(rp.data(), L.rowptr.p, (n + 1) * sizeof(int), cudaMemcpyDeviceToHost, st));
    if (nnz) UFVM_CUDA(cudaMemcpyAsync(col.data(), L.col.p, nnz * sizeof(int), cudaMemcpyDeviceToHost, st));
    UFVM_CUDA(cudaMemcpyAsync(parents.data(), L.parents.p, n * sizeof(int), cudaMemcpyDeviceToHost, st));
    UFVM_CUDA(cudaMemcpyAsync(cs.data(), L.childStart.p, (nc + 1) * sizeof(int), cudaMemcpyDeviceToHost, st));
    UFVM_CUDA(cudaMemcpyAsync(child.data(), L.child.p, n * sizeof(int), cudaMemcpyDeviceToHost, st));
    UFVM_CUDA(cudaStreamSynchronize(st));
    const std::vector<int>& P = perm[l];
    const std::vector<int>& I = inv[l];
    int W = 0;
    for (int i = 0; i < n; ++i) W = std::max(W, rp[i + 1] - rp[i]);
    std::vector<int> ell((size_t)W * n, -1), parP(n), chP, chS(nc + 1, 0);
    chP.reserve(n);
    for (int q = 0; q < n; ++q) {
      const int i = P[q];
      for (int k = rp[i]; k < rp[i + 1]; ++k) ell[(size_t)(k - rp[i]) * n + q] = I[col[k]];
      parP[q] = cperm ? inv[l + 1][parents[i]] : parents[i];
    }
    for (int Q = 0; Q < nc; ++Q) {
      const int Pn = cperm ? perm[l + 1][Q] : Q;
      for (int k = cs[Pn]; k < cs[Pn + 1]; ++k) chP.push_back(I[child[k]]);
      chS[Q + 1] = (int)chP.size();
    }
    if ((int)chP.size() != n) { set_error("build_ell: children do not cover the level"); return UFVM_E_INVALID; }
    UFVM_CHECK(upload_vec(L.perm, P, st));
    UFVM_CHECK(upload_vec(L.inv, I, st));
    UFVM_CHECK(upload_vec(L.ellCol, ell, st));
    UFVM_CHECK(upload_vec(L.parentsP, parP, st));
    UFVM_CHECK(upload_vec(L.childP, chP, st));
    UFVM_CHECK(upload_vec(L.childStartP, chS, st));
    {  // Galerkin target of every fine entry: -1 inside the aggregate, else the coarse position
      std::vector<int> crp(nc + 1), ccol(std::max(C.nnz, 1));
      UFVM_CUDA(cudaMemcpyAsync(crp.data(), C.rowptr.p, (nc + 1) * sizeof(int), cudaMemcpyDeviceToHost, st));
      if (C.nnz)
        UFVM_CUDA(cudaMemcpyAsync(ccol.data(), C.col.p, C.nnz * sizeof(int), cudaMemcpyDeviceToHost, st));
      UFVM_CUDA(cudaStreamSynchronize(st));
      std::vector<int> gp(std::max(nnz, 1), -2);
      for (int i = 0; i < n; ++i) {
        const int Pi = parents[i];
        for (int k = rp[i]; k < rp[i + 1]; ++k) {
          const int Q = parents[col[k]];
          if (Q == Pi) { gp[k] = -1; continue; }
          for (int t = crp[Pi]; t < crp[Pi + 1]; ++t)
            if (ccol[t] == Q) { gp[k] = t; break; }
        }
      }
      UFVM_CHECK(upload_vec(L.gpos, gp, st));
    }
    UFVM_CHECK(dalloc(L.ellAnb, std::max<size_t>((size_t)W * n, 1)));
    if (l == 0) {  // FP64 ELL copy of the momentum matrix for the U solve
      UFVM_CHECK(dalloc(L.uAnb, std::max<size_t>((size_t)W * n, 1)));
      UFVM_CHECK(dalloc(L.uAc, n));
      UFVM_CHECK(dalloc(L.uBc, n));
      UFVM_CHECK(dalloc(L.uX, n));
    }
    UFVM_CUDA(cudaStreamSynchronize(st));  // the host vectors above go out of scope
    L.ellW = W;
    L.ell_valid = true;
  }
  return UFVM_OK;
}

int Service::solve_u(bool g) {
  const int ns = (int)cases.size();
  const ufvm_settings& s = S;
  cudaGraphConditionalHandle h = 0;
  k_u_to_ell<<<nwc, kBlock, 0, stream>>>(slotTab.p, levTab.p, ns, wc.p);
  // the first residual is taken for every slot
  k_set_active<<<nblocks(ns), kBlock, 0, stream>>>(uctl.p, ns);
  if (ures_items) k_res64_items<<<nwc, kBlock, 0, stream>>>(wures_items.p, uctl.p, part.p);
  else k_res64_abs<<<nwc, kBlock, 0, stream>>>(slotTab.p, levTab.p, ns, wc.p, uctl.p, part.p);
  k_slot_sum<<<ns, 256, 0, stream>>>(cstart.p, cend.p, part.p, part.p + nwc + 8);
  // (in a captured tick the while node starts from its default condition 1: a body whose
  // slots are all inactive does nothing and its k_ctrl ends the loop)
  k_ctrl<<<1, 256, 0, stream>>>(slotTab.p, ns, part.p + nwc + 8, uctl.p, 1, s.u_n_iter, s.u_rrf, 1, SCAL_U_R0,
                                SCAL_U_R1, anyflag.p, 0, h, loopcnt.p, 0);
  UFVM_LAUNCH_CHECK();
  auto body = [&]() -> int {
    bool chained = false;
    for (int pass = 0; pass < 2; ++pass)
      for (int q = pass; q < ucolors; ++q) {  // the backward pass skips the repeated colour
        const int c = pass == 0 ? q : ucolors - 1 - q;
        if (ucol_cnt[c] == 0) continue;
        if (u_items) {
          UFVM_CHECK(launch_colour(chained, k_mc64_items, ucol_cnt[c], stream,
                                   (const U0Item*)(wu_items.p + ucol_off[c]), (const SolveCtl*)uctl.p));
          chained = true;
        } else {
          k_mc64<<<ucol_cnt[c], kBlock, 0, stream>>>(slotTab.p, levTab.p, ns, wu_col.p + ucol_off[c], c, uctl.p);
          chained = false;
        }
      }
    if (ures_items)
      UFVM_CHECK(launch_k(chained, k_res64_items, dim3(nwc), dim3(kBlock), 0, stream, wures_items.p, uctl.p, part.p));
    else
      UFVM_CHECK(launch_k(chained, k_res64_abs, dim3(nwc), dim3(kBlock), 0, stream, slotTab.p, levTab.p, ns, wc.p,
                          uctl.p, part.p));
    UFVM_CHECK(launch_k(true, k_slot_sum, dim3(ns), dim3(256), 0, stream, cstart.p, cend.p, part.p,
                        part.p + nwc + 8));
    UFVM_CHECK(launch_k(true, k_ctrl, dim3(1), dim3(256), 0, stream, slotTab.p, ns, part.p + nwc + 8, uctl.p, 0,
                        s.u_n_iter, s.u_rrf, 1, SCAL_U_R0, SCAL_U_R1, anyflag.p, g, h, loopcnt.p, 0));
    return UFVM_OK;
  };
  if (g) {
    UFVM_CHECK(loop_begin(0, &h));
    const int st = body();
    UFVM_CHECK(loop_end());
    UFVM_CHECK(st);
  } else {
    int any = 0;
    for (int it = 0; it < s.u_n_iter; ++it) {
      ++n_usweeps;
      UFVM_CHECK(body());
      if (it & 1) {
        UFVM_CUDA(cudaMemcpyAsync(&any, anyflag.p, sizeof(int), cudaMemcpyDeviceToHost, stream));
        UFVM_CUDA(cudaStreamSynchronize(stream));
        if (!any) break;
      }
    }
  }
  k_u_from_ell<<<nwc, kBlock, 0, stream>>>(slotTab.p, levTab.p, ns, wc.p);
  UFVM_LAUNCH_CHECK();
  return UFVM_OK;
}

int Service::solve_p(bool g) {
  const int ns = (int)cases.size();
  const ufvm_settings& s = S;
  cudaGraphConditionalHandle h = 0;
  k_set_active<<<nblocks(ns), kBlock, 0, stream>>>(pctl.p, ns);
  // FP32 copy of level 0 and FP64 Galerkin products, then their FP32 copies
  k_lev_to32<<<nwrows[0], kBlock, 0, stream>>>(levTab.p, ns, 0, wrows[0].p, pctl.p);
  for (int l = 0; l + 1 < Lmax; ++l) {
    k_galerkin_b<<<nwrows[l + 1], kBlock, 0, stream>>>(levTab.p, ns, l, wrows[l + 1].p, pctl.p);
    k_lev_to32<<<nwrows[l + 1], kBlock, 0, stream>>>(levTab.p, ns, l + 1, wrows[l + 1].p, pctl.p);
  }
  k_coarse_factor<<<ns, 1024, sizeof(DenseFactorSmem), stream>>>(levTab.p, ns, dcoarsest.p, cinv.p);
  UFVM_LAUNCH_CHECK();
  k_res64_rhs<<<nwc, kBlock, 0, stream>>>(slotTab.p, levTab.p, ns, wc.p, pctl.p, part.p);
  k_slot_sum<<<ns, 256, 0, stream>>>(cstart.p, cend.p, part.p, part.p + nwc + 8);
  k_ctrl<<<1, 256, 0, stream>>>(slotTab.p, ns, part.p + nwc + 8, pctl.p, 1, s.p_max_cycles, s.p_termination, 0,
                                SCAL_P_R0, SCAL_P_R1, anyflag.p, 0, h, loopcnt.p, 1);
  UFVM_LAUNCH_CHECK();
  auto smooth = [&](int l, int sweeps) -> int {
    bool chained = false;
    for (int k = 0; k < sweeps; ++k)
      for (int pass = 0; pass < 2; ++pass)
        for (int q = pass; q < maxcol[l]; ++q) {  // the backward pass skips the repeated colour
          const int c = pass == 0 ? q : maxcol[l] - 1 - q;
          if (smcnt[l][c] == 0) continue;
          if (l == 0 && l0_items)
            UFVM_CHECK(launch_colour(chained, k_mc32_l0, smcnt[0][c], stream,
                                     (const L0Item*)(wsm0.p + smoff[0][c]), (const SolveCtl*)pctl.p));
          else
            UFVM_CHECK(launch_colour(chained, k_mc32, smcnt[l][c], stream, (const LevDesc*)levTab.p, ns, l,
                                     (const int2*)(wsm[l].p + smoff[l][c]), c, (const SolveCtl*)pctl.p));
          chained = true;
        }
    return UFVM_OK;
  };
  // flexible-CG scratch: (z, q_old) partials and sums, ((p, q), (p, r)) partials and sums
  const size_t o_zs = ((size_t)nwc + 1) & ~(size_t)1, o_pp = (o_zs + ns + 1) & ~(size_t)1,
               o_ps = o_pp + 2 * (size_t)nwc;
  double* zq_part = fcg.p;
  double* zq_sum = fcg.p + o_zs;
  double2* pqr_part = reinterpret_cast<double2*>(fcg.p + o_pp);
  double2* pqr_sum = reinterpret_cast<double2*>(fcg.p + o_ps);
  auto cycle = [&]() -> int {
    // large levels as grid-wide launches, the small ones per slot in one CTA; every launch after
    // the body's first kernel is chained except a sweep's first colour
    const dim3 B(kBlock);
    for (int l = 0; l < maxg; ++l) {
      UFVM_CHECK(smooth(l, s.p_pre_sweep));
      UFVM_CHECK(launch_k(true, k_res32, dim3(nwnc[l]), B, 0, stream, levTab.p, ns, l, wnc[l].p, pctl.p));
      UFVM_CHECK(launch_k(true, k_restrict32, dim3(nwrc[l]), B, 0, stream, levTab.p, ns, l, wrc[l].p, pctl.p));
    }
    const bool after = maxg > 0;  // a kernel of this body came before
    if (use_packing && npk_tasks > 0) {
      UFVM_CHECK(launch_k(after, k_coarse_vcycle_pk, dim3(npk_tasks), dim3(kBlockPack), 0, stream, levTab.p, ns,
                          dcoarsest.p, dgstart.p, cinv.p, s.p_pre_sweep, s.p_post_sweep, pctl.p, dpk_tasks.p));
    } else {
      UFVM_CHECK(launch_k(after, k_coarse_vcycle, dim3(ns), dim3(1024), 0, stream, levTab.p, ns, dcoarsest.p,
                          dgstart.p, cinv.p, s.p_pre_sweep, s.p_post_sweep, pctl.p, dcta_order.p));
    }
    for (int l = maxg - 1; l >= 0; --l) {
      UFVM_CHECK(launch_k(true, k_prolong32, dim3(nwnc[l]), B, 0, stream, levTab.p, ns, l, wnc[l].p, pctl.p));
      UFVM_CHECK(smooth(l, s.p_post_sweep));
    }
    if (s.p_krylov) {
      UFVM_CHECK(launch_k(true, k_fcg_zq, dim3(nwc), B, 0, stream, slotTab.p, levTab.p, ns, wc.p, pctl.p, zq_part));
      UFVM_CHECK(launch_k(true, k_slot_sum, dim3(ns), dim3(256), 0, stream, cstart.p, cend.p, zq_part, zq_sum));
      UFVM_CHECK(launch_k(true, k_fcg_p, dim3(nwc), B, 0, stream, slotTab.p, levTab.p, ns, wc.p, pctl.p, zq_sum,
                          pqr_sum));
      UFVM_CHECK(launch_k(true, k_fcg_q, dim3(nwc), B, 0, stream, slotTab.p, levTab.p, ns, wc.p, pctl.p, pqr_part));
      UFVM_CHECK(launch_k(true, k_slot_sum2, dim3(ns), dim3(256), 0, stream, cstart.p, cend.p, pqr_part, pqr_sum));
      UFVM_CHECK(launch_k(true, k_fcg_update, dim3(nwc), B, 0, stream, slotTab.p, levTab.p, ns, wc.p, pctl.p,
                          pqr_sum, part.p));
    } else {
      UFVM_CHECK(launch_k(true, k_update64, dim3(nwc), B, 0, stream, slotTab.p, levTab.p, ns, wc.p, pctl.p));
      UFVM_CHECK(launch_k(true, k_res64_rhs, dim3(nwc), B, 0, stream, slotTab.p, levTab.p, ns, wc.p, pctl.p,
                          part.p));
    }
    UFVM_CHECK(launch_k(true, k_slot_sum, dim3(ns), dim3(256), 0, stream, cstart.p, cend.p, part.p,
                        part.p + nwc + 8));
    UFVM_CHECK(launch_k(true, k_ctrl, dim3(1), dim3(256), 0, stream, slotTab.p, ns, part.p + nwc + 8, pctl.p, 0,
                        s.p_max_cycles, s.p_termination, 0, SCAL_P_R0, SCAL_P_R1, anyflag.p, g, h, loopcnt.p, 1));
    return UFVM_OK;
  };
  if (g) {
    UFVM_CHECK(loop_begin(1, &h));
    const int st = cycle();
    UFVM_CHECK(loop_end());
    return st;
  }
  int any = 1;
  for (int cyc = 0; cyc < s.p_max_cycles; ++cyc) {
    ++n_pcycles;
    UFVM_CHECK(cycle());
    if (cyc & 1) {
      UFVM_CUDA(cudaMemcpyAsync(&any, anyflag.p, sizeof(int), cudaMemcpyDeviceToHost, stream));
      UFVM_CUDA(cudaStreamSynchronize(stream));
      if (!any) break;
    }
  }
  return UFVM_OK;
}

// The device work of one steady SIMPLE iteration of every resident case (cfdRunCase.m:92-142
// order). g: being captured into the tick graph (no host synchronisation, no hierarchy
// builds, no phase events).
int Service::enqueue_tick(bool g, std::vector<std::pair<int, int>>& marks) {
  const int ns = (int)cases.size();
  int evn = 0;
  auto mark = [&](int phase) -> int {
    if (g) return UFVM_OK;
    if ((int)evpool.size() <= evn) {
      cudaEvent_t e;
      UFVM_CUDA(cudaEventCreate(&e));
      evpool.push_back(e);
    }
    UFVM_CUDA(cudaEventRecord(evpool[evn], stream));
    marks.push_back({phase, evn++});
    return UFVM_OK;
  };
  UFVM_CUDA(cudaMemsetAsync(flags.p, 0, (size_t)ns * FLAG_N * sizeof(int), stream));
  BatchLaunch b = batch();
  UFVM_CHECK(mark(PH_UPDATE));
  UFVM_CHECK(stage_update_fields(b));
  for (int comp = 0; comp < 3; ++comp) {
    UFVM_CHECK(mark(PH_ASM_U));
    if (comp == 0) UFVM_CHECK(stage_uface_interior(b));
    UFVM_CHECK(stage_assemble_u(b, comp, true));
    k_copy_scal<<<nblocks(ns), kBlock, 0, stream>>>(slotTab.p, ns, SCAL_RMS, SCAL_U_RMS + comp);
    k_copy_scal<<<nblocks(ns), kBlock, 0, stream>>>(slotTab.p, ns, SCAL_MAX, SCAL_U_MAX + comp);
    UFVM_CHECK(mark(PH_SOLVE_U));
    UFVM_CHECK(solve_u(g));
    UFVM_CHECK(mark(PH_CORR_U));
    UFVM_CHECK(stage_correct_u(b, comp));
  }
  int maxp = 0;
  for (auto* c : cases) maxp = std::max(maxp, c->P.n);
  for (int k = 0; k < S.n_correctors; ++k) {
    UFVM_CHECK(mark(PH_ASM_P));
    UFVM_CHECK(stage_assemble_p(b));
    k_copy_scal<<<nblocks(ns), kBlock, 0, stream>>>(slotTab.p, ns, SCAL_RMS, SCAL_P_RMS);
    k_copy_scal<<<nblocks(ns), kBlock, 0, stream>>>(slotTab.p, ns, SCAL_MAX, SCAL_P_MAX);
    UFVM_CHECK(mark(PH_HIER));
    if (!g) {
      std::vector<Case*> need;
      for (auto* c : cases) {
        if (needs_hierarchy(*c)) need.push_back(c);
        c->p_solves++;
      }
      UFVM_CHECK(build_hierarchies(need));
      if (!need.empty()) {
        tables_dirty = true;
        UFVM_CHECK(rebuild_tables());
        b = batch();
      }
    }
    UFVM_CHECK(mark(PH_SOLVE_P));
    UFVM_CHECK(solve_p(g));
    UFVM_CHECK(mark(PH_CORR_P));
    UFVM_CHECK(stage_correct_p(b, maxp, nullptr));
  }
  UFVM_CHECK(mark(PH_N));
  return UFVM_OK;
}

bool Service::needs_hierarchy(const Case& c) const {
  return !c.hierarchy_valid ||
         (S.hierarchy_reuse > 0 && c.p_solves > 0 && (c.p_solves % S.hierarchy_reuse) == 0);
}

// Kernel nodes of a graph (for the launch count the service reports); -1 if the graph cannot
// be inspected, with the error cleared so it is not taken for a failed launch later.
static long long count_kernels(cudaGraph_t g) {
  size_t n = 0;
  cudaError_t e = cudaGraphGetNodes(g, nullptr, &n);
  if (e != cudaSuccess) {
    std::fprintf(stderr, "ufvm: cudaGraphGetNodes: %s\n", cudaGetErrorString(e));
    cudaGetLastError();
    return -1;
  }
  std::vector<cudaGraphNode_t> nodes(n);
  if (n) e = cudaGraphGetNodes(g, nodes.data(), &n);
  if (e != cudaSuccess) {
    std::fprintf(stderr, "ufvm: cudaGraphGetNodes: %s\n", cudaGetErrorString(e));
    cudaGetLastError();
    return -1;
  }
  long long k = 0;
  for (auto nd : nodes) {
    // the type query fails on the conditional nodes themselves (their kernels are counted
    // from the body graphs); such a node is skipped and the error cleared
    cudaGraphNodeType t;
    e = cudaGraphNodeGetType(nd, &t);
    if (e != cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    if (t == cudaGraphNodeTypeKernel) ++k;
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    std::fprintf(stderr, "ufvm: graph inspection left an error: %s\n", cudaGetErrorString(e));
    return -1;
  }
  return k;
}

int Service::capture_tick() {
  bodies.clear();
  if (gexec) { cudaGraphExecDestroy(gexec); gexec = nullptr; }
  if (graph) { cudaGraphDestroy(graph); graph = nullptr; }
  graph_valid = false;
  std::vector<std::pair<int, int>> marks;
  UFVM_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
  int st = enqueue_tick(true, marks);
  if (main_stream && stream != main_stream) {  // an error inside a loop body: close its capture
    stream = main_stream;
    cudaGraph_t gb = nullptr;
    cudaStreamEndCapture(bstream, &gb);
  }
  cudaGraph_t gt = nullptr;
  const cudaError_t ee = cudaStreamEndCapture(stream, &gt);
  if (st != UFVM_OK) {
    if (gt) cudaGraphDestroy(gt);
    cudaGetLastError();
    return st;
  }
  if (ee != cudaSuccess) {
    set_error(std::string("cudaStreamEndCapture: ") + cudaGetErrorString(ee));
    cudaGetLastError();
    return UFVM_E_CUDA;
  }
  graph = gt;
  {
    const cudaError_t pend = cudaGetLastError();
    if (pend != cudaSuccess) std::fprintf(stderr, "ufvm: error pending after the capture: %s\n", cudaGetErrorString(pend));
  }
  static_kernels = count_kernels(graph);
  ubody_kernels = pbody_kernels = 0;
  for (auto& bb : bodies) (bb.first == 0 ? ubody_kernels : pbody_kernels) = count_kernels(bb.second);
  bodies.clear();
  UFVM_CUDA(cudaGraphInstantiate(&gexec, graph, 0));
  {
    const cudaError_t pend = cudaGetLastError();
    if (pend != cudaSuccess) std::fprintf(stderr, "ufvm: error pending after instantiation: %s\n", cudaGetErrorString(pend));
  }
  graph_valid = true;
  ++n_captures;
  return UFVM_OK;
}

// One steady SIMPLE iteration of every resident case.
int Service::iterate(std::vector<double>& res, std::vector<int>& conv) {
  const int ns = (int)cases.size();
  res.assign((size_t)ns * 16, 0.0);
  conv.assign(ns, 0);
  if (ns == 0) return UFVM_OK;
  for (auto* c : cases) {
    const long long b0 = t_dev_bytes;
    if (c->lev.empty() || !c->lev[0].rowptr.p) UFVM_CHECK(c->fresh_level0());
    if (!c->lev[0].color_valid) { UFVM_CHECK(build_coloring(c->lin, c->lev[0])); tables_dirty = true; }
    c->dev_bytes += t_dev_bytes - b0;
  }
  auto host_ms_since = [](std::chrono::steady_clock::time_point t) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t).count();
  };
  double rebuild_ms = 0.0;
  if (tables_dirty) {
    const auto h0 = std::chrono::steady_clock::now();
    UFVM_CHECK(rebuild_tables());
    rebuild_ms = host_ms_since(h0);
  }
  ++n_iter_calls;
  // a tick without hierarchy builds runs as one graph launch (captured when the tables change)
  bool g = use_graph != 0;
  for (auto* c : cases) {
    if (!g) break;
    for (int k = 0; k < S.n_correctors; ++k) {
      const long long ps = c->p_solves + k;
      if (!c->hierarchy_valid || (S.hierarchy_reuse > 0 && ps > 0 && (ps % S.hierarchy_reuse) == 0)) g = false;
    }
  }
  std::vector<std::pair<int, int>> marks;
  if (g) {
    {
      const cudaError_t pend = cudaGetLastError();
      if (pend != cudaSuccess) {
        set_error(std::string("error pending before the tick: ") + cudaGetErrorString(pend));
        return UFVM_E_CUDA;
      }
    }
    if (!graph_valid) {
      const auto h1 = std::chrono::steady_clock::now();
      const int cst = capture_tick();
      const double cms = host_ms_since(h1);
      host_capture_ms += cms;
      last_rebuild_ms = rebuild_ms + cms;  // the host cost of a change of the slot set
      if (cst != UFVM_OK) {
        // keep serving: this and later ticks are launched eagerly
        std::fprintf(stderr, "ufvm: capturing the tick graph failed (%s); ticks are launched eagerly\n", get_error());
        cudaGetLastError();
        use_graph = 0;
        g = false;
      }
    }
  }
  host_rebuild_ms += rebuild_ms;
  if (g) {
    UFVM_CUDA(cudaGraphLaunch(gexec, stream));
    for (auto* c : cases) c->p_solves += S.n_correctors;
    ++n_graph_ticks;
  } else {
    UFVM_CHECK(enqueue_tick(false, marks));
  }
  // rows written by an outlet with fixed p change the scale domain (Q12)
  for (auto* c : cases) {
    const int before = c->rowsU;
    for (int ip = 0; ip < c->P.n; ++ip)
      if (c->P.type[ip] == UFVM_PATCH_OUTLET && c->P.bcP[ip] == UFVM_BC_FIXED_VALUE && c->P.count[ip] > 0) {
        const int row0 = (c->S.quirks & UFVM_Q12_OUTLET_U_FACE_ROWS) ? c->P.start[ip] : c->M.Nc + c->P.start[ip] - c->M.Fi;
        c->rowsU = std::max(c->rowsU, row0 + c->P.count[ip]);
      }
    if (c->rowsU != before) tables_dirty = true;
  }
  std::vector<double> h((size_t)ns * SCAL_SLOT_N);
  std::vector<int> fl((size_t)ns * FLAG_N);
  UFVM_CUDA(cudaMemcpyAsync(h.data(), scal.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost, stream));
  UFVM_CUDA(cudaMemcpyAsync(fl.data(), flags.p, fl.size() * sizeof(int), cudaMemcpyDeviceToHost, stream));
  unsigned long long lc[2] = {0, 0};
  UFVM_CUDA(cudaMemcpyAsync(lc, loopcnt.p, sizeof(lc), cudaMemcpyDeviceToHost, stream));
  UFVM_CUDA(cudaStreamSynchronize(stream));
  {
    const cudaError_t pend = cudaGetLastError();
    if (pend != cudaSuccess) {
      set_error(std::string(g ? "graph tick: " : "eager tick: ") + cudaGetErrorString(pend));
      return UFVM_E_CUDA;
    }
  }
  if (g && static_kernels >= 0 && ubody_kernels >= 0 && pbody_kernels >= 0)
    launches_total += static_kernels + ubody_kernels * (long long)(lc[0] - loops_seen[0]) +
                      pbody_kernels * (long long)(lc[1] - loops_seen[1]);
  loops_seen[0] = lc[0];
  loops_seen[1] = lc[1];
  for (size_t q = 0; q + 1 < marks.size(); ++q) {
    float ms = 0;
    UFVM_CUDA(cudaEventElapsedTime(&ms, evpool[marks[q].second], evpool[marks[q + 1].second]));
    ph_ms[marks[q].first] += ms;
  }
  int maxcyc = 0;
  for (int q = 0; q < ns; ++q) {
    const double* x = &h[(size_t)q * SCAL_SLOT_N];
    double* r = &res[(size_t)q * 16];
    for (int c = 0; c < 3; ++c) { r[c] = x[SCAL_U_RMS + c]; r[4 + c] = x[SCAL_U_MAX + c]; }
    r[3] = x[SCAL_P_RMS]; r[7] = x[SCAL_P_MAX];
    r[8] = x[SCAL_U_R0]; r[12] = x[SCAL_U_R1]; r[11] = x[SCAL_P_R0]; r[15] = x[SCAL_P_R1];
    r[9] = x[SCAL_CYC];
    maxcyc = std::max(maxcyc, (int)r[9]);
    const ufvm_settings& cs = cases[q]->S;
    conv[q] = (r[0] <= cs.tol_u && r[1] <= cs.tol_u && r[2] <= cs.tol_u && r[3] <= cs.tol_p) ? 1 : 0;
    if (fl[(size_t)q * FLAG_N + FLAG_ZERO_DIAG]) conv[q] = -UFVM_E_ZERO_DIAG;
    if (fl[(size_t)q * FLAG_N + FLAG_BAD_BC]) conv[q] = -UFVM_E_BC_UNSUPPORTED;
    for (int i = 0; i < 4; ++i)
      if (std::isnan(r[i])) conv[q] = -UFVM_E_NAN;
  }
  if (g) n_pcycles += (long long)maxcyc * S.n_correctors;
  return UFVM_OK;
}

// Times one kernel of the tick on the current resident batch, `reps` times after one warm-up,
// and returns the average device time of one unit and its compulsory bytes (every array
// touched once per pass; neighbour gathers of x counted as cache hits). Units:
//   0: one symmetric FP64 multicolour Gauss-Seidel sweep of every slot's level 0 (k_mc64 on
//      the ELL copy, 2 x colours - 1 launches): 2 x (32 B per row -- ac, bc, x written, x read
//      once -- + 12 B per nonzero), less the rows of the last colour, which the backward pass
//      skips;
//   1: the same sweep in FP32 over the V-cycle's level 0 (k_mc32, colour-permuted ELL):
//      2 x (16 B per row -- ac, bc, x written, x read once -- + 8 B per nonzero);
//   2: the flexible-CG product q = A p with its two dot products (k_fcg_q): 36 B/row + 12 B/nz;
//   3: the momentum assembly of the three components as a tick runs it (k_uface_int over the
//      interior faces for all three, then per component k_uface_bnd, k_assemble_u, k_du_boundary
//      and the residual reduction): per component, per cell 8 phi + 24 grad phi + 16 (ac, bc),
//      per interior face 8 index + 8 mdot + 8 gamma + 8 gDiff + 24 T + 8 gf + 16 (two
//      off-diagonals) bytes;
//   4: the pressure-correction assembly (k_rhiechow, k_assemble_p and the mass-imbalance
//      reduction): per cell 8 p + 24 grad p + 24 U + 24 DU + 16 (ac, bc), per interior face
//      8 index + 8 gf + 24 Sf + 24 eCF + 8 |CF| + 8 mdot old + 8 mdot new + 16 (C1, C2) +
//      16 (two off-diagonals) bytes;
//   5: the field update (boundary values, the Gauss gradients of U and p with their boundary
//      fixes, the velocity scale): over the Nc + Fb rows R, per U component 8 read + 24 gradient
//      written, 8 + 24 for p; per face 24 Sf, per interior face 8 index + 8 gf, per cell 8 V
//      for each of the two gradients;
//   6: one pass of the packed coarse V-cycle kernel (k_coarse_vcycle_pk) over every slot's
//      levels below its grid levels: latency-bound; bytes counted as five passes (a symmetric
//      pre- and post-sweep, the residual) over each such level's 16 B per row + 8 B per nonzero.
// The sweeps overwrite the slots' correction vectors, which the next assembly re-zeroes; units
// 3-5 rewrite matrices and fields from the current state (unit 4 also advances the face mass
// flux), so a batch profiled with them is only fit for timing.
int Service::profile(int kernel, int reps, double* ms, double* bytes) {
  const int ns = (int)cases.size();
  if (ns == 0 || reps <= 0) { set_error("profile: no resident case or reps <= 0"); return UFVM_E_INVALID; }
  if (tables_dirty) UFVM_CHECK(rebuild_tables());
  double N = 0, NNZ = 0;
  for (auto* c : cases) { N += c->M.Nc; NNZ += c->M.nnz; }
  if (kernel == 0) k_u_to_ell<<<nwc, kBlock, 0, stream>>>(slotTab.p, levTab.p, ns, wc.p);
  auto unit = [&]() -> int {
    if (kernel == 0) {
      for (int pass = 0; pass < 2; ++pass)
        for (int q = pass; q < ucolors; ++q) {
          const int c = pass == 0 ? q : ucolors - 1 - q;
          if (ucol_cnt[c] == 0) continue;
          if (u_items) k_mc64_items<<<ucol_cnt[c], kBlock, 0, stream>>>(wu_items.p + ucol_off[c], uctl.p);
          else
            k_mc64<<<ucol_cnt[c], kBlock, 0, stream>>>(slotTab.p, levTab.p, ns, wu_col.p + ucol_off[c], c, uctl.p);
        }
    } else if (kernel == 1) {
      for (int pass = 0; pass < 2; ++pass)
        for (int q = pass; q < maxcol[0]; ++q) {
          const int c = pass == 0 ? q : maxcol[0] - 1 - q;
          if (smcnt[0][c] == 0) continue;
          if (l0_items) k_mc32_l0<<<smcnt[0][c], kBlock, 0, stream>>>(wsm0.p + smoff[0][c], pctl.p);
          else k_mc32<<<smcnt[0][c], kBlock, 0, stream>>>(levTab.p, ns, 0, wsm[0].p + smoff[0][c], c, pctl.p);
        }
    } else if (kernel == 2) {
      k_fcg_q<<<nwc, kBlock, 0, stream>>>(slotTab.p, levTab.p, ns, wc.p, pctl.p,
                                          reinterpret_cast<double2*>(fcg.p + (((size_t)nwc + 1) & ~(size_t)1) +
                                                                     (((size_t)ns + 1) & ~(size_t)1)));
    } else if (kernel == 3) {
      const BatchLaunch b = batch();
      UFVM_CHECK(stage_uface_interior(b));
      for (int comp = 0; comp < 3; ++comp) UFVM_CHECK(stage_assemble_u(b, comp, true));
    } else if (kernel == 4) {
      UFVM_CHECK(stage_assemble_p(batch()));
    } else if (kernel == 5) {
      UFVM_CHECK(stage_update_fields(batch()));
    } else {
      if (use_packing && npk_tasks > 0)
        k_coarse_vcycle_pk<<<npk_tasks, kBlockPack, 0, stream>>>(levTab.p, ns, dcoarsest.p, dgstart.p, cinv.p,
                                                                S.p_pre_sweep, S.p_post_sweep, pctl.p, dpk_tasks.p);
      else
        k_coarse_vcycle<<<ns, 1024, 0, stream>>>(levTab.p, ns, dcoarsest.p, dgstart.p, cinv.p, S.p_pre_sweep,
                                                 S.p_post_sweep, pctl.p, dcta_order.p);
    }
    UFVM_LAUNCH_CHECK();
    return UFVM_OK;
  };
  if (kernel < 0 || kernel > 6) { set_error("profile: unknown kernel id"); return UFVM_E_INVALID; }
  if (kernel == 1 || kernel == 2 || kernel == 6) {
    for (auto* c : cases)
      if (!c->hierarchy_valid) { set_error("profile: a resident case has no AMG hierarchy yet"); return UFVM_E_INVALID; }
    if (Lmax < 2 || nwsm.empty()) { set_error("profile: no AMG hierarchy yet"); return UFVM_E_INVALID; }
  }
  if (kernel == 1) {
    N = 0; NNZ = 0;
    for (auto* c : cases)
      if (c->hierarchy_valid && c->n_levels > 1) { N += c->M.Nc; NNZ += c->M.nnz; }
  }
  k_set_active<<<nblocks(ns), kBlock, 0, stream>>>(uctl.p, ns);
  k_set_active<<<nblocks(ns), kBlock, 0, stream>>>(pctl.p, ns);
  UFVM_CHECK(unit());
  cudaEvent_t a, b;
  UFVM_CUDA(cudaEventCreate(&a));
  UFVM_CUDA(cudaEventCreate(&b));
  UFVM_CUDA(cudaEventRecord(a, stream));
  for (int r = 0; r < reps; ++r) UFVM_CHECK(unit());
  UFVM_CUDA(cudaEventRecord(b, stream));
  UFVM_CUDA(cudaEventSynchronize(b));
  float t = 0;
  UFVM_CUDA(cudaEventElapsedTime(&t, a, b));
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  *ms = t / reps;
  double Fi = 0, F = 0, R = 0;
  for (auto* c : cases) { Fi += c->M.Fi; F += c->M.F; R += c->M.Nc + c->M.Fb; }
  // rows of the last colour that the backward pass skips (slots with the most colours only)
  double skipN = 0, skipNNZ = 0;
  if (kernel <= 1) {
    const int C = kernel == 0 ? ucolors : maxcol[0];
    for (auto* c : cases) {
      const Level& L0 = c->lev[0];
      if (!L0.color_valid || L0.ncolor != C || (int)L0.h_colorStart.size() <= C) continue;
      if (kernel == 1 && !(c->hierarchy_valid && c->n_levels > 1)) continue;
      const double last = (double)(L0.h_colorStart[C] - L0.h_colorStart[C - 1]);
      skipN += last;
      skipNNZ += (double)c->M.nnz * last / (double)c->M.Nc;
    }
  }
  if (kernel == 0) *bytes = 2.0 * (32.0 * N + 12.0 * NNZ) - (32.0 * skipN + 12.0 * skipNNZ);
  else if (kernel == 1) *bytes = 2.0 * (16.0 * N + 8.0 * NNZ) - (16.0 * skipN + 8.0 * skipNNZ);
  else if (kernel == 2) *bytes = 36.0 * N + 12.0 * NNZ;
  else if (kernel == 3) *bytes = 3.0 * (48.0 * N + 80.0 * Fi);
  else if (kernel == 4) *bytes = 96.0 * N + 120.0 * Fi;
  else if (kernel == 5) *bytes = (3 * 32.0 + 32.0) * R + 2 * (24.0 * F + 16.0 * Fi + 8.0 * N);
  else {
    double b = 0;
    for (int q = 0; q < ns && q < (int)h_gstart.size(); ++q)
      for (int l = h_gstart[q]; l <= h_coarsest[q] && l < cases[q]->n_levels; ++l)
        b += 5.0 * (16.0 * cases[q]->lev[l].n + 8.0 * cases[q]->lev[l].nnz);
    *bytes = b;
  }
  return UFVM_OK;
}

// Destroy calls cannot report to a caller; a failure is printed once and then cleared so that
// it is not mistaken later for a failed launch of another case or service.
static void destroy_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    std::fprintf(stderr, "ufvm: %s failed during service teardown: %s\n", what, cudaGetErrorString(e));
    cudaGetLastError();
  }
}

Service::~Service() {
  if (stream) destroy_check(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
  if (gexec) destroy_check(cudaGraphExecDestroy(gexec), "cudaGraphExecDestroy");
  if (graph) destroy_check(cudaGraphDestroy(graph), "cudaGraphDestroy");
  gexec = nullptr;
  graph = nullptr;
  for (cudaStream_t bs : build_streams) destroy_check(cudaStreamDestroy(bs), "cudaStreamDestroy");
  build_streams.clear();
  if (build_event) destroy_check(cudaEventDestroy(build_event), "cudaEventDestroy");
  build_event = nullptr;
  for (auto* c : cases) delete c;
  cases.clear();
  for (auto* a : {&scal, &part, &fcg}) dfree(*a);
  dfree(flags); dfree(cstart); dfree(cend); dfree(ustart); dfree(uend); dfree(anyflag); dfree(loopcnt);
  dfree(slotTab); dfree(levTab); dfree(uctl); dfree(pctl);
  for (auto* a : {&wc, &wf, &wb, &wu, &wu_col}) dfree(*a);
  for (auto& a : wrows) dfree(a);
  for (auto& a : wsm) dfree(a);
  for (auto& a : wnc) dfree(a);
  for (auto& a : wrc) dfree(a);
  dfree(dcoarsest); dfree(dgstart); dfree(cinv); dfree(dcta_order); dfree(dpk_tasks); dfree(wsm0); dfree(wu_items); dfree(wures_items);
  lin.release();
  for (auto e : evpool) destroy_check(cudaEventDestroy(e), "cudaEventDestroy");
  if (bstream) destroy_check(cudaStreamDestroy(bstream), "cudaStreamDestroy");
  if (stream) destroy_check(cudaStreamDestroy(stream), "cudaStreamDestroy");
  destroy_check(cudaGetLastError(), "a CUDA call");
}

}  // namespace ufvm
