// amg.cu -- agglomeration AMG: hierarchy build and V/W/F cycles.
//
//   cfdAgglomerate         solve/AMG/cfdAgglomerate.m:7-17
//   cfdAgglomerateLevel    solve/AMG/cfdAgglomerateLevel.m:13-105
//   Galerkin by summation  assemble/assembleAgglomeratedLHS.m:16-30
//   cycles / driver        solve/AMG/cfdApplyVCycle.m, cfdApplyWCycle.m, cfdApplyFCycle.m,
//                          cfdApplyAMG.m:9-57, cfdRestrict.m, cfdProlongate.m
//
// The reference agglomerates with a sequential greedy sweep over seeds in natural order.
// It is reproduced here exactly, but in parallel, by deterministic reservations: every
// unprocessed seed reserves the cells it would claim (itself, its strong unassigned
// neighbours and their strong unassigned neighbours) with atomicMax on a key that
// prefers the lowest seed index; a seed commits only if it holds all its reservations.
// Claim sets only shrink as cells get assigned, so a committed seed's claims are the
// ones it would make in the sequential sweep, and the final `parents` map is identical.
// Orphans are attached in rounds that respect their natural-order dependencies.
#include <atomic>
#include "amg.cuh"

namespace ufvm {

__global__ void k_maxanb(int n, const int* __restrict__ rp, const double* __restrict__ anb, double* maxAnb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double m = -INFINITY;
  for (int k = rp[i]; k < rp[i + 1]; ++k) m = dmax(m, -anb[k]);
  maxAnb[i] = m;
}

__global__ void k_strong(int n, const int* __restrict__ rp, const double* __restrict__ anb,
                         const double* __restrict__ maxAnb, signed char* strong) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double m = maxAnb[i];
  for (int k = rp[i]; k < rp[i + 1]; ++k) strong[k] = ((-anb[k]) / m) > 0.5 ? 1 : 0;
}

struct AggArgs {
  int n;
  const int *rp, *col;
  const signed char* strong;
  int* parents;
  int* status;  // 0 unprocessed seed, 1 done
  unsigned long long* resv;
  int* win;
  int* seedflag;
  int* remaining;
};

__device__ __forceinline__ unsigned long long agg_key(unsigned int round, int s) {
  return ((unsigned long long)round << 32) | (unsigned long long)(0xffffffffu - (unsigned int)s);
}

__global__ void k_agg_reserve(AggArgs a, unsigned int round) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= a.n || a.status[s] != 0) return;
  if (__ldcg(a.parents + s) != -1) {  // claimed by an earlier committed seed: not a seed
    a.status[s] = 1;
    return;
  }
  atomicAdd(a.remaining, 1);
  const unsigned long long key = agg_key(round, s);
  atomicMax(a.resv + s, key);
  for (int k = a.rp[s]; k < a.rp[s + 1]; ++k) {
    const int c = a.col[k];
    if (!a.strong[k] || __ldcg(a.parents + c) != -1) continue;
    atomicMax(a.resv + c, key);
    for (int k2 = a.rp[c]; k2 < a.rp[c + 1]; ++k2) {
      const int g = a.col[k2];
      if (a.strong[k2] && __ldcg(a.parents + g) == -1) atomicMax(a.resv + g, key);
    }
  }
}

__global__ void k_agg_check(AggArgs a, unsigned int round) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= a.n) return;
  a.win[s] = 0;
  if (a.status[s] != 0) return;
  const unsigned long long key = agg_key(round, s);
  bool ok = __ldcg(a.resv + s) == key;
  for (int k = a.rp[s]; k < a.rp[s + 1] && ok; ++k) {
    const int c = a.col[k];
    if (!a.strong[k] || __ldcg(a.parents + c) != -1) continue;
    ok = __ldcg(a.resv + c) == key;
    for (int k2 = a.rp[c]; k2 < a.rp[c + 1] && ok; ++k2) {
      const int g = a.col[k2];
      if (a.strong[k2] && __ldcg(a.parents + g) == -1) ok = __ldcg(a.resv + g) == key;
    }
  }
  a.win[s] = ok ? 1 : 0;
}

// Winners apply the sequential seed step (cfdAgglomerateLevel.m:28-64) on their own cells.
__global__ void k_agg_commit(AggArgs a) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= a.n || !a.win[s]) return;
  a.status[s] = 1;
  bool any = false;
  for (int k = a.rp[s]; k < a.rp[s + 1]; ++k)
    if (a.strong[k] && __ldcg(a.parents + a.col[k]) == -1) { any = true; break; }
  if (!any) return;  // single-cell aggregate: undone, the seed stays unassigned
  a.seedflag[s] = 1;
  __stcg(a.parents + s, s);
  // first generation, in cconn order
  for (int k = a.rp[s]; k < a.rp[s + 1]; ++k) {
    const int c = a.col[k];
    if (a.strong[k] && __ldcg(a.parents + c) == -1) __stcg(a.parents + c, -2 - s);  // mark as child
  }
  // second generation from the first-generation children, in children order
  for (int k = a.rp[s]; k < a.rp[s + 1]; ++k) {
    const int c = a.col[k];
    if (!(a.strong[k] && __ldcg(a.parents + c) == -2 - s)) continue;
    for (int k2 = a.rp[c]; k2 < a.rp[c + 1]; ++k2) {
      const int g = a.col[k2];
      if (a.strong[k2] && __ldcg(a.parents + g) == -1) __stcg(a.parents + g, s);
    }
  }
  for (int k = a.rp[s]; k < a.rp[s + 1]; ++k) {
    const int c = a.col[k];
    if (__ldcg(a.parents + c) == -2 - s) __stcg(a.parents + c, s);
  }
}

// orphans (cfdAgglomerateLevel.m:66-83), in rounds that respect natural order
__global__ void k_orphan_round(int n, const int* __restrict__ rp, const int* __restrict__ col,
                               const double* __restrict__ anb, const double* __restrict__ maxAnb,
                               const int* __restrict__ isOrphan, const int* __restrict__ resPrev, int* resNext,
                               int* parents, int* newflag, int* remaining) {
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= n || !isOrphan[o] || resPrev[o]) return;
  for (int k = rp[o]; k < rp[o + 1]; ++k) {
    const int j = col[k];
    if (j < o && isOrphan[j] && !resPrev[j]) { atomicAdd(remaining, 1); return; }
  }
  double strength = 0.0;
  int par = -1;
  for (int k = rp[o]; k < rp[o + 1]; ++k) {
    const int nb = col[k];
    const int pn = __ldcg(parents + nb);
    if (pn != -1) {
      const double sv = (-anb[k]) / maxAnb[nb];
      if (strength < sv) { strength = sv; par = pn; }
    }
  }
  if (par == -1) { par = n + o; newflag[o] = 1; }
  __stcg(parents + o, par);
  resNext[o] = 1;
}

__global__ void k_is_orphan(int n, const int* __restrict__ parents, int* isOrphan, int* res) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  isOrphan[i] = parents[i] == -1 ? 1 : 0;
  res[i] = 0;
}

__global__ void k_relabel(int n, int nseed, const int* __restrict__ seedRank, const int* __restrict__ orphRank,
                          int* parents) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int id = parents[i];
  parents[i] = id < n ? seedRank[id] : nseed + orphRank[id - n];
}

__global__ void k_count_children(int n, const int* __restrict__ parents, int* cnt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) atomicAdd(cnt + parents[i], 1);
}

__global__ void k_fill_children(int n, const int* __restrict__ parents, int* cur, int* child) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) child[atomicAdd(cur + parents[i], 1)] = i;
}

__global__ void k_sort_children(int nc, const int* __restrict__ cs, int* child) {
  const int P = blockIdx.x * blockDim.x + threadIdx.x;
  if (P >= nc) return;
  const int a = cs[P], b = cs[P + 1];
  for (int q = a + 1; q < b; ++q) {
    const int v = child[q];
    int r = q - 1;
    while (r >= a && child[r] > v) { child[r + 1] = child[r]; --r; }
    child[r + 1] = v;
  }
}

__global__ void k_child_nnz(int nc, const int* __restrict__ cs, const int* __restrict__ child,
                            const int* __restrict__ rp, int* cnt) {
  const int P = blockIdx.x * blockDim.x + threadIdx.x;
  if (P >= nc) return;
  int s = 0;
  for (int q = cs[P]; q < cs[P + 1]; ++q) s += rp[child[q] + 1] - rp[child[q]];
  cnt[P] = s;
}

// coarse cconn in discovery order (cfdAgglomerateLevel.m:89-98)
__global__ void k_coarse_conn(int nc, const int* __restrict__ cs, const int* __restrict__ child,
                              const int* __restrict__ rp, const int* __restrict__ col, const int* __restrict__ parents,
                              const int* __restrict__ estart, int* scratch, int* ccnt) {
  const int P = blockIdx.x * blockDim.x + threadIdx.x;
  if (P >= nc) return;
  int* lst = scratch + estart[P];
  int m = 0;
  for (int q = cs[P]; q < cs[P + 1]; ++q) {
    const int c = child[q];
    for (int k = rp[c]; k < rp[c + 1]; ++k) {
      const int Q = parents[col[k]];
      if (Q == P) continue;
      bool seen = false;
      for (int t = 0; t < m && !seen; ++t) seen = lst[t] == Q;
      if (!seen) lst[m++] = Q;
    }
  }
  ccnt[P] = m;
}

__global__ void k_coarse_copy(int nc, const int* __restrict__ estart, const int* __restrict__ scratch,
                              const int* __restrict__ crp, int* ccol) {
  const int P = blockIdx.x * blockDim.x + threadIdx.x;
  if (P >= nc) return;
  const int* lst = scratch + estart[P];
  for (int t = 0; t < crp[P + 1] - crp[P]; ++t) ccol[crp[P] + t] = lst[t];
}

// Galerkin by summation in fine natural order (assembleAgglomeratedLHS.m:16-30)
template <typename T>
__global__ void k_galerkin(int nc, const int* __restrict__ cs, const int* __restrict__ child,
                           const int* __restrict__ rp, const int* __restrict__ col, const int* __restrict__ parents,
                           const T* __restrict__ ac, const T* __restrict__ anb, const int* __restrict__ crp,
                           const int* __restrict__ ccol, T* cac, T* canb) {
  const int P = blockIdx.x * blockDim.x + threadIdx.x;
  if (P >= nc) return;
  const int c0 = crp[P], c1 = crp[P + 1];
  for (int t = c0; t < c1; ++t) canb[t] = 0;
  T AC = 0;
  for (int q = cs[P]; q < cs[P + 1]; ++q) {
    const int c = child[q];
    AC = AC + ac[c];
    for (int k = rp[c]; k < rp[c + 1]; ++k) {
      const int Q = parents[col[k]];
      if (Q == P) {
        AC = AC + anb[k];
      } else {
        int pos = c0;
        while (pos < c1 && ccol[pos] != Q) ++pos;
        if (pos < c1) canb[pos] = canb[pos] + anb[k];
      }
    }
  }
  cac[P] = AC;
}

// ---------------------------------------------------------------------------------
int agglomerate_level(LinCtx& c, AggScratch& w, Level& F, Level& C, int* nCoarse) {
  const int n = F.n;
  UFVM_CHECK(c.ensure(n));
  UFVM_CHECK(dalloc(w.maxAnb, n));
  UFVM_CHECK(dalloc(w.strong, std::max(F.nnz, 1)));
  UFVM_CHECK(dalloc(w.status, n));
  UFVM_CHECK(dalloc(w.win, n));
  UFVM_CHECK(dalloc(w.seedflag, n + 1));
  UFVM_CHECK(dalloc(w.newflag, n + 1));
  UFVM_CHECK(dalloc(w.seedRank, n + 1));
  UFVM_CHECK(dalloc(w.orphRank, n + 1));
  UFVM_CHECK(dalloc(w.resv, n));
  UFVM_CHECK(dalloc(w.res0, n));
  UFVM_CHECK(dalloc(w.res1, n));
  UFVM_CHECK(dalloc(F.parents, n));
  cudaStream_t st = c.stream;
  k_maxanb<<<nblocks(n), kBlock, 0, st>>>(n, F.rowptr.p, F.anb.p, w.maxAnb.p);
  k_strong<<<nblocks(n), kBlock, 0, st>>>(n, F.rowptr.p, F.anb.p, w.maxAnb.p, w.strong.p);
  UFVM_LAUNCH_CHECK();
  UFVM_CUDA(cudaMemsetAsync(F.parents.p, 0xff, n * sizeof(int), st));
  UFVM_CUDA(cudaMemsetAsync(w.status.p, 0, n * sizeof(int), st));
  UFVM_CUDA(cudaMemsetAsync(w.seedflag.p, 0, (n + 1) * sizeof(int), st));
  UFVM_CUDA(cudaMemsetAsync(w.newflag.p, 0, (n + 1) * sizeof(int), st));
  UFVM_CUDA(cudaMemsetAsync(w.resv.p, 0, n * sizeof(unsigned long long), st));
  AggArgs a{n, F.rowptr.p, F.col.p, w.strong.p, F.parents.p, w.status.p, w.resv.p, w.win.p, w.seedflag.p, c.iflag.p};
  // Every round commits at least the lowest unprocessed seed, so n + 1 rounds bound it. The
  // host reads the count of unprocessed seeds after batches of rounds that double in length
  // (4, 8, 16, ... up to 64): a round after the last one finds no unprocessed seed and its
  // kernels return at once, so a longer batch changes no result, only how often the host waits.
  unsigned int round = 0;
  int batch = 4;
  for (;;) {
    int rem = 0;
    for (int k = 0; k < batch; ++k) {
      ++round;
      UFVM_CUDA(cudaMemsetAsync(c.iflag.p, 0, sizeof(int), st));
      k_agg_reserve<<<nblocks(n), kBlock, 0, st>>>(a, round);
      k_agg_check<<<nblocks(n), kBlock, 0, st>>>(a, round);
      k_agg_commit<<<nblocks(n), kBlock, 0, st>>>(a);
    }
    UFVM_LAUNCH_CHECK();
    UFVM_CUDA(cudaMemcpyAsync(&rem, c.iflag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    UFVM_CUDA(cudaStreamSynchronize(st));
    if (rem == 0) break;
    if (round > (unsigned int)n + 8) { set_error("agglomeration rounds did not terminate"); return UFVM_E_INVALID; }
    batch = std::min(2 * batch, 64);
  }
  // orphans
  k_is_orphan<<<nblocks(n), kBlock, 0, st>>>(n, F.parents.p, w.status.p /* isOrphan */, w.res0.p);
  UFVM_CUDA(cudaMemsetAsync(w.res1.p, 0, n * sizeof(int), st));
  // orphan rounds in batches as above (a round after the last finds every orphan resolved)
  for (int r = 0, ob = 2;; ob = std::min(2 * ob, 32)) {
    for (int k = 0; k < ob; ++k, ++r) {
      UFVM_CUDA(cudaMemsetAsync(c.iflag.p, 0, sizeof(int), st));
      k_orphan_round<<<nblocks(n), kBlock, 0, st>>>(n, F.rowptr.p, F.col.p, F.anb.p, w.maxAnb.p, w.status.p,
                                                    w.res0.p, w.res1.p, F.parents.p, w.newflag.p, c.iflag.p);
      UFVM_CUDA(cudaMemcpyAsync(w.res0.p, w.res1.p, n * sizeof(int), cudaMemcpyDeviceToDevice, st));
    }
    UFVM_LAUNCH_CHECK();
    int rem = 0;
    UFVM_CUDA(cudaMemcpyAsync(&rem, c.iflag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    UFVM_CUDA(cudaStreamSynchronize(st));
    if (rem == 0) break;
    if (r > n + 8) { set_error("orphan rounds did not terminate"); return UFVM_E_INVALID; }
  }
  // relabel: seed parents in seed order, then orphans' new parents in orphan order
  int nseed = 0, norph = 0;
  UFVM_CHECK(scan_exclusive(c, w.seedflag.p, w.seedRank.p, n, &nseed));
  UFVM_CHECK(scan_exclusive(c, w.newflag.p, w.orphRank.p, n, &norph));
  k_relabel<<<nblocks(n), kBlock, 0, st>>>(n, nseed, w.seedRank.p, w.orphRank.p, F.parents.p);
  UFVM_LAUNCH_CHECK();
  const int nc = nseed + norph;
  *nCoarse = nc;
  // children of each coarse row, sorted by fine index
  UFVM_CHECK(dalloc(w.cnt, nc + 1));
  UFVM_CHECK(dalloc(F.childStart, nc + 1));
  UFVM_CHECK(dalloc(F.child, n));
  UFVM_CUDA(cudaMemsetAsync(w.cnt.p, 0, (nc + 1) * sizeof(int), st));
  k_count_children<<<nblocks(n), kBlock, 0, st>>>(n, F.parents.p, w.cnt.p);
  UFVM_CHECK(scan_exclusive(c, w.cnt.p, F.childStart.p, nc, nullptr));
  UFVM_CUDA(cudaMemcpyAsync(w.cnt.p, F.childStart.p, nc * sizeof(int), cudaMemcpyDeviceToDevice, st));
  k_fill_children<<<nblocks(n), kBlock, 0, st>>>(n, F.parents.p, w.cnt.p, F.child.p);
  k_sort_children<<<nblocks(nc), kBlock, 0, st>>>(nc, F.childStart.p, F.child.p);
  UFVM_LAUNCH_CHECK();
  // coarse connectivity
  UFVM_CHECK(dalloc(w.estart, nc + 1));
  k_child_nnz<<<nblocks(nc), kBlock, 0, st>>>(nc, F.childStart.p, F.child.p, F.rowptr.p, w.cnt.p);
  int etot = 0;
  UFVM_CHECK(scan_exclusive(c, w.cnt.p, w.estart.p, nc, &etot));
  UFVM_CHECK(dalloc(w.lists, std::max(etot, 1)));
  k_coarse_conn<<<nblocks(nc), kBlock, 0, st>>>(nc, F.childStart.p, F.child.p, F.rowptr.p, F.col.p, F.parents.p,
                                                w.estart.p, w.lists.p, w.cnt.p);
  UFVM_LAUNCH_CHECK();
  C.n = nc;
  UFVM_CHECK(dalloc(C.rowptr, nc + 1));
  int cnnz = 0;
  UFVM_CHECK(scan_exclusive(c, w.cnt.p, C.rowptr.p, nc, &cnnz));
  C.nnz = cnnz;
  UFVM_CHECK(dalloc(C.col, std::max(cnnz, 1)));
  k_coarse_copy<<<nblocks(nc), kBlock, 0, st>>>(nc, w.estart.p, w.lists.p, C.rowptr.p, C.col.p);
  UFVM_LAUNCH_CHECK();
  UFVM_CHECK(dalloc(C.ac, nc));
  UFVM_CHECK(dalloc(C.anb, std::max(cnnz, 1)));
  UFVM_CHECK(dalloc(C.bc, nc));
  UFVM_CHECK(dalloc(C.dphi, nc));
  UFVM_CUDA(cudaMemsetAsync(C.bc.p, 0, nc * sizeof(double), st));
  UFVM_CUDA(cudaMemsetAsync(C.dphi.p, 0, nc * sizeof(double), st));
  C.sched_valid = false;
  C.color_valid = false;
  C.mc_valid = false;
  return galerkin(c, F, C);
}

int galerkin(LinCtx& c, Level& F, Level& C) {
  k_galerkin<double><<<nblocks(C.n), kBlock, 0, c.stream>>>(C.n, F.childStart.p, F.child.p, F.rowptr.p, F.col.p,
                                                             F.parents.p, F.ac.p, F.anb.p, C.rowptr.p, C.col.p,
                                                             C.ac.p, C.anb.p);
  UFVM_LAUNCH_CHECK();
  return UFVM_OK;
}

int galerkin32(LinCtx& c, Level& F, Level& C) {
  k_galerkin<float><<<nblocks(C.n), kBlock, 0, c.stream>>>(C.n, F.childStart.p, F.child.p, F.rowptr.p, F.col.p,
                                                            F.parents.p, F.ac32.p, F.anb32.p, C.rowptr.p, C.col.p,
                                                            C.ac32.p, C.anb32.p);
  UFVM_LAUNCH_CHECK();
  return UFVM_OK;
}

void AggScratch::release() {
  dfree(maxAnb); dfree(strong); dfree(status); dfree(win); dfree(seedflag); dfree(newflag); dfree(seedRank);
  dfree(orphRank); dfree(resv); dfree(res0); dfree(res1); dfree(cnt); dfree(estart); dfree(lists);
}

// ---------------------------------------------------------------------------------
// AMG driver on a hierarchy whose level 0 is the assembled p matrix.
// A rebuild (every p solve in the reference, cfdApplyAMG.m:19) keeps the previous hierarchy's
// coarse-level device arrays and hands them to the new levels, whose allocations (dalloc) reuse an
// array that is large enough instead of freeing and allocating it again; every schedule,
// colouring and copy cached on a level is invalidated, since the new level's pattern may differ.
static void reset_level_caches(Level& L) {
  L.sched_valid = false;
  L.nfwd = L.nbwd = L.maxw = 0;
  L.dc_epoch = 0;
  L.dc_quirks = 0;
  for (int k = 0; k < 4; ++k) {
    L.sell_valid[k] = false;
    L.sellW[k] = 0;
    L.sell_epoch[k] = 0;
  }
  L.color_valid = false;
  L.ncolor = 0;
  L.h_colorStart.clear();
  L.mc_valid = false;
  L.mcW = 0;
  L.mc_epoch = 0;
  L.ell_valid = false;
  L.ellW = 0;
}

int AmgSolver::build(std::vector<Level>& lev, int max_coarse, int quirks, int* n_levels) {
  std::vector<Level> pool(lev.begin() + 1, lev.end());
  lev.resize(1);
  size_t next = 0;
  auto release_pool = [&]() {
    for (size_t k = next; k < pool.size(); ++k) free_level(pool[k]);
    pool.clear();
  };
  int il = 0;
  while (il < max_coarse) {
    ++il;
    Level coarse;
    if (next < pool.size()) {
      coarse = pool[next];
      pool[next++] = Level();
      reset_level_caches(coarse);
    }
    int np = 0;
    const int st = agglomerate_level(ctx, agg, lev[il - 1], coarse, &np);
    if (st != UFVM_OK) {
      free_level(coarse);
      release_pool();
      return st;
    }
    if (np == 1 && !(quirks & UFVM_Q16_ONE_CELL_COARSEST)) {
      // repaired: a single aggregate of the pure-Neumann operator has a ~0 diagonal
      free_level(coarse);
      --il;
      break;
    }
    lev.push_back(coarse);
    if (np <= 5) break;
  }
  release_pool();
  *n_levels = il + 1;
  return UFVM_OK;
}

void free_level(Level& L, bool keep_matrix) {
  if (!keep_matrix) { dfree(L.rowptr); dfree(L.col); dfree(L.ac); dfree(L.anb); dfree(L.bc); dfree(L.dphi); }
  dfree(L.parents); dfree(L.tpos); dfree(L.lord); dfree(L.r); dfree(L.dc); dfree(L.rc); dfree(L.lvl); dfree(L.fwdRows);
  dfree(L.fwdStart); dfree(L.bwdRows); dfree(L.bwdStart); dfree(L.color); dfree(L.colorRows); dfree(L.colorStart);
  dfree(L.childStart); dfree(L.child); dfree(L.ac32); dfree(L.anb32); dfree(L.bc32); dfree(L.dphi32); dfree(L.r32);
  dfree(L.fr); dfree(L.fp); dfree(L.fq);
  dfree(L.perm); dfree(L.inv); dfree(L.ellCol); dfree(L.parentsP); dfree(L.childP); dfree(L.childStartP); dfree(L.gpos);
  dfree(L.ellAnb); dfree(L.uAnb); dfree(L.uAc); dfree(L.uBc); dfree(L.uX);
  dfree(L.mcRow); dfree(L.mcCol); dfree(L.mcAnb); dfree(L.mcAc); dfree(L.mcBc);
  for (int k = 0; k < 4; ++k) {
    dfree(L.sellCol[k]); dfree(L.sellA[k]);
    L.sell_valid[k] = false;
    L.sell_epoch[k] = 0;
  }
  L.mc_valid = false;
  L.mc_epoch = 0;
  L.ell_valid = false;
  L.sched_valid = false;
  L.color_valid = false;
  L.dc_epoch = 0;
}

int AmgSolver::smooth(std::vector<Level>& lev, int l, int n_iter, double rrf) {
  return solve_algebraic_system(ctx, lev[l], smoother, n_iter, rrf, quirks, nullptr, nullptr, nullptr);
}

int AmgSolver::restrict_(std::vector<Level>& lev, int l, int pre) {
  if (pre >= 0) UFVM_CHECK(smooth(lev, l, pre, 0.1));
  UFVM_CHECK(restrict_residual(ctx, lev[l], lev[l + 1]));
  if (!(quirks & UFVM_Q6_COARSE_DPHI_KEPT))
    UFVM_CUDA(cudaMemsetAsync(lev[l + 1].dphi.p, 0, lev[l + 1].n * sizeof(double), ctx.stream));
  return UFVM_OK;
}

int AmgSolver::prolong_(std::vector<Level>& lev, int l, double rrf) {
  UFVM_CHECK(prolong(ctx, lev[l - 1], lev[l]));
  return smooth(lev, l - 1, post, rrf);
}

int AmgSolver::cycle(std::vector<Level>& lev, int L, double rrf, double* fin) {
  auto R = [&](int l, int p) { return restrict_(lev, l, p); };
  auto Pr = [&](int l) { return prolong_(lev, l, rrf); };
  auto solveC = [&]() { return smooth(lev, L, post, 0.1); };
  if (cycle_type != UFVM_CYCLE_V && L < 3) {
    set_error("W/F-cycle needs at least 4 AMG levels (the reference indexes level 0)");
    return UFVM_E_AMG_LEVELS;
  }
  for (int l = 0; l < L; ++l) UFVM_CHECK(R(l, pre));
  UFVM_CHECK(solveC());
  if (cycle_type == UFVM_CYCLE_W || cycle_type == UFVM_CYCLE_F) {
    UFVM_CHECK(Pr(L)); UFVM_CHECK(R(L - 1, -1)); UFVM_CHECK(solveC());
    UFVM_CHECK(Pr(L)); UFVM_CHECK(Pr(L - 1)); UFVM_CHECK(R(L - 2, -1)); UFVM_CHECK(R(L - 1, pre)); UFVM_CHECK(solveC());
    UFVM_CHECK(Pr(L)); UFVM_CHECK(Pr(L - 1)); UFVM_CHECK(Pr(L - 2));
    UFVM_CHECK(R(L - 3, -1)); UFVM_CHECK(R(L - 2, pre)); UFVM_CHECK(R(L - 1, pre)); UFVM_CHECK(solveC());
    if (cycle_type == UFVM_CYCLE_W) {
      UFVM_CHECK(Pr(L)); UFVM_CHECK(Pr(L - 1)); UFVM_CHECK(R(L - 2, -1)); UFVM_CHECK(R(L - 1, pre)); UFVM_CHECK(solveC());
      UFVM_CHECK(Pr(L)); UFVM_CHECK(R(L - 1, -1)); UFVM_CHECK(solveC());
    }
  }
  for (int l = L; l >= 1; --l) UFVM_CHECK(Pr(l));
  return sum_abs_residual(ctx, lev[0], lev[0].dphi.p, fin);
}

int AmgSolver::apply(std::vector<Level>& lev, bool rebuild, int* n_levels, double* r0, double* r1) {
  if (rebuild) UFVM_CHECK(build(lev, max_coarse, quirks, n_levels));
  else {
    for (int l = 1; l < *n_levels; ++l) {
      UFVM_CHECK(galerkin(ctx, lev[l - 1], lev[l]));
      UFVM_CUDA(cudaMemsetAsync(lev[l].bc.p, 0, lev[l].n * sizeof(double), ctx.stream));
      UFVM_CUDA(cudaMemsetAsync(lev[l].dphi.p, 0, lev[l].n * sizeof(double), ctx.stream));
    }
  }
  const int L = *n_levels - 1;
  double init = 0;
  UFVM_CHECK(sum_abs_residual(ctx, lev[0], lev[0].dphi.p, &init));
  double fin = init;
  int ncyc = 1;
  // the matrices are final from here to the end of this solve: a fresh epoch lets the smoother
  // calls of the cycles share each level's DILU factor
  static std::atomic<unsigned long long> epochs{0};
  struct EpochScope {
    LinCtx& c;
    ~EpochScope() { c.factor_epoch = 0; }
  } scope{ctx};
  ctx.factor_epoch = epochs.fetch_add(1) + 1;
  while (ncyc <= max_cycles && fin > rrf * init) {
    UFVM_CHECK(cycle(lev, L, rrf, &fin));
    ++ncyc;
  }
  cycles_used = ncyc - 1;
  *r0 = init;
  *r1 = fin;
  return UFVM_OK;
}

}  // namespace ufvm
