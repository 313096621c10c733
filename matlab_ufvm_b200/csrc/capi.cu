// capi.cu -- the extern "C" boundary of libufvm.so (declared in include/ufvm.h) and the
// steady SIMPLE driver (top/cfdRunCase.m:92-142).
#include <chrono>
#include <cmath>
#include <cstring>
#include <mutex>

#include "amg.cuh"

namespace ufvm {

static thread_local std::string g_err;
void set_error(const std::string& m) { g_err = m; }
const char* get_error() { return g_err.c_str(); }
double host_ms_now() {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

Case::~Case() {
  if (amg) {
    amg->agg.release();
    delete amg;
  }
  for (size_t l = 0; l < lev.size(); ++l) {
    if (l == 0) { lev[0].rowptr.p = nullptr; lev[0].col.p = nullptr; }  // shared with the mesh
    free_level(lev[l]);
  }
  lin.release();
  DMesh& m = M;
  for (auto* a : {&m.owner, &m.neigh, &m.cfStart, &m.cfFace, &m.rowptr, &m.col, &m.ownSlot, &m.neiSlot, &m.bPatch})
    dfree(*a);
  for (auto* a : {&m.fCx, &m.fCy, &m.fCz, &m.Sx, &m.Sy, &m.Sz, &m.area, &m.CNx, &m.CNy, &m.CNz, &m.eCx, &m.eCy, &m.eCz,
                  &m.gDiff, &m.Tx, &m.Ty, &m.Tz, &m.gf, &m.wd, &m.vol, &m.cCx, &m.cCy, &m.cCz})
    dfree(*a);
  for (auto* a : {&D.ptype, &D.pstart, &D.pcount, &D.bcU, &D.bcP}) dfree(*a);
  dfree(D.pnsum);
  for (int c = 0; c < 3; ++c) { dfree(U[c]); dfree(gp[c]); dfree(gPP[c]); dfree(DU[c]); dfree(vU[c]); }
  for (int k = 0; k < 9; ++k) dfree(gU[k]);
  dfree(p); dfree(PP); dfree(mdot); dfree(fC1); dfree(fC2); dfree(vP); dfree(tmp3); dfree(uft);
  dfree(part); dfree(red); dfree(flags); dfree(scal); dfree(slot);
  dfree(wl.cells); dfree(wl.faces); dfree(wl.bfaces); dfree(wl.urows);
  dfree(wl.cstart); dfree(wl.cend); dfree(wl.ustart); dfree(wl.uend);
  if (stream && owns_stream) cudaStreamDestroy(stream);
}

// solve/cfdSolveEquation.m:11-18
int Case::solve(int eq, double* r0, double* r1) {
  if (eq == UFVM_EQ_P && S.p_amg) {
    AmgSolver& A = *amg;
    A.smoother = S.p_smoother; A.quirks = S.quirks; A.pre = S.p_pre_sweep; A.post = S.p_post_sweep;
    A.max_cycles = S.p_max_cycles; A.max_coarse = S.p_max_coarse_levels; A.cycle_type = S.p_cycle;
    A.rrf = S.p_termination;
    const bool rebuild = S.hierarchy_reuse <= 0 || !hierarchy_valid || (p_solves % S.hierarchy_reuse) == 0;
    ++p_solves;
    UFVM_CHECK(A.apply(lev, rebuild, &n_levels, r0, r1));
    hierarchy_valid = true;
    last_amg_cycles = A.cycles_used;
    return UFVM_OK;
  }
  const int sm = eq == UFVM_EQ_P ? S.p_smoother : S.u_smoother;
  const int nit = eq == UFVM_EQ_P ? 10 : S.u_n_iter;
  const double rrf = eq == UFVM_EQ_P ? 0.1 : S.u_rrf;
  return solve_algebraic_system(lin, lev[0], sm, nit, rrf, S.quirks, r0, r1, nullptr);
}

// one steady iteration of cfdRunCase (update -> U(x,y,z) -> p x nCorrectors -> convergence)
int Case::iterate(double* res, int* converged) {
  UFVM_CHECK(update_fields());
  for (int c = 0; c < 3; ++c) {
    UFVM_CHECK(assemble_u(c, &res[c], &res[4 + c]));
    UFVM_CHECK(solve(UFVM_EQ_U, &res[8 + c], &res[12 + c]));
    UFVM_CHECK(correct_u(c));
  }
  for (int k = 0; k < S.n_correctors; ++k) {
    UFVM_CHECK(assemble_p(&res[3], &res[7]));
    UFVM_CHECK(solve(UFVM_EQ_P, &res[11], &res[15]));
    UFVM_CHECK(correct_p());
  }
  UFVM_CUDA(cudaStreamSynchronize(stream));
  for (int i = 0; i < 4; ++i)
    if (std::isnan(res[i])) { set_error("Divergence detected!"); return UFVM_E_NAN; }
  *converged = (res[0] <= S.tol_u && res[1] <= S.tol_u && res[2] <= S.tol_u && res[3] <= S.tol_p) ? 1 : 0;
  return UFVM_OK;
}

// Builds a case in place. `shared` is a stream owned by the caller (a service), or null
// for a case that owns its own stream.
int create_case_into(Case& C, const ufvm_mesh_desc* mesh, const ufvm_settings& settings, const int32_t* bc_type_u,
                     const int32_t* bc_type_p, const double* bc_val_u, const double* bc_val_p, const double* U0,
                     const double* p0, const double* mdot0, cudaStream_t shared) {
  C.S = settings;
  if (shared) {
    C.stream = shared;
    C.owns_stream = false;
  } else if (cudaStreamCreateWithFlags(&C.stream, cudaStreamNonBlocking) != cudaSuccess) {
    C.stream = nullptr;
    set_error("cudaStreamCreate failed (no CUDA device?)");
    return UFVM_E_CUDA;
  }
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&C.nsm, cudaDevAttrMultiProcessorCount, dev);
  C.lin.stream = C.stream;
  C.lin.nsm = C.nsm;
  C.amg = new AmgSolver(C.lin);
  UFVM_CHECK(C.build_mesh(mesh));
  UFVM_CHECK(C.init_fields(bc_type_u, bc_type_p, bc_val_u, bc_val_p, U0, p0, mdot0));
  UFVM_CHECK(C.lin.ensure(C.M.F));
  return UFVM_OK;
}

}  // namespace ufvm

using namespace ufvm;

struct ufvm_case {
  Case c;
};

#define API_GUARD(expr)                                  \
  try {                                                  \
    return (expr);                                       \
  } catch (const std::exception& ex) {                   \
    set_error(std::string("exception: ") + ex.what());   \
    return UFVM_E_INVALID;                               \
  }

extern "C" {

const char* ufvm_last_error(void) { return get_error(); }
const char* ufvm_version(void) { return "ufvm-b200 0.1 (sm_100a, FP64 reference-order + MCGS/FP32-AMG)"; }

int ufvm_case_create(const ufvm_mesh_desc* mesh, const ufvm_settings* settings, const int32_t* bc_type_u,
                     const int32_t* bc_type_p, const double* bc_val_u, const double* bc_val_p, const double* U0,
                     const double* p0, const double* mdot0, ufvm_case** out) {
  if (!mesh || !settings || !bc_type_u || !bc_type_p || !bc_val_u || !bc_val_p || !out) {
    set_error("null argument");
    return UFVM_E_INVALID;
  }
  *out = nullptr;
  ufvm_case* h = new ufvm_case();
  const int st = ufvm::create_case_into(h->c, mesh, *settings, bc_type_u, bc_type_p, bc_val_u, bc_val_p, U0, p0,
                                        mdot0, nullptr);
  if (st != UFVM_OK) {
    delete h;
    return st;
  }
  *out = h;
  return UFVM_OK;
}

int ufvm_case_destroy(ufvm_case* c) {
  delete c;
  return UFVM_OK;
}

int ufvm_case_sizes(const ufvm_case* c, int64_t* s) {
  if (!c || !s) return UFVM_E_INVALID;
  s[0] = c->c.M.Nc; s[1] = c->c.M.F; s[2] = c->c.M.Fi; s[3] = c->c.M.nnz;
  return UFVM_OK;
}

int ufvm_update_fields(ufvm_case* c) {
  if (!c) return UFVM_E_INVALID;
  API_GUARD(c->c.update_fields());
}

int ufvm_assemble_equation(ufvm_case* c, int eq, int comp, double* rms, double* mx) {
  if (!c || !rms || !mx || (eq != UFVM_EQ_U && eq != UFVM_EQ_P)) return UFVM_E_INVALID;
  if (eq == UFVM_EQ_U) {
    if (comp < 0 || comp > 2) return UFVM_E_INVALID;
    API_GUARD(c->c.assemble_u(comp, rms, mx));
  }
  API_GUARD(c->c.assemble_p(rms, mx));
}

int ufvm_solve_equation(ufvm_case* c, int eq, double* r0, double* r1) {
  if (!c || !r0 || !r1 || (eq != UFVM_EQ_U && eq != UFVM_EQ_P)) return UFVM_E_INVALID;
  API_GUARD(c->c.solve(eq, r0, r1));
}

int ufvm_correct_equation(ufvm_case* c, int eq, int comp) {
  if (!c || (eq != UFVM_EQ_U && eq != UFVM_EQ_P)) return UFVM_E_INVALID;
  if (eq == UFVM_EQ_U) {
    if (comp < 0 || comp > 2) return UFVM_E_INVALID;
    API_GUARD(c->c.correct_u(comp));
  }
  API_GUARD(c->c.correct_p());
}

int ufvm_simple_iteration(ufvm_case* c, double* res, int* converged) {
  if (!c || !res || !converged) return UFVM_E_INVALID;
  API_GUARD(c->c.iterate(res, converged));
}

int ufvm_run_case(ufvm_case* c, int max_iter, int* iterations, double* res) {
  if (!c || !res) return UFVM_E_INVALID;
  int conv = 0, it = 0;
  while (it < max_iter) {
    ++it;
    const int st = c->c.iterate(res, &conv);
    if (st != UFVM_OK) {
      if (iterations) *iterations = it;
      return st;
    }
    if (conv) break;
  }
  if (iterations) *iterations = it;
  return conv ? UFVM_OK : UFVM_E_NOT_CONVERGED;
}

static int copy_out(cudaStream_t st, const double* d, size_t n, double* host, int64_t cap, int64_t& off) {
  if ((int64_t)(off + n) > cap) { set_error("host buffer too small"); return UFVM_E_INVALID; }
  if (n) UFVM_CUDA(cudaMemcpyAsync(host + off, d, n * sizeof(double), cudaMemcpyDeviceToHost, st));
  off += n;
  return UFVM_OK;
}

int ufvm_get_field(ufvm_case* h, const char* name, double* host, int64_t n, int64_t* written) {
  if (!h || !name) return UFVM_E_INVALID;
  Case& C = h->c;
  const size_t R = C.M.Nc + C.M.Fb;
  std::string s(name);
  int64_t off = 0;
  int st = UFVM_OK;
  auto put = [&](const double* d, size_t cnt) {
    if (!host) { off += cnt; return; }  // size query
    if (st == UFVM_OK) st = copy_out(C.stream, d, cnt, host, n, off);
  };
  if (s == "U") { for (int c = 0; c < 3; ++c) put(C.U[c].p, C.rowsU); }
  else if (s == "gradU") { for (int k = 0; k < 9; ++k) put(C.gU[k].p, R); }
  else if (s == "p") put(C.p.p, R);
  else if (s == "gradp") { for (int d = 0; d < 3; ++d) put(C.gp[d].p, R); }
  else if (s == "PP") put(C.PP.p, R);
  else if (s == "gradPP") { for (int d = 0; d < 3; ++d) put(C.gPP[d].p, R); }
  else if (s == "DU") { for (int c = 0; c < 3; ++c) put(C.DU[c].p, R); }
  else if (s == "mdot") put(C.mdot.p, C.M.F);
  else if (s == "fluxC1") put(C.fC1.p, C.M.F);
  else if (s == "fluxC2") put(C.fC2.p, C.M.F);
  else if (s == "ac") put(C.lev[0].ac.p, C.M.Nc);
  else if (s == "bc") put(C.lev[0].bc.p, C.M.Nc);
  else if (s == "anb") put(C.lev[0].anb.p, C.M.nnz);
  else if (s == "dphi") put(C.lev[0].dphi.p, C.M.Nc);
  else if (s == "scaleU") {
    if (host && n >= 1) host[0] = C.scaleU;
    off = 1;
  } else {
    set_error("unknown field " + s);
    return UFVM_E_INVALID;
  }
  if (st != UFVM_OK) return st;
  UFVM_CUDA(cudaStreamSynchronize(C.stream));
  if (written) *written = off;
  return UFVM_OK;
}

int ufvm_set_field(ufvm_case* h, const char* name, const double* host, int64_t n) {
  if (!h || !name || !host) return UFVM_E_INVALID;
  Case& C = h->c;
  const size_t R = C.M.Nc + C.M.Fb;
  std::string s(name);
  std::vector<std::pair<double*, size_t>> dst;
  if (s == "U") { for (int c = 0; c < 3; ++c) dst.push_back({C.U[c].p, (size_t)C.rowsU}); }
  else if (s == "p") dst.push_back({C.p.p, R});
  else if (s == "mdot") dst.push_back({C.mdot.p, (size_t)C.M.F});
  else if (s == "DU") { for (int c = 0; c < 3; ++c) dst.push_back({C.DU[c].p, R}); }
  else if (s == "gradp") { for (int d = 0; d < 3; ++d) dst.push_back({C.gp[d].p, R}); }
  else if (s == "gradU") { for (int k = 0; k < 9; ++k) dst.push_back({C.gU[k].p, R}); }
  else if (s == "dphi") dst.push_back({C.lev[0].dphi.p, (size_t)C.M.Nc});
  else { set_error("unknown field " + s); return UFVM_E_INVALID; }
  size_t tot = 0;
  for (auto& d : dst) tot += d.second;
  if ((int64_t)tot != n) { set_error("size mismatch for " + s); return UFVM_E_INVALID; }
  size_t off = 0;
  for (auto& d : dst) {
    UFVM_CUDA(cudaMemcpyAsync(d.first, host + off, d.second * sizeof(double), cudaMemcpyHostToDevice, C.stream));
    off += d.second;
  }
  UFVM_CUDA(cudaStreamSynchronize(C.stream));
  return UFVM_OK;
}

int ufvm_get_geometry(ufvm_case* h, const char* name, double* host, int64_t n) {
  if (!h || !name || !host) return UFVM_E_INVALID;
  Case& C = h->c;
  DMesh& M = C.M;
  std::string s(name);
  std::vector<const double*> comps;
  size_t cnt = M.F;
  if (s == "Sf") comps = {M.Sx.p, M.Sy.p, M.Sz.p};
  else if (s == "centroid_f") comps = {M.fCx.p, M.fCy.p, M.fCz.p};
  else if (s == "CN") comps = {M.CNx.p, M.CNy.p, M.CNz.p};
  else if (s == "eCN") comps = {M.eCx.p, M.eCy.p, M.eCz.p};
  else if (s == "T") comps = {M.Tx.p, M.Ty.p, M.Tz.p};
  else if (s == "area") comps = {M.area.p};
  else if (s == "gDiff") comps = {M.gDiff.p};
  else if (s == "gf") comps = {M.gf.p};
  else if (s == "walldist") comps = {M.wd.p};
  else if (s == "volume") { comps = {M.vol.p}; cnt = M.Nc; }
  else if (s == "centroid_c") { comps = {M.cCx.p, M.cCy.p, M.cCz.p}; cnt = M.Nc; }
  else { set_error("unknown geometry " + s); return UFVM_E_INVALID; }
  const size_t nc = comps.size();
  if ((int64_t)(cnt * nc) > n) { set_error("host buffer too small"); return UFVM_E_INVALID; }
  std::vector<double> tmp(cnt);
  for (size_t c = 0; c < nc; ++c) {
    UFVM_CUDA(cudaMemcpy(tmp.data(), comps[c], cnt * sizeof(double), cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < cnt; ++i) host[i * nc + c] = tmp[i];
  }
  return UFVM_OK;
}

int ufvm_get_levels(ufvm_case* h, int* n_levels, int64_t* sizes, int max_levels) {
  if (!h || !n_levels) return UFVM_E_INVALID;
  Case& C = h->c;
  *n_levels = C.n_levels;
  if (sizes)
    for (int l = 0; l < std::min(max_levels, C.n_levels); ++l) sizes[l] = C.lev[l].n;
  return UFVM_OK;
}

int ufvm_get_level_array(ufvm_case* h, int level, const char* name, void* host, int64_t n, int64_t* written) {
  if (!h || !name) return UFVM_E_INVALID;
  Case& C = h->c;
  if (level < 0 || level >= C.n_levels) { set_error("level out of range"); return UFVM_E_INVALID; }
  Level& L = C.lev[level];
  std::string s(name);
  const void* src = nullptr;
  size_t cnt = 0, es = 4;
  if (s == "parents") { src = L.parents.p; cnt = level + 1 < C.n_levels ? L.n : 0; }
  else if (s == "rowptr") { src = L.rowptr.p; cnt = L.n + 1; }
  else if (s == "col") { src = L.col.p; cnt = L.nnz; }
  else if (s == "color") { src = L.color.p; cnt = L.color_valid ? L.n : 0; }
  else if (s == "ac") { src = L.ac.p; cnt = L.n; es = 8; }
  else if (s == "anb") { src = L.anb.p; cnt = L.nnz; es = 8; }
  else { set_error("unknown level array " + s); return UFVM_E_INVALID; }
  if (written) *written = cnt;
  if (!host) return UFVM_OK;
  if ((int64_t)cnt > n) { set_error("host buffer too small"); return UFVM_E_INVALID; }
  if (cnt) UFVM_CUDA(cudaMemcpy(host, src, cnt * es, cudaMemcpyDeviceToHost));
  return UFVM_OK;
}

// ---------------------------------------------------------------- stand-alone matrix API
static Level borrow(int32_t n, const int32_t* rp, const int32_t* col, const double* ac, const double* anb,
                    const double* bc, double* dphi, int nnz) {
  Level L;
  L.n = n; L.nnz = nnz;
  L.rowptr.p = const_cast<int*>(rp); L.col.p = const_cast<int*>(col);
  L.ac.p = const_cast<double*>(ac); L.anb.p = const_cast<double*>(anb);
  L.bc.p = const_cast<double*>(bc); L.dphi.p = dphi;
  return L;
}

static void unborrow(Level& L) {
  L.rowptr.p = nullptr; L.col.p = nullptr; L.ac.p = nullptr; L.anb.p = nullptr; L.bc.p = nullptr; L.dphi.p = nullptr;
  free_level(L);
}

static int nnz_of(int32_t n, const int32_t* rp, cudaStream_t st, int* out) {
  int v = 0;
  UFVM_CUDA(cudaMemcpyAsync(&v, rp + n, sizeof(int), cudaMemcpyDeviceToHost, st));
  UFVM_CUDA(cudaStreamSynchronize(st));
  *out = v;
  return UFVM_OK;
}

int ufvm_compute_residuals_array(int32_t n, const int32_t* rowptr, const int32_t* col, const double* ac,
                                 const double* anb, const double* bc, const double* dphi, double* r, void* stream) {
  if (n <= 0 || !rowptr || !col || !ac || !anb || !bc || !dphi || !r) { set_error("bad argument"); return UFVM_E_INVALID; }
  LinCtx c;
  c.stream = (cudaStream_t)stream;
  Level L = borrow(n, rowptr, col, ac, anb, bc, const_cast<double*>(dphi), 0);
  const int st = residual(c, L, dphi, r);
  unborrow(L);
  return st;
}

int ufvm_solve_sor(int32_t n, const int32_t* rowptr, const int32_t* col, const double* ac, const double* anb,
                   const double* bc, double* dphi, void* stream) {
  if (n <= 0 || !rowptr || !col || !ac || !anb || !bc || !dphi) { set_error("bad argument"); return UFVM_E_INVALID; }
  LinCtx c;
  c.stream = (cudaStream_t)stream;
  int nnz = 0;
  UFVM_CHECK(nnz_of(n, rowptr, c.stream, &nnz));
  Level L = borrow(n, rowptr, col, ac, anb, bc, dphi, nnz);
  int st = gs_sweep(c, L);
  cudaStreamSynchronize(c.stream);
  unborrow(L);
  c.release();
  return st;
}

int ufvm_factorize_ilu(int32_t n, const int32_t* rowptr, const int32_t* col, const double* ac, const double* anb,
                       double* dc, int32_t quirks, void* stream) {
  if (n <= 0 || !rowptr || !col || !ac || !anb || !dc) { set_error("bad argument"); return UFVM_E_INVALID; }
  LinCtx c;
  c.stream = (cudaStream_t)stream;
  int nnz = 0;
  UFVM_CHECK(nnz_of(n, rowptr, c.stream, &nnz));
  Level L = borrow(n, rowptr, col, ac, anb, nullptr, nullptr, nnz);
  L.dc.p = dc;
  L.dc.n = n;
  int st = ilu_factor(c, L, quirks);
  cudaStreamSynchronize(c.stream);
  L.dc.p = nullptr;
  unborrow(L);
  c.release();
  return st;
}

int ufvm_solve_ilu(int32_t n, const int32_t* rowptr, const int32_t* col, const double* ac, const double* anb,
                   const double* bc, const double* dc, double* dphi, void* stream) {
  if (n <= 0 || !rowptr || !col || !ac || !anb || !bc || !dc || !dphi) { set_error("bad argument"); return UFVM_E_INVALID; }
  LinCtx c;
  c.stream = (cudaStream_t)stream;
  int nnz = 0;
  UFVM_CHECK(nnz_of(n, rowptr, c.stream, &nnz));
  Level L = borrow(n, rowptr, col, ac, anb, bc, dphi, nnz);
  L.dc.p = const_cast<double*>(dc);
  L.dc.n = n;
  int st = ilu_sweep(c, L);
  cudaStreamSynchronize(c.stream);
  L.dc.p = nullptr;
  unborrow(L);
  c.release();
  return st;
}

int ufvm_solve_algebraic_system(int32_t n, const int32_t* rowptr, const int32_t* col, const double* ac,
                                const double* anb, const double* bc, double* dphi, int32_t smoother, int32_t n_iter,
                                double rrf, int32_t quirks, double* r0, double* r1, int32_t* iters, void* stream) {
  if (n <= 0 || !rowptr || !col || !ac || !anb || !bc || !dphi) { set_error("bad argument"); return UFVM_E_INVALID; }
  LinCtx c;
  c.stream = (cudaStream_t)stream;
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&c.nsm, cudaDevAttrMultiProcessorCount, dev);
  int nnz = 0;
  UFVM_CHECK(nnz_of(n, rowptr, c.stream, &nnz));
  Level L = borrow(n, rowptr, col, ac, anb, bc, dphi, nnz);
  int it = 0;
  int st = solve_algebraic_system(c, L, smoother, n_iter, rrf, quirks, r0, r1, &it);
  if (iters) *iters = it;
  cudaStreamSynchronize(c.stream);
  unborrow(L);
  c.release();
  return st;
}

// Profiling of the stand-alone kernels: schedules, colourings and factors are prepared and
// one launch is made untimed; then every timed launch follows a read of twice the L2 size (the
// cache holds clean unrelated lines, nothing of the system and nothing dirty) and is bracketed
// by CUDA events on the caller's stream.
__global__ void k_flush_read(const float4* __restrict__ a, size_t n4, float* sink) {
  float s = 0.f;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n4; i += (size_t)gridDim.x * blockDim.x) {
    const float4 v = a[i];
    s += v.x + v.y + v.z + v.w;
  }
  if (s == 1.2345e-30f) *sink = s;  // never true for the zeroed buffer; keeps the loads
}

int ufvm_profile_plain_kernel(int32_t kernel, int32_t n, const int32_t* rowptr, const int32_t* col, const double* ac,
                              const double* anb, const double* bc, double* dphi, int32_t reps, double* ms_per_launch,
                              double* bytes_per_launch, void* stream) {
  if (n <= 0 || !rowptr || !col || !ac || !anb || !bc || !dphi || reps <= 0 || !ms_per_launch || !bytes_per_launch ||
      kernel < 0 || kernel > 3) {
    set_error("ufvm_profile_plain_kernel: bad argument");
    return UFVM_E_INVALID;
  }
  LinCtx c;
  c.stream = (cudaStream_t)stream;
  int dev = 0;
  UFVM_CUDA(cudaGetDevice(&dev));
  cudaDeviceGetAttribute(&c.nsm, cudaDevAttrMultiProcessorCount, dev);
  int l2 = 0;
  cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev);
  int nnz = 0;
  UFVM_CHECK(nnz_of(n, rowptr, c.stream, &nnz));
  Level L = borrow(n, rowptr, col, ac, anb, bc, dphi, nnz);
  DArr<double> r;
  DArr<float4> flush;
  DArr<float> sink;
  cudaEvent_t a = nullptr, b = nullptr;
  auto body = [&]() -> int {
    const size_t n4 = std::max<size_t>(2 * (size_t)std::max(l2, 1 << 20) / sizeof(float4), 1);
    UFVM_CHECK(dalloc(flush, n4));
    UFVM_CHECK(dalloc(sink, 1));
    UFVM_CUDA(cudaMemsetAsync(flush.p, 0, n4 * sizeof(float4), c.stream));
    UFVM_CHECK(c.ensure(n));
    if (kernel == 0) UFVM_CHECK(dalloc(r, n));
    if (kernel == 1 || kernel == 3) UFVM_CHECK(build_schedule(c, L));
    if (kernel == 2) UFVM_CHECK(mcgs_prepare(c, L));
    if (kernel == 3) {
      UFVM_CHECK(ilu_factor(c, L, 0));
    }
    auto unit = [&]() -> int {
      if (kernel == 0) return residual(c, L, L.dphi.p, r.p);
      if (kernel == 1) return gs_sweep(c, L);
      if (kernel == 2) return mcgs_sweep(c, L);
      return ilu_sweep(c, L);
    };
    UFVM_CHECK(unit());
    UFVM_CUDA(cudaEventCreate(&a));
    UFVM_CUDA(cudaEventCreate(&b));
    double total = 0;
    for (int k = 0; k < reps; ++k) {
      k_flush_read<<<4 * c.nsm, 512, 0, c.stream>>>(flush.p, n4, sink.p);
      UFVM_LAUNCH_CHECK();
      UFVM_CUDA(cudaEventRecord(a, c.stream));
      UFVM_CHECK(unit());
      UFVM_CUDA(cudaEventRecord(b, c.stream));
      UFVM_CUDA(cudaEventSynchronize(b));
      float t = 0;
      UFVM_CUDA(cudaEventElapsedTime(&t, a, b));
      total += t;
    }
    if (kernel == 1 || kernel == 3) UFVM_CHECK(check_barrier(c));
    *ms_per_launch = total / reps;
    const double pass = 36.0 * n + 12.0 * nnz;  // one read of the system and x, one vector written
    double sweep = 2.0 * pass;
    if (kernel == 2 && L.ncolor > 0) {  // the backward pass skips the repeated last colour's rows
      const double last = (double)(L.h_colorStart[L.ncolor] - L.h_colorStart[L.ncolor - 1]);
      sweep -= 36.0 * last + 12.0 * nnz * (last / n);
    }
    *bytes_per_launch = kernel == 0 ? pass : kernel == 3 ? pass + 40.0 * n + 24.0 * nnz : sweep;
    return UFVM_OK;
  };
  const int st = body();
  if (a) cudaEventDestroy(a);
  if (b) cudaEventDestroy(b);
  cudaStreamSynchronize(c.stream);
  dfree(flush);
  dfree(sink);
  dfree(r);
  unborrow(L);
  c.release();
  return st;
}

int ufvm_agglomerate_level(int32_t n, const int32_t* rowptr, const int32_t* col, const double* ac, const double* anb,
                           int32_t* parents, int32_t* c_rowptr, int32_t* c_col, double* c_ac, double* c_anb,
                           int32_t* n_coarse, int32_t* nnz_coarse, void* stream) {
  if (n <= 0 || !rowptr || !col || !ac || !anb || !parents || !c_rowptr || !c_col || !c_ac || !c_anb || !n_coarse ||
      !nnz_coarse) {
    set_error("bad argument");
    return UFVM_E_INVALID;
  }
  LinCtx c;
  c.stream = (cudaStream_t)stream;
  int nnz = 0;
  UFVM_CHECK(nnz_of(n, rowptr, c.stream, &nnz));
  Level F = borrow(n, rowptr, col, ac, anb, nullptr, nullptr, nnz);
  Level C;
  AggScratch w;
  int nc = 0;
  int st = agglomerate_level(c, w, F, C, &nc);
  if (st == UFVM_OK) {
    *n_coarse = nc;
    *nnz_coarse = C.nnz;
    cudaMemcpyAsync(parents, F.parents.p, n * sizeof(int), cudaMemcpyDeviceToDevice, c.stream);
    cudaMemcpyAsync(c_rowptr, C.rowptr.p, (nc + 1) * sizeof(int), cudaMemcpyDeviceToDevice, c.stream);
    cudaMemcpyAsync(c_col, C.col.p, C.nnz * sizeof(int), cudaMemcpyDeviceToDevice, c.stream);
    cudaMemcpyAsync(c_ac, C.ac.p, nc * sizeof(double), cudaMemcpyDeviceToDevice, c.stream);
    cudaMemcpyAsync(c_anb, C.anb.p, C.nnz * sizeof(double), cudaMemcpyDeviceToDevice, c.stream);
    if (cudaStreamSynchronize(c.stream) != cudaSuccess) { set_error("copy-out failed"); st = UFVM_E_CUDA; }
  }
  F.rowptr.p = nullptr; F.col.p = nullptr; F.ac.p = nullptr; F.anb.p = nullptr;
  free_level(F);
  free_level(C);
  w.release();
  c.release();
  return st;
}

}  // extern "C"
