// simple.cu -- per-iteration SIMPLE stages on the GPU, batched over cases.
//
// Every stage kernel runs over a work list of (slot, block) pairs and reads the case it
// works on from a descriptor table, so one launch advances every resident case; a single
// case is a one-entry table. Every cell-centric kernel visits a cell's faces in the cell's
// iFaces order (interior faces in face order, then boundary faces in face order;
// cfdReadPolyMesh.m:153-181). That is exactly the order in which the reference's face-loop
// scatter (assemble/cfdAssembleIntoGlobalMatrixFaceFluxes.m:25-55) and Gauss-gradient loop
// (compute/cfdComputeGradientGauss0.m:47-63) add contributions into a given cell, so the
// gathers reproduce the sequential sums without atomics. Per-face fluxes are recomputed on
// both sides of an interior face with identical code (identical bits).
//
// Algorithmic bytes (FP64 values, int32 indices) per cell of the momentum assembly (one
// component): cells 8 phi + 72 grad + 24 (ac, bc, DU) + 8 vol; faces (read from both
// sides) 8 mdot + 8 gf + 8 gDiff + 24 T + 24 S + 24 CN + 8 idx.
#include "amg.cuh"
#include "simple.cuh"

namespace ufvm {

MeshView Case::mv() const {
  MeshView v;
  v.Nc = M.Nc; v.F = M.F; v.Fi = M.Fi; v.Fb = M.Fb; v.nnz = M.nnz;
  v.owner = M.owner.p; v.neigh = M.neigh.p; v.cfStart = M.cfStart.p; v.cfFace = M.cfFace.p;
  v.rowptr = M.rowptr.p; v.col = M.col.p; v.bPatch = M.bPatch.p;
  v.Sx = M.Sx.p; v.Sy = M.Sy.p; v.Sz = M.Sz.p; v.area = M.area.p; v.CNx = M.CNx.p; v.CNy = M.CNy.p; v.CNz = M.CNz.p;
  v.eCx = M.eCx.p; v.eCy = M.eCy.p; v.eCz = M.eCz.p; v.gDiff = M.gDiff.p; v.Tx = M.Tx.p; v.Ty = M.Ty.p; v.Tz = M.Tz.p;
  v.gf = M.gf.p; v.wd = M.wd.p; v.vol = M.vol.p;
  v.ptype = D.ptype.p; v.pstart = D.pstart.p; v.pcount = D.pcount.p; v.bcU = D.bcU.p; v.bcP = D.bcP.p;
  v.pnsum = D.pnsum.p;
  return v;
}

FieldView Case::fv() {
  FieldView v;
  v.rowsU = rowsU;
  v.U0 = U[0].p; v.U1 = U[1].p; v.U2 = U[2].p;
  for (int k = 0; k < 9; ++k) v.gU[k] = gU[k].p;
  v.p = p.p; v.gp0 = gp[0].p; v.gp1 = gp[1].p; v.gp2 = gp[2].p;
  v.PP = PP.p; v.gPP0 = gPP[0].p; v.gPP1 = gPP[1].p; v.gPP2 = gPP[2].p;
  v.DU0 = DU[0].p; v.DU1 = DU[1].p; v.DU2 = DU[2].p;
  v.mdot = mdot.p; v.fC1 = fC1.p; v.fC2 = fC2.p;
  v.vU0 = vU[0].p; v.vU1 = vU[1].p; v.vU2 = vU[2].p; v.vP = vP.p;
  v.tmp3 = tmp3.p;
  v.uft = uft.p;
  return v;
}

SlotDesc Case::desc() {
  SlotDesc d;
  d.m = mv();
  d.f = fv();
  d.nu = S.nu; d.urf_u = S.urf_u; d.urf_p = S.urf_p; d.fdt = S.false_dt;
  d.quirks = S.quirks; d.fixed = S.fixed_element; d.rowsU = rowsU; d.pad = 0;
  Level& L = lev[0];
  d.ac = L.ac.p; d.bc = L.bc.p; d.anb = L.anb.p; d.dphi = L.dphi.p;
  d.scal = scal.p;
  d.flags = flags.p;
  return d;
}

static int make_work(DArr<int2>& w, int& cnt, int n, cudaStream_t st) {
  const int nb = std::max(nblocks(n), 1);
  std::vector<int2> h(nb);
  for (int b = 0; b < nb; ++b) h[b] = make_int2(0, b);
  UFVM_CHECK(dalloc(w, nb));
  UFVM_CUDA(cudaMemcpyAsync(w.p, h.data(), nb * sizeof(int2), cudaMemcpyHostToDevice, st));
  cnt = nb;
  return UFVM_OK;
}

// (re)upload this case's one-entry slot table and work lists
int Case::sync_slot() {
  UFVM_CHECK(dalloc(scal, SCAL_N * 4));
  UFVM_CHECK(dalloc(flags, FLAG_N));
  SlotDesc d = desc();
  UFVM_CHECK(dalloc(slot, 1));
  UFVM_CUDA(cudaMemcpyAsync(slot.p, &d, sizeof(SlotDesc), cudaMemcpyHostToDevice, stream));
  if (!wl.cells.p) {
    UFVM_CHECK(make_work(wl.cells, wl.ncells, M.Nc, stream));
    UFVM_CHECK(make_work(wl.faces, wl.nfaces, M.F, stream));
    UFVM_CHECK(make_work(wl.bfaces, wl.nbfaces, M.Fb, stream));
    int z = 0, e = wl.ncells;
    UFVM_CHECK(up(wl.cstart, &z, 1));
    UFVM_CHECK(up(wl.cend, &e, 1));
    UFVM_CHECK(up(wl.ustart, &z, 1));
  }
  if (wl.urows_for != rowsU) {
    UFVM_CHECK(make_work(wl.urows, wl.nurows, rowsU, stream));
    UFVM_CHECK(up(wl.uend, &wl.nurows, 1));
    wl.urows_for = rowsU;
  }
  UFVM_CHECK(dalloc(part, 2 * (size_t)std::max(wl.ncells, wl.nurows) + 8));
  return UFVM_OK;
}

// ================================================================ host orchestration (single case)
int Case::update_fields() {
  UFVM_CHECK(sync_slot());
  UFVM_CHECK(stage_update_fields(batch()));
  double sc = 0;
  UFVM_CUDA(cudaMemcpyAsync(&sc, scal.p + SCAL_SCALE, sizeof(double), cudaMemcpyDeviceToHost, stream));
  UFVM_CUDA(cudaStreamSynchronize(stream));
  scaleU = sc;
  return UFVM_OK;
}

BatchLaunch Case::batch() {
  return BatchLaunch{slot.p, wl.cells.p, wl.ncells, wl.faces.p, wl.nfaces, wl.bfaces.p, wl.nbfaces, wl.urows.p,
                     wl.nurows, wl.cstart.p, wl.cend.p, wl.ustart.p, wl.uend.p, 1, part.p, stream};
}

int Case::fresh_level0() {
  if (lev.empty()) lev.resize(1);
  Level& L = lev[0];
  if (!L.rowptr.p) {
    L.n = M.Nc; L.nnz = M.nnz;
    L.rowptr = M.rowptr;  // shared with the mesh (freed with the mesh)
    L.col = M.col;
    UFVM_CHECK(dalloc(L.ac, M.Nc));
    UFVM_CHECK(dalloc(L.bc, M.Nc));
    UFVM_CHECK(dalloc(L.anb, std::max(M.nnz, 1)));
    UFVM_CHECK(dalloc(L.dphi, M.Nc));
  }
  UFVM_CUDA(cudaMemsetAsync(L.dphi.p, 0, M.Nc * sizeof(double), stream));
  return UFVM_OK;
}

int Case::assemble_u(int comp, double* rms, double* mx) {
  UFVM_CHECK(fresh_level0());
  UFVM_CHECK(sync_slot());
  UFVM_CUDA(cudaMemsetAsync(flags.p, 0, FLAG_N * sizeof(int), stream));
  BatchLaunch b = batch();
  UFVM_CHECK(stage_assemble_u(b, comp));
  double out[2];
  int zd = 0;
  UFVM_CUDA(cudaMemcpyAsync(out, scal.p + SCAL_RMS, 2 * sizeof(double), cudaMemcpyDeviceToHost, stream));
  UFVM_CUDA(cudaMemcpyAsync(&zd, flags.p + FLAG_ZERO_DIAG, sizeof(int), cudaMemcpyDeviceToHost, stream));
  UFVM_CUDA(cudaStreamSynchronize(stream));
  if (zd) { set_error("****** Divide by Zero ******* (ac == 0 in U equation)"); return UFVM_E_ZERO_DIAG; }
  *rms = out[0];
  *mx = out[1];
  return UFVM_OK;
}

int Case::assemble_p(double* rms, double* mx) {
  UFVM_CHECK(fresh_level0());
  UFVM_CHECK(sync_slot());
  UFVM_CUDA(cudaMemsetAsync(flags.p, 0, FLAG_N * sizeof(int), stream));
  BatchLaunch b = batch();
  UFVM_CHECK(stage_assemble_p(b));
  double out[2];
  int bad = 0;
  UFVM_CUDA(cudaMemcpyAsync(out, scal.p + SCAL_RMS, 2 * sizeof(double), cudaMemcpyDeviceToHost, stream));
  UFVM_CUDA(cudaMemcpyAsync(&bad, flags.p + FLAG_BAD_BC, sizeof(int), cudaMemcpyDeviceToHost, stream));
  UFVM_CUDA(cudaStreamSynchronize(stream));
  if (bad) { set_error("p boundary condition not implemented for this patch type"); return UFVM_E_BC_UNSUPPORTED; }
  *rms = out[0];
  *mx = out[1];
  return UFVM_OK;
}

int Case::correct_u(int comp) {
  UFVM_CHECK(sync_slot());
  BatchLaunch b = batch();
  return stage_correct_u(b, comp);
}

int Case::correct_p() {
  UFVM_CHECK(sync_slot());
  BatchLaunch b = batch();
  const int q12 = (S.quirks & UFVM_Q12_OUTLET_U_FACE_ROWS) ? 1 : 0;
  UFVM_CHECK(stage_correct_p(b, P.n, tmp3.p));
  // rows written by an outlet with fixed p (face-indexed rows under Q12)
  for (int ip = 0; ip < P.n; ++ip)
    if (P.type[ip] == UFVM_PATCH_OUTLET && P.bcP[ip] == UFVM_BC_FIXED_VALUE && P.count[ip] > 0) {
      const int row0 = q12 ? P.start[ip] : M.Nc + P.start[ip] - M.Fi;
      rowsU = std::max(rowsU, row0 + P.count[ip]);
    }
  return UFVM_OK;
}

int Case::init_fields(const int32_t* bcu, const int32_t* bcp, const double* vu, const double* vp, const double* U0h,
                      const double* p0h, const double* mdot0h) {
  const int Nc = M.Nc, Fb = M.Fb, F = M.F;
  P.bcU.assign(bcu, bcu + P.n);
  P.bcP.assign(bcp, bcp + P.n);
  UFVM_CHECK(up(D.bcU, bcu, P.n));
  UFVM_CHECK(up(D.bcP, bcp, P.n));
  // U rows: Nc + Fb, plus the face-indexed rows an outlet with fixed p writes under Q12
  rowsU = Nc + Fb;
  rowsUcap = rowsU;
  for (int ip = 0; ip < P.n; ++ip) {
    if (P.type[ip] == UFVM_PATCH_OUTLET && bcp[ip] == UFVM_BC_FIXED_VALUE && (S.quirks & UFVM_Q12_OUTLET_U_FACE_ROWS)) {
      if (P.start[ip] < Nc) { set_error("outlet face rows overlap interior cells"); return UFVM_E_BC_UNSUPPORTED; }
      rowsUcap = std::max(rowsUcap, P.start[ip] + P.count[ip]);
    }
  }
  std::vector<double> h(rowsUcap, 0.0), hv(std::max(Fb, 1));
  for (int c = 0; c < 3; ++c) {
    std::fill(h.begin(), h.end(), 0.0);
    if (U0h) for (int e = 0; e < Nc; ++e) h[e] = U0h[3 * (size_t)e + c];
    UFVM_CHECK(up(U[c], h.data(), rowsUcap));
    for (int k = 0; k < Fb; ++k) hv[k] = vu[3 * (size_t)k + c];
    UFVM_CHECK(up(vU[c], hv.data(), Fb));
  }
  std::fill(h.begin(), h.end(), 0.0);
  if (p0h) for (int e = 0; e < Nc; ++e) h[e] = p0h[e];
  UFVM_CHECK(up(p, h.data(), Nc + Fb));
  UFVM_CHECK(up(vP, vp, Fb));
  const size_t R = Nc + Fb;
  for (int k = 0; k < 9; ++k) UFVM_CHECK(dalloc(gU[k], R));
  for (int d = 0; d < 3; ++d) { UFVM_CHECK(dalloc(gp[d], R)); UFVM_CHECK(dalloc(gPP[d], R)); }
  UFVM_CHECK(dalloc(PP, R));
  UFVM_CUDA(cudaMemsetAsync(PP.p, 0, R * sizeof(double), stream));
  for (int d = 0; d < 3; ++d) UFVM_CUDA(cudaMemsetAsync(gPP[d].p, 0, R * sizeof(double), stream));
  for (int c = 0; c < 3; ++c) {
    UFVM_CHECK(dalloc(DU[c], R));
    UFVM_CUDA(cudaMemsetAsync(DU[c].p, 0, R * sizeof(double), stream));
  }
  UFVM_CHECK(dalloc(mdot, F));
  UFVM_CHECK(dalloc(uft, 3 * 7 * (size_t)F));  // [comp][term][face]
  UFVM_CHECK(dalloc(fC1, F));
  UFVM_CHECK(dalloc(fC2, F));
  UFVM_CUDA(cudaMemsetAsync(fC1.p, 0, F * sizeof(double), stream));
  UFVM_CUDA(cudaMemsetAsync(fC2.p, 0, F * sizeof(double), stream));
  UFVM_CHECK(dalloc(tmp3, 3 * (size_t)std::max(Fb, 1)));
  UFVM_CHECK(fresh_level0());
  UFVM_CHECK(sync_slot());
  if (mdot0h) UFVM_CUDA(cudaMemcpyAsync(mdot.p, mdot0h, F * sizeof(double), cudaMemcpyHostToDevice, stream));
  BatchLaunch b = batch();
  UFVM_CHECK(stage_init(b, mdot0h == nullptr));
  UFVM_CUDA(cudaStreamSynchronize(stream));
  return UFVM_OK;
}

}  // namespace ufvm
