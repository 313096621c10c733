// mesh.cu -- mesh geometry on the GPU, restating utilities/IO/cfdProcessOpenFoamMesh.m:15-155.
//
// Bytes per face (face pass): points gathered (4 x 24 B for a quad), 7 doubles written.
// These kernels run once per case at admission; they are not on the iteration loop.
#include "case.cuh"

namespace ufvm {

// cfdProcessOpenFoamMesh.m:21-56: face centre -> triangle fan -> centroid, Sf, area.
__global__ void k_face_geometry(int F, const int* __restrict__ fstart, const int* __restrict__ fnodes,
                                const double* __restrict__ pts, double* fCx, double* fCy, double* fCz,
                                double* Sx, double* Sy, double* Sz, double* area) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= F) return;
  const int s = fstart[f], nn = fstart[f + 1] - s;
  double c0 = 0, c1 = 0, c2 = 0;
  for (int q = 0; q < nn; ++q) {
    const double* p = pts + 3 * (size_t)fnodes[s + q];
    c0 = c0 + p[0]; c1 = c1 + p[1]; c2 = c2 + p[2];
  }
  c0 = c0 / nn; c1 = c1 / nn; c2 = c2 / nn;
  double cen0 = 0, cen1 = 0, cen2 = 0, S0 = 0, S1 = 0, S2 = 0, A = 0;
  for (int t = 0; t < nn; ++t) {
    const double* p2 = pts + 3 * (size_t)fnodes[s + t];
    const double* p3 = pts + 3 * (size_t)fnodes[s + (t + 1 < nn ? t + 1 : 0)];
    const double lc0 = ((c0 + p2[0]) + p3[0]) / 3, lc1 = ((c1 + p2[1]) + p3[1]) / 3, lc2 = ((c2 + p2[2]) + p3[2]) / 3;
    const double a0 = p2[0] - c0, a1 = p2[1] - c1, a2 = p2[2] - c2;
    const double b0 = p3[0] - c0, b1 = p3[1] - c1, b2 = p3[2] - c2;
    const double l0 = 0.5 * (a1 * b2 - a2 * b1);
    const double l1 = 0.5 * (a2 * b0 - a0 * b2);
    const double l2 = 0.5 * (a0 * b1 - a1 * b0);
    const double la = sqrt(dot3(l0, l1, l2, l0, l1, l2));
    cen0 = cen0 + la * lc0; cen1 = cen1 + la * lc1; cen2 = cen2 + la * lc2;
    S0 = S0 + l0; S1 = S1 + l1; S2 = S2 + l2;
    A = A + la;
  }
  fCx[f] = cen0 / A; fCy[f] = cen1 / A; fCz[f] = cen2 / A;
  Sx[f] = S0; Sy[f] = S1; Sz[f] = S2;
  area[f] = A;
}

// cfdProcessOpenFoamMesh.m:60-104: pyramid decomposition about a rough centre. With Q5
// the rough centre sums the centroids of GLOBAL faces 0..nf-1 (local index used as a
// global face index), as the reference does.
__global__ void k_cell_geometry(int Nc, int q5, const int* __restrict__ cfStart, const int* __restrict__ cfFace,
                                const int* __restrict__ owner, const double* __restrict__ fCx,
                                const double* __restrict__ fCy, const double* __restrict__ fCz,
                                const double* __restrict__ Sx, const double* __restrict__ Sy,
                                const double* __restrict__ Sz, double* vol, double* cCx, double* cCy,
                                double* cCz) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= Nc) return;
  const int s = cfStart[e], nf = cfStart[e + 1] - s;
  double c0 = 0, c1 = 0, c2 = 0;
  for (int q = 0; q < nf; ++q) {
    const int f = q5 ? q : cfFace[s + q];
    c0 = c0 + fCx[f]; c1 = c1 + fCy[f]; c2 = c2 + fCz[f];
  }
  c0 = c0 / nf; c1 = c1 / nf; c2 = c2 / nf;
  double v0 = 0, v1 = 0, v2 = 0, sv = 0;
  for (int q = 0; q < nf; ++q) {
    const int f = cfFace[s + q];
    const double sg = owner[f] == e ? 1.0 : -1.0;
    const double S0 = Sx[f] * sg, S1 = Sy[f] * sg, S2 = Sz[f] * sg;
    const double C0 = fCx[f] - c0, C1 = fCy[f] - c1, C2 = fCz[f] - c2;
    const double lv = dot3(S0, S1, S2, C0, C1, C2) / 3;
    const double l0 = 0.75 * fCx[f] + 0.25 * c0, l1 = 0.75 * fCy[f] + 0.25 * c1, l2 = 0.75 * fCz[f] + 0.25 * c2;
    v0 = v0 + l0 * lv; v1 = v1 + l1 * lv; v2 = v2 + l2 * lv;
    sv = sv + lv;
  }
  cCx[e] = v0 / sv; cCy[e] = v1 / sv; cCz[e] = v2 / sv;
  vol[e] = sv;
}

// cfdProcessOpenFoamMesh.m:108-155: CN, eCN, gDiff, T, gf, walldist.
__global__ void k_face_geometry2(int F, int Fi, const int* __restrict__ owner, const int* __restrict__ neigh,
                                 const double* __restrict__ fCx, const double* __restrict__ fCy,
                                 const double* __restrict__ fCz, const double* __restrict__ Sx,
                                 const double* __restrict__ Sy, const double* __restrict__ Sz,
                                 const double* __restrict__ area, const double* __restrict__ cCx,
                                 const double* __restrict__ cCy, const double* __restrict__ cCz, double* CNx,
                                 double* CNy, double* CNz, double* eCx, double* eCy, double* eCz, double* gDiff,
                                 double* Tx, double* Ty, double* Tz, double* gf, double* wd) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= F) return;
  const double A = area[f];
  const int o = owner[f];
  const double S0 = Sx[f], S1 = Sy[f], S2 = Sz[f];
  if (f < Fi) {
    const int n = neigh[f];
    const double n0 = S0 / A, n1 = S1 / A, n2 = S2 / A;
    const double C0 = cCx[n] - cCx[o], C1 = cCy[n] - cCy[o], C2 = cCz[n] - cCz[o];
    const double mcn = sqrt(dot3(C0, C1, C2, C0, C1, C2));
    const double e0 = C0 / mcn, e1 = C1 / mcn, e2 = C2 / mcn;
    const double E0 = A * e0, E1 = A * e1, E2 = A * e2;
    gDiff[f] = sqrt(dot3(E0, E1, E2, E0, E1, E2)) / sqrt(dot3(C0, C1, C2, C0, C1, C2));
    CNx[f] = C0; CNy[f] = C1; CNz[f] = C2;
    eCx[f] = e0; eCy[f] = e1; eCz[f] = e2;
    Tx[f] = S0 - E0; Ty[f] = S1 - E1; Tz[f] = S2 - E2;
    const double cf0 = fCx[f] - cCx[o], cf1 = fCy[f] - cCy[o], cf2 = fCz[f] - cCz[o];
    const double ff0 = cCx[n] - fCx[f], ff1 = cCy[n] - fCy[f], ff2 = cCz[n] - fCz[f];
    gf[f] = dot3(cf0, cf1, cf2, n0, n1, n2) / (dot3(cf0, cf1, cf2, n0, n1, n2) + dot3(ff0, ff1, ff2, n0, n1, n2));
    wd[f] = 0;
  } else {
    const double C0 = fCx[f] - cCx[o], C1 = fCy[f] - cCy[o], C2 = fCz[f] - cCz[o];
    gDiff[f] = (A * A) / dot3(C0, C1, C2, S0, S1, S2);
    const double mcn = sqrt(dot3(C0, C1, C2, C0, C1, C2));
    const double e0 = C0 / mcn, e1 = C1 / mcn, e2 = C2 / mcn;
    const double E0 = A * e0, E1 = A * e1, E2 = A * e2;
    CNx[f] = C0; CNy[f] = C1; CNz[f] = C2;
    eCx[f] = e0; eCy[f] = e1; eCz[f] = e2;
    Tx[f] = S0 - E0; Ty[f] = S1 - E1; Tz[f] = S2 - E2;
    gf[f] = 1;
    wd[f] = dot3(C0, C1, C2, S0, S1, S2) / sqrt(dot3(S0, S1, S2, S0, S1, S2));
  }
}

// Sum over a noSlip patch of n_c^2 for c = 0..2, sequential in face order (the value
// MATLAB's dot() of two row vectors returns, cfdAssembleDiffusionTerm.m:535,541,547). One block
// per patch: the block stages a chunk of the patch's faces through shared memory with coalesced
// loads and forms the squares in parallel; threads 0..2 then add one component each in face
// order, so each sum is the same chain of additions as the sequential loop.
constexpr int kNsumChunk = 256;
__global__ void __launch_bounds__(kNsumChunk) k_patch_nsum(const int* __restrict__ pstart, const int* __restrict__ pn,
                                                           const double* __restrict__ Sx, const double* __restrict__ Sy,
                                                           const double* __restrict__ Sz,
                                                           const double* __restrict__ area, double* out) {
  __shared__ double sq[3][kNsumChunk];
  const int p = blockIdx.x, t = threadIdx.x;
  const int n = pn[p], f0 = pstart[p];
  double s = 0;
  for (int base = 0; base < n; base += kNsumChunk) {
    const int j = base + t;
    if (j < n) {
      const int f = f0 + j;
      const double A = area[f];
      const double n0 = Sx[f] / A, n1 = Sy[f] / A, n2 = Sz[f] / A;
      sq[0][t] = n0 * n0; sq[1][t] = n1 * n1; sq[2][t] = n2 * n2;
    }
    __syncthreads();
    if (t < 3) {
      const int cnt = min(kNsumChunk, n - base);
      for (int k = 0; k < cnt; ++k) s = s + sq[t][k];
    }
    __syncthreads();
  }
  if (t < 3) out[3 * p + t] = s;
}

int Case::build_mesh(const ufvm_mesh_desc* d) {
  const int F = d->n_faces, Fi = d->n_interior;
  int nc = 0;
  for (int f = 0; f < F; ++f) nc = std::max(nc, d->owner[f] + 1);
  for (int f = 0; f < Fi; ++f) nc = std::max(nc, d->neighbour[f] + 1);
  if (F <= 0 || Fi < 0 || Fi > F || nc <= 0) {
    set_error("invalid mesh sizes");
    return UFVM_E_INVALID;
  }
  M.Nc = nc; M.F = F; M.Fi = Fi; M.Fb = F - Fi;
  // host connectivity (cfdReadPolyMesh.m:153-181, cfdProcessOpenFoamMesh.m:158-172)
  std::vector<int> cnt(nc, 0), icnt(nc, 0);
  for (int f = 0; f < Fi; ++f) { cnt[d->owner[f]]++; cnt[d->neighbour[f]]++; icnt[d->owner[f]]++; icnt[d->neighbour[f]]++; }
  for (int f = Fi; f < F; ++f) cnt[d->owner[f]]++;
  h_cfStart.assign(nc + 1, 0);
  h_rowptr.assign(nc + 1, 0);
  for (int e = 0; e < nc; ++e) { h_cfStart[e + 1] = h_cfStart[e] + cnt[e]; h_rowptr[e + 1] = h_rowptr[e] + icnt[e]; }
  M.nnz = h_rowptr[nc];
  h_cfFace.assign(h_cfStart[nc], 0);
  h_col.assign(M.nnz, 0);
  std::vector<int> cur(h_cfStart.begin(), h_cfStart.end() - 1), curr(h_rowptr.begin(), h_rowptr.end() - 1);
  h_ownSlot.assign(Fi, 0); h_neiSlot.assign(Fi, 0);
  for (int f = 0; f < Fi; ++f) {
    const int o = d->owner[f], n = d->neighbour[f];
    h_cfFace[cur[o]++] = f; h_ownSlot[f] = curr[o]; h_col[curr[o]++] = n;
    h_cfFace[cur[n]++] = f; h_neiSlot[f] = curr[n]; h_col[curr[n]++] = o;
  }
  for (int f = Fi; f < F; ++f) h_cfFace[cur[d->owner[f]]++] = f;
  // patches
  P.n = d->n_patches;
  P.type.assign(d->patch_type, d->patch_type + P.n);
  P.start.assign(d->patch_start, d->patch_start + P.n);
  P.count.assign(d->patch_n, d->patch_n + P.n);
  std::vector<int> bpatch(M.Fb, -1);
  for (int p = 0; p < P.n; ++p) {
    if (P.start[p] < Fi || P.start[p] + P.count[p] > F) { set_error("patch outside boundary faces"); return UFVM_E_INVALID; }
    for (int j = 0; j < P.count[p]; ++j) bpatch[P.start[p] + j - Fi] = p;
  }
  for (int k = 0; k < M.Fb; ++k)
    if (bpatch[k] < 0) { set_error("boundary face not covered by a patch"); return UFVM_E_INVALID; }
  // upload topology
  UFVM_CHECK(up(M.owner, d->owner, F));
  UFVM_CHECK(up(M.neigh, d->neighbour, std::max(Fi, 1)));
  UFVM_CHECK(up(M.cfStart, h_cfStart.data(), nc + 1));
  UFVM_CHECK(up(M.cfFace, h_cfFace.data(), h_cfFace.size()));
  UFVM_CHECK(up(M.rowptr, h_rowptr.data(), nc + 1));
  UFVM_CHECK(up(M.col, h_col.data(), std::max(M.nnz, 1)));
  UFVM_CHECK(up(M.ownSlot, h_ownSlot.data(), std::max(Fi, 1)));
  UFVM_CHECK(up(M.neiSlot, h_neiSlot.data(), std::max(Fi, 1)));
  UFVM_CHECK(up(M.bPatch, bpatch.data(), std::max(M.Fb, 1)));
  UFVM_CHECK(up(D.ptype, P.type.data(), P.n));
  UFVM_CHECK(up(D.pstart, P.start.data(), P.n));
  UFVM_CHECK(up(D.pcount, P.count.data(), P.n));
  // geometry
  DArr<double> pts;
  DArr<int> fstart, fnodes;
  UFVM_CHECK(up(pts, d->points, 3 * (size_t)d->n_points));
  UFVM_CHECK(up(fstart, d->face_start, F + 1));
  UFVM_CHECK(up(fnodes, d->face_nodes, d->face_start[F]));
  for (auto* a : {&M.fCx, &M.fCy, &M.fCz, &M.Sx, &M.Sy, &M.Sz, &M.area, &M.CNx, &M.CNy, &M.CNz, &M.eCx, &M.eCy,
                  &M.eCz, &M.gDiff, &M.Tx, &M.Ty, &M.Tz, &M.gf, &M.wd})
    UFVM_CHECK(dalloc(*a, F));
  for (auto* a : {&M.vol, &M.cCx, &M.cCy, &M.cCz}) UFVM_CHECK(dalloc(*a, nc));
  k_face_geometry<<<nblocks(F), kBlock, 0, stream>>>(F, fstart.p, fnodes.p, pts.p, M.fCx.p, M.fCy.p, M.fCz.p, M.Sx.p,
                                                     M.Sy.p, M.Sz.p, M.area.p);
  UFVM_LAUNCH_CHECK();
  k_cell_geometry<<<nblocks(nc), kBlock, 0, stream>>>(nc, (S.quirks & UFVM_Q5_ROUGH_CENTRE) ? 1 : 0, M.cfStart.p,
                                                      M.cfFace.p, M.owner.p, M.fCx.p, M.fCy.p, M.fCz.p, M.Sx.p,
                                                      M.Sy.p, M.Sz.p, M.vol.p, M.cCx.p, M.cCy.p, M.cCz.p);
  UFVM_LAUNCH_CHECK();
  k_face_geometry2<<<nblocks(F), kBlock, 0, stream>>>(F, Fi, M.owner.p, M.neigh.p, M.fCx.p, M.fCy.p, M.fCz.p, M.Sx.p,
                                                      M.Sy.p, M.Sz.p, M.area.p, M.cCx.p, M.cCy.p, M.cCz.p, M.CNx.p,
                                                      M.CNy.p, M.CNz.p, M.eCx.p, M.eCy.p, M.eCz.p, M.gDiff.p,
                                                      M.Tx.p, M.Ty.p, M.Tz.p, M.gf.p, M.wd.p);
  UFVM_LAUNCH_CHECK();
  UFVM_CHECK(dalloc(D.pnsum, 3 * std::max(P.n, 1)));
  if ((S.quirks & UFVM_Q14_NOSLIP_PATCH_SUM) && P.n > 0) {  // only the reference's patch-wide sum reads it
    k_patch_nsum<<<P.n, kNsumChunk, 0, stream>>>(D.pstart.p, D.pcount.p, M.Sx.p, M.Sy.p, M.Sz.p, M.area.p, D.pnsum.p);
    UFVM_LAUNCH_CHECK();
  } else {
    UFVM_CUDA(cudaMemsetAsync(D.pnsum.p, 0, 3 * std::max(P.n, 1) * sizeof(double), stream));
  }
  UFVM_CUDA(cudaStreamSynchronize(stream));
  dfree(pts); dfree(fstart); dfree(fnodes);
  return UFVM_OK;
}

}  // namespace ufvm
