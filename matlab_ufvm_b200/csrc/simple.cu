// simple.cu -- per-iteration SIMPLE stages on the GPU.
//
// Every cell-centric kernel visits a cell's faces in the cell's iFaces order (interior
// faces in face order, then boundary faces in face order; cfdReadPolyMesh.m:153-181). That
// is exactly the order in which the reference's face-loop scatter
// (assemble/cfdAssembleIntoGlobalMatrixFaceFluxes.m:25-55) and Gauss-gradient loop
// (compute/cfdComputeGradientGauss0.m:47-63) add contributions into a given cell, so the
// gathers below reproduce the sequential sums without atomics. Per-face fluxes are
// recomputed on both sides of an interior face with identical code (identical bits).
//
// Algorithmic bytes (FP64 values, int32 indices) per cell-iteration of the momentum
// assembly (one component): cells 8 phi + 72 grad + 24 (ac, bc, DU) + 8 vol;
// faces (x2 sides) 8 mdot + 8 gf + 8 gDiff + 24 T + 24 S + 24 CN + 8 idx.
#include "amg.cuh"

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
  return v;
}

__device__ __forceinline__ double* Uc(const FieldView& f, int c) { return c == 0 ? f.U0 : (c == 1 ? f.U1 : f.U2); }
__device__ __forceinline__ double* DUc(const FieldView& f, int c) { return c == 0 ? f.DU0 : (c == 1 ? f.DU1 : f.DU2); }
__device__ __forceinline__ double* gpd(const FieldView& f, int d) { return d == 0 ? f.gp0 : (d == 1 ? f.gp1 : f.gp2); }
__device__ __forceinline__ double* gPPd(const FieldView& f, int d) { return d == 0 ? f.gPP0 : (d == 1 ? f.gPP1 : f.gPP2); }
__device__ __forceinline__ const double* vUc(const FieldView& f, int c) { return c == 0 ? f.vU0 : (c == 1 ? f.vU1 : f.vU2); }

// ---------------------------------------------------------------- boundary conditions
// update/cfdUpdateBoundaryConditions.m:13-96 (per-iteration: fixed values only)
__global__ void k_bc_update(MeshView m, FieldView f) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m.Fb) return;
  const int p = m.bPatch[k], ty = m.ptype[p], tu = m.bcU[p], tp = m.bcP[p];
  const int b = m.Nc + k;
  if ((ty == UFVM_PATCH_WALL && (tu == UFVM_BC_FIXED_VALUE || tu == UFVM_BC_NOSLIP)) ||
      ((ty == UFVM_PATCH_INLET || ty == UFVM_PATCH_OUTLET) && tu == UFVM_BC_FIXED_VALUE)) {
    f.U0[b] = f.vU0[k]; f.U1[b] = f.vU1[k]; f.U2[b] = f.vU2[k];
  }
  if (tp == UFVM_BC_FIXED_VALUE && (ty == UFVM_PATCH_WALL || ty == UFVM_PATCH_INLET || ty == UFVM_PATCH_OUTLET))
    f.p[b] = f.vP[k];
}

__device__ __forceinline__ void tangential(const MeshView& m, FieldView& f, int fc, int b, int o, int c0, int c1) {
  const double S0 = m.Sx[fc], S1 = m.Sy[fc], S2 = m.Sz[fc];
  const double nS = sqrt(dot3(S0, S1, S2, S0, S1, S2));
  const double n0 = S0 / nS, n1 = S1 / nS, n2 = S2 / nS;
  const double un = dot3(f.U0[o], f.U1[o], f.U2[o], n0, n1, n2);
  for (int c = c0; c <= c1; ++c) {
    const double nc = c == 0 ? n0 : (c == 1 ? n1 : n2);
    Uc(f, c)[b] = Uc(f, c)[o] - un * nc;
  }
}

// initialize/cfdInitializeBoundaryConditions.m (initial boundary values)
__global__ void k_bc_init(MeshView m, FieldView f) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m.Fb) return;
  const int fc = m.Fi + k, p = m.bPatch[k], ty = m.ptype[p], tu = m.bcU[p], tp = m.bcP[p];
  const int b = m.Nc + k, o = m.owner[fc];
  if (tu == UFVM_BC_FIXED_VALUE || tu == UFVM_BC_NOSLIP) {
    f.U0[b] = f.vU0[k]; f.U1[b] = f.vU1[k]; f.U2[b] = f.vU2[k];
  } else if (tu == UFVM_BC_ZERO_GRADIENT) {
    if (ty == UFVM_PATCH_INLET) f.U0[b] = f.U0[o];  // linear index: first component only
    else { f.U0[b] = f.U0[o]; f.U1[b] = f.U1[o]; f.U2[b] = f.U2[o]; }
  } else {
    tangential(m, f, fc, b, o, 0, 2);
  }
  f.p[b] = tp == UFVM_BC_FIXED_VALUE ? f.vP[k] : f.p[o];
}

// initialize/cfdInitializeMdotField.m:72-86 (rho = ones over faces, 'Average')
__global__ void k_mdot_init(MeshView m, FieldView f) {
  const int fc = blockIdx.x * blockDim.x + threadIdx.x;
  if (fc >= m.F) return;
  double u0, u1, u2, rf;
  if (fc < m.Fi) {
    const int o = m.owner[fc], n = m.neigh[fc];
    const double w = m.gf[fc];
    u0 = w * f.U0[n] + (1 - w) * f.U0[o];
    u1 = w * f.U1[n] + (1 - w) * f.U1[o];
    u2 = w * f.U2[n] + (1 - w) * f.U2[o];
    rf = w * 1.0 + (1 - w) * 1.0;
  } else {
    const int b = m.Nc + fc - m.Fi;
    u0 = f.U0[b]; u1 = f.U1[b]; u2 = f.U2[b];
    rf = 1.0;
  }
  f.mdot[fc] = rf * dot3(m.Sx[fc], m.Sy[fc], m.Sz[fc], u0, u1, u2);
}

// ---------------------------------------------------------------- Gauss gradient
struct GradArgs {
  const double* phi[3];
  double* g[9];  // g[c * 3 + d]
};

template <int NC>
__global__ void k_grad_cells(MeshView m, GradArgs a, int q1) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= m.Nc) return;
  double g[NC][3];
#pragma unroll
  for (int c = 0; c < NC; ++c) g[c][0] = g[c][1] = g[c][2] = 0.0;
  const int s = m.cfStart[e], ne = m.cfStart[e + 1];
  for (int q = s; q < ne; ++q) {
    const int fc = m.cfFace[q];
    const double S0 = m.Sx[fc], S1 = m.Sy[fc], S2 = m.Sz[fc];
    if (fc < m.Fi) {
      const int o = m.owner[fc], n = m.neigh[fc];
      const double w = m.gf[fc];
      const bool own = o == e;
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const double phf = w * a.phi[c][n] + (1 - w) * a.phi[c][o];
        if (own) { g[c][0] = g[c][0] + phf * S0; g[c][1] = g[c][1] + phf * S1; g[c][2] = g[c][2] + phf * S2; }
        else { g[c][0] = g[c][0] - phf * S0; g[c][1] = g[c][1] - phf * S1; g[c][2] = g[c][2] - phf * S2; }
      }
    } else {
      const int b = m.Nc + fc - m.Fi;
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const double pb = a.phi[q1 ? 0 : c][b];
        g[c][0] = g[c][0] + pb * S0; g[c][1] = g[c][1] + pb * S1; g[c][2] = g[c][2] + pb * S2;
      }
    }
  }
  const double v = m.vol[e];
#pragma unroll
  for (int c = 0; c < NC; ++c)
#pragma unroll
    for (int d = 0; d < 3; ++d) a.g[c * 3 + d][e] = g[c][d] / v;
}

// boundary rows: owner copy, then the wall / inlet / outlet correction (cfdUpdateGradient.m:81-255)
template <int NC>
__global__ void k_grad_bfix(MeshView m, GradArgs a, int q1) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m.Fb) return;
  const int fc = m.Fi + k, o = m.owner[fc], b = m.Nc + k;
  const int ty = m.ptype[m.bPatch[k]];
  const bool fix = ty == UFVM_PATCH_WALL || ty == UFVM_PATCH_INLET || ty == UFVM_PATCH_OUTLET;
  const double d0 = m.CNx[fc], d1 = m.CNy[fc], d2 = m.CNz[fc];
  const double dmag = sqrt(dot3(d0, d1, d2, d0, d1, d2));
  const double e0 = d0 / dmag, e1 = d1 / dmag, e2 = d2 / dmag;
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    const double g0 = a.g[c * 3][o], g1 = a.g[c * 3 + 1][o], g2 = a.g[c * 3 + 2][o];
    if (!fix) {
      a.g[c * 3][b] = g0; a.g[c * 3 + 1][b] = g1; a.g[c * 3 + 2][b] = g2;
      continue;
    }
    const int pc = (q1 && ty != UFVM_PATCH_WALL) ? 0 : c;
    const double ge = dot3(g0, g1, g2, e0, e1, e2);
    const double sn = (a.phi[pc][b] - a.phi[pc][o]) / dmag;
    a.g[c * 3][b] = (g0 - ge * e0) + sn * e0;
    a.g[c * 3 + 1][b] = (g1 - ge * e1) + sn * e1;
    a.g[c * 3 + 2][b] = (g2 - ge * e2) + sn * e2;
  }
}

int Case::gradient(double* const* phi, int ncomp, double* const* grad, bool vector_field) {
  GradArgs a;
  for (int c = 0; c < 3; ++c) a.phi[c] = c < ncomp ? phi[c] : nullptr;
  for (int k = 0; k < 9; ++k) a.g[k] = k < 3 * ncomp ? grad[k] : nullptr;
  const int q1 = (vector_field && (S.quirks & UFVM_Q1_VEC_BOUNDARY_COMPONENT)) ? 1 : 0;
  const MeshView m = mv();
  if (ncomp == 3) {
    k_grad_cells<3><<<nblocks(M.Nc), kBlock, 0, stream>>>(m, a, q1);
    k_grad_bfix<3><<<nblocks(M.Fb), kBlock, 0, stream>>>(m, a, q1);
  } else {
    k_grad_cells<1><<<nblocks(M.Nc), kBlock, 0, stream>>>(m, a, 0);
    k_grad_bfix<1><<<nblocks(M.Fb), kBlock, 0, stream>>>(m, a, 0);
  }
  UFVM_LAUNCH_CHECK();
  return UFVM_OK;
}

// ---------------------------------------------------------------- scale (cfdUpdateScale.m:15-28)
__global__ void k_minmax(int rows, const double* __restrict__ a0, const double* __restrict__ a1,
                         const double* __restrict__ a2, double* part) {
  __shared__ double sh[32];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double mx = -INFINITY, mn = INFINITY;
  if (i < rows) {
    mx = dmax(dmax(a0[i], a1[i]), a2[i]);
    mn = dmin(dmin(a0[i], a1[i]), a2[i]);
  }
  mx = block_reduce<1>(mx, sh);
  if (threadIdx.x == 0) part[2 * blockIdx.x] = mx;
  mn = block_reduce<2>(mn, sh);
  if (threadIdx.x == 0) part[2 * blockIdx.x + 1] = mn;
}

// stage 2 for (sum, max) / (max, min) pairs; OP2 chooses the second reduction
template <int OP1, int OP2>
__global__ void k_final2(int np, const double* __restrict__ part, double* out) {
  __shared__ double sh[32];
  double a = OP1 == 0 ? 0.0 : -INFINITY, b = OP2 == 1 ? -INFINITY : INFINITY;
  for (int k = threadIdx.x; k < np; k += blockDim.x) {
    a = OP1 == 0 ? a + part[2 * k] : dmax(a, part[2 * k]);
    b = OP2 == 1 ? dmax(b, part[2 * k + 1]) : dmin(b, part[2 * k + 1]);
  }
  a = block_reduce<OP1>(a, sh);
  if (threadIdx.x == 0) out[0] = a;
  b = block_reduce<OP2>(b, sh);
  if (threadIdx.x == 0) out[1] = b;
}

// ---------------------------------------------------------------- momentum assembly
struct AsmArgs {
  int comp, quirks;
  double nu, urf, fdt, scale;
  double *ac, *bc, *anb, *DUout, *part;
  int* zero_diag;
};

// Average:Corrected face gradient of the scalar column ph with gradient g[0..2]
// (interpolate/cfdInterpolateGradientsFromElementsToInteriorFaces.m:23-70; Q4 weights).
__device__ __forceinline__ void face_grad_corr(const MeshView& m, int fc, int o, int n, const double* g0,
                                               const double* g1, const double* g2, const double* ph, bool q4,
                                               double& r0, double& r1, double& r2) {
  const double w = m.gf[fc];
  double a0, a1, a2;
  if (q4) {
    a0 = (1 - w) * g0[n] + w * g0[o]; a1 = (1 - w) * g1[n] + w * g1[o]; a2 = (1 - w) * g2[n] + w * g2[o];
  } else {
    a0 = w * g0[n] + (1 - w) * g0[o]; a1 = w * g1[n] + (1 - w) * g1[o]; a2 = w * g2[n] + (1 - w) * g2[o];
  }
  const double d0 = m.CNx[fc], d1 = m.CNy[fc], d2 = m.CNz[fc];
  const double dmag = sqrt(dot3(d0, d1, d2, d0, d1, d2));
  const double e0 = d0 / dmag, e1 = d1 / dmag, e2 = d2 / dmag;
  const double lgm = (ph[n] - ph[o]) / dmag;
  const double agm = dot3(a0, a1, a2, e0, e1, e2);
  r0 = (a0 - agm * e0) + lgm * e0;
  r1 = (a1 - agm * e1) + lgm * e1;
  r2 = (a2 - agm * e2) + lgm * e2;
}

// cfdAssembleEquation('U', comp): convection (upwind) + convection divergence, diffusion,
// explicit stress, pressure gradient, false transient, URF, scaled residual, DU.
__global__ void __launch_bounds__(kBlock) k_assemble_u(MeshView m, FieldView f, AsmArgs a) {
  __shared__ double sh[32];
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  double rr = 0.0, rm = 0.0;
  if (e < m.Nc) {
    const int comp = a.comp;
    const double* ph = Uc(f, comp);
    const int s = m.cfStart[e], ne = m.cfStart[e + 1];
    const int r0 = m.rowptr[e];
    double acv = 0.0, bcv = 0.0, eff = 0.0;
    // (1) convection, sign +1 (cfdAssembleConvectionTerm.m:103-232)
    for (int q = s; q < ne; ++q) {
      const int fc = m.cfFace[q];
      const double psi = f.mdot[fc];
      if (fc < m.Fi) {
        const int o = m.owner[fc], n = m.neigh[fc];
        const double C1 = 1.0 * dmax(psi, 0.0);
        const double C2 = -1.0 * dmax(-psi, 0.0);
        const double T = (C1 * ph[o] + C2 * ph[n]) + 0.0;
        if (o == e) { acv = acv + C1; a.anb[r0 + q - s] = 0.0 + C2; bcv = bcv - T; eff = eff + psi; }
        else { acv = acv - C2; a.anb[r0 + q - s] = 0.0 - C1; bcv = bcv + T; eff = eff - psi; }
      } else {
        const int b = m.Nc + fc - m.Fi;
        const int ty = m.ptype[m.bPatch[fc - m.Fi]];
        double C1 = 0.0, T = 0.0;
        if (ty == UFVM_PATCH_INLET || ty == UFVM_PATCH_OUTLET) {
          C1 = 1.0 * dmax(psi, 0.0);
          const double C2 = -1.0 * dmax(-psi, 0.0);
          T = (C1 * ph[e] + C2 * ph[b]) + 0.0;
        }
        acv = acv + C1;
        bcv = bcv - T;
        eff = eff + psi;
      }
    }
    {  // cfdAssembleConvectionDivergenceTerm
      const double fce = dmax(eff, 0.0) - eff;
      const double fve = -dmax(eff, 0.0) * ph[e];
      const double fte = fce * ph[e] + fve;
      acv = acv + fce;
      bcv = bcv - fte;
    }
    // (2) diffusion, sign -1 (cfdAssembleDiffusionTerm.m:94-690)
    const bool q4 = (a.quirks & UFVM_Q4_GRAD_WEIGHTS_SWAPPED) != 0;
    const double* g0 = f.gU[comp * 3];
    const double* g1 = f.gU[comp * 3 + 1];
    const double* g2 = f.gU[comp * 3 + 2];
    const double nu = a.nu;
    for (int q = s; q < ne; ++q) {
      const int fc = m.cfFace[q];
      if (fc < m.Fi) {
        const int o = m.owner[fc], n = m.neigh[fc];
        double gf0, gf1, gf2;
        face_grad_corr(m, fc, o, n, g0, g1, g2, ph, q4, gf0, gf1, gf2);
        const double w = m.gf[fc];
        const double gam = w * nu + (1 - w) * nu;
        const double C1 = (1.0 * gam) * m.gDiff[fc];
        const double C2 = (-1.0 * gam) * m.gDiff[fc];
        const double V = (-1.0 * gam) * dot3(gf0, gf1, gf2, m.Tx[fc], m.Ty[fc], m.Tz[fc]);
        const double T = (C1 * ph[o] + C2 * ph[n]) + V;
        const int k = r0 + q - s;
        if (o == e) { acv = acv + C1; a.anb[k] = a.anb[k] + C2; bcv = bcv - T; }
        else { acv = acv - C2; a.anb[k] = a.anb[k] - C1; bcv = bcv + T; }
      } else {
        const int kb = fc - m.Fi, b = m.Nc + kb, p = m.bPatch[kb];
        const int ty = m.ptype[p], tu = m.bcU[p];
        const double gam = nu;
        double C1 = 0.0, T = 0.0;
        if ((ty == UFVM_PATCH_WALL || ty == UFVM_PATCH_INLET) && tu == UFVM_BC_FIXED_VALUE) {
          C1 = (1.0 * gam) * m.gDiff[fc];
          const double C2 = (-1.0 * gam) * m.gDiff[fc];
          const double V = (-1.0 * gam) * dot3(g0[b], g1[b], g2[b], m.Tx[fc], m.Ty[fc], m.Tz[fc]);
          T = (C1 * ph[e] + C2 * ph[b]) + V;
        } else if (ty == UFVM_PATCH_WALL && tu == UFVM_BC_NOSLIP) {
          // cfdAssembleDiffusionTermWallNoslipBC (:479-562): Q3, Q14, Q15
          const double A = m.area[fc];
          const double n0 = m.Sx[fc] / A, n1 = m.Sy[fc] / A, n2 = m.Sz[fc] / A;
          const int c2 = comp == 0 ? 1 : 0, c3 = comp == 2 ? 1 : 2;
          const double nc = comp == 0 ? n0 : (comp == 1 ? n1 : n2);
          const double nn2 = c2 == 0 ? n0 : n1;
          const double nn3 = c3 == 1 ? n1 : n2;
          const double dn = m.wd[fc];
          const double TM = (a.quirks & UFVM_Q3_NOSLIP_GAMMA_TWICE) ? gam / dn : 1.0;
          const double fac = (a.quirks & UFVM_Q14_NOSLIP_PATCH_SUM) ? (1 - m.pnsum[3 * p + comp]) : (1 - nc * nc);
          const double third = (a.quirks & UFVM_Q15_NOSLIP_THIRD_SIGN) ? -1.0 : 1.0;
          const double coef = ((1.0 * gam) * A / dn) * TM;
          C1 = coef * fac;
          const double* U2c = Uc(f, c2);
          const double* U3c = Uc(f, c3);
          const double inner = (ph[b] * fac + (U2c[e] - U2c[b]) * nn2 * nc) + third * ((U3c[e] - U3c[b]) * nn3 * nc);
          const double bcf = coef * inner;
          T = (C1 * ph[e] + 0.0 * ph[b]) + bcf;
        } else if (ty == UFVM_PATCH_SYMMETRY || ty == UFVM_PATCH_EMPTY) {
          const double A = m.area[fc];
          const double n0 = m.Sx[fc] / A, n1 = m.Sy[fc] / A, n2 = m.Sz[fc] / A;
          const double dd = dot3(m.CNx[fc], m.CNy[fc], m.CNz[fc], n0, n1, n2);
          const double l0 = comp == 0 ? 0.0 : 1.0, l1 = comp == 1 ? 0.0 : 1.0, l2 = comp == 2 ? 0.0 : 1.0;
          const double nc = comp == 0 ? n0 : (comp == 1 ? n1 : n2);
          const double dv = dot3(f.U0[e] * l0, f.U1[e] * l1, f.U2[e] * l2, n0 * l0, n1 * l1, n2 * l2);
          C1 = ((((1.0 * 2) * gam) * A) * (nc * nc)) / dd;
          const double V = (((((-1.0 * 2) * gam) * A) * dv) * nc) / dd;
          T = (C1 * ph[e] + 0.0 * ph[b]) + V;
        }
        acv = acv + C1;
        bcv = bcv - T;
      }
    }
    // (3) explicit stress div(nu*transp(grad(U))), sign -1 (cfdAssembleExplicitStressTerm.m:13-49, Q2)
    const bool q2 = (a.quirks & UFVM_Q2_STRESS_NOT_TRANSPOSED) != 0;
    const double* s0 = q2 ? f.gU[comp * 3 + 0] : f.gU[0 * 3 + comp];
    const double* s1 = q2 ? f.gU[comp * 3 + 1] : f.gU[1 * 3 + comp];
    const double* s2 = q2 ? f.gU[comp * 3 + 2] : f.gU[2 * 3 + comp];
    for (int q = s; q < ne; ++q) {
      const int fc = m.cfFace[q];
      double x0, x1, x2, gam;
      if (fc < m.Fi) {
        const int o = m.owner[fc], n = m.neigh[fc];
        const double w = m.gf[fc];
        x0 = w * s0[n] + (1 - w) * s0[o]; x1 = w * s1[n] + (1 - w) * s1[o]; x2 = w * s2[n] + (1 - w) * s2[o];
        gam = w * nu + (1 - w) * nu;
        const double T = (-1.0 * gam) * ((x0 * m.Sx[fc] + x1 * m.Sy[fc]) + x2 * m.Sz[fc]);
        const int k = r0 + q - s;
        if (o == e) { acv = acv + 0.0; a.anb[k] = a.anb[k] + 0.0; bcv = bcv - T; }
        else { acv = acv - 0.0; a.anb[k] = a.anb[k] - 0.0; bcv = bcv + T; }
      } else {
        const int b = m.Nc + fc - m.Fi;
        x0 = s0[b]; x1 = s1[b]; x2 = s2[b];
        gam = nu;
        const double T = (-1.0 * gam) * ((x0 * m.Sx[fc] + x1 * m.Sy[fc]) + x2 * m.Sz[fc]);
        acv = acv + 0.0;
        bcv = bcv - T;
      }
    }
    // (4) grad(p), sign +1 (cfdAssemblePressureGradientTerm.m:11-40)
    const double V = m.vol[e];
    {
      const double fte = (1.0 * V) * gpd(f, comp)[e];
      acv = acv + 0.0;
      bcv = bcv - fte;
    }
    // (5) false transient (cfdAssembleFalseTransientTerm.m:15-49)
    {
      const double fce = (V * 1.0) / a.fdt;
      const double fte = fce * ph[e];
      acv = acv + fce;
      bcv = bcv - fte;
    }
    // (6) URF (cfdApplyURF.m:13-16)
    acv = acv / a.urf;
    a.ac[e] = acv;
    a.bc[e] = bcv;
    if (acv == 0.0) atomicExch(a.zero_diag, 1);
    // (7) scaled residual terms (cfdComputeNormalizedResidual.m:55-88)
    const double r = bcv / (acv * a.scale);
    rr = r * r;
    rm = fabs(r);
    // (8) DU = V / ac (cfdPostAssembleEquation.m:37-42)
    a.DUout[e] = V / acv;
  }
  rr = block_reduce<0>(rr, sh);
  if (threadIdx.x == 0) a.part[2 * blockIdx.x] = rr;
  rm = block_reduce<1>(rm, sh);
  if (threadIdx.x == 0) a.part[2 * blockIdx.x + 1] = rm;
}

__global__ void k_copy_owner(int Nc, int Fi, int Fb, const int* __restrict__ owner, double* v) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < Fb) v[Nc + k] = v[owner[Fi + k]];
}

// ---------------------------------------------------------------- Rhie-Chow (cfdAssembleMdotTerm.m)
__global__ void k_rhiechow(MeshView m, FieldView f, double urfU, int quirks, int* bad_bc) {
  const int fc = blockIdx.x * blockDim.x + threadIdx.x;
  if (fc >= m.F) return;
  const double S0 = m.Sx[fc], S1 = m.Sy[fc], S2 = m.Sz[fc];
  if (fc < m.Fi) {
    const int o = m.owner[fc], n = m.neigh[fc];
    const double w = m.gf[fc];
    const double db0 = w * f.DU0[n] + (1 - w) * f.DU0[o];
    const double db1 = w * f.DU1[n] + (1 - w) * f.DU1[o];
    const double db2 = w * f.DU2[n] + (1 - w) * f.DU2[o];
    const double ub0 = w * f.U0[n] + (1 - w) * f.U0[o];
    const double ub1 = w * f.U1[n] + (1 - w) * f.U1[o];
    const double ub2 = w * f.U2[n] + (1 - w) * f.U2[o];
    const double mprev = f.mdot[fc];
    const double pos = mprev > 0 ? 1.0 : 0.0;
    const double rf = 1.0 * pos + 1.0 * (1 - pos);
    const bool q4 = (quirks & UFVM_Q4_GRAD_WEIGHTS_SWAPPED) != 0;
    double gb0, gb1, gb2;
    if (q4) {
      gb0 = (1 - w) * f.gp0[n] + w * f.gp0[o]; gb1 = (1 - w) * f.gp1[n] + w * f.gp1[o]; gb2 = (1 - w) * f.gp2[n] + w * f.gp2[o];
    } else {
      gb0 = w * f.gp0[n] + (1 - w) * f.gp0[o]; gb1 = w * f.gp1[n] + (1 - w) * f.gp1[o]; gb2 = w * f.gp2[n] + (1 - w) * f.gp2[o];
    }
    double gc0, gc1, gc2;
    face_grad_corr(m, fc, o, n, f.gp0, f.gp1, f.gp2, f.p, q4, gc0, gc1, gc2);
    const double Ub = dot3(ub0, ub1, ub2, S0, S1, S2);
    double V = 0 + rf * Ub;
    const double D0 = db0 * S0, D1 = db1 * S1, D2 = db2 * S2;
    const double mD = sqrt(dot3(D0, D1, D2, D0, D1, D2));
    const double eD0 = D0 / mD, eD1 = D1 / mD, eD2 = D2 / mD;
    const double ec0 = m.eCx[fc], ec1 = m.eCy[fc], ec2 = m.eCz[fc];
    const double den = dot3(ec0, ec1, ec2, eD0, eD1, eD2);
    const double E0 = (mD * ec0) / den, E1 = (mD * ec1) / den, E2 = (mD * ec2) / den;
    const double cn0 = m.CNx[fc], cn1 = m.CNy[fc], cn2 = m.CNz[fc];
    const double geo = sqrt(dot3(E0, E1, E2, E0, E1, E2)) / sqrt(dot3(cn0, cn1, cn2, cn0, cn1, cn2));
    const double T0 = D0 - E0, T1 = D1 - E1, T2 = D2 - E2;
    const double FC = 0 + rf * geo;
    const double FF = 0 - rf * geo;
    V = V - rf * dot3(gc0, gc1, gc2, T0, T1, T2);
    V = V + rf * dot3(gb0, gb1, gb2, D0, D1, D2);
    V = V + (1 - urfU) * (mprev - rf * Ub);
    f.mdot[fc] = (FC * f.p[o] + FF * f.p[n]) + V;
    f.fC1[fc] = FC;
    f.fC2[fc] = FF;
    return;
  }
  const int kb = fc - m.Fi, b = m.Nc + kb, p = m.bPatch[kb], o = m.owner[fc];
  const int ty = m.ptype[p], tp = m.bcP[p];
  if (ty == UFVM_PATCH_INLET && tp != UFVM_BC_FIXED_VALUE) {
    // cfdAssembleMdotTermInletInletBC (:281-350)
    const double Usf = dot3(S0, S1, S2, f.U0[b], f.U1[b], f.U2[b]);
    const double V = 0 + 1.0 * Usf;
    f.mdot[fc] = (0.0 * f.p[o] + 0.0 * f.p[b]) + V;
    f.fC1[fc] = 0.0;
    f.fC2[fc] = 0.0;
  } else if (ty == UFVM_PATCH_OUTLET && tp == UFVM_BC_FIXED_VALUE) {
    // cfdAssembleMdotTermOutletFixedValueBC (:799-905)
    const double rb = 1.0;
    const double D0 = f.DU0[b] * S0, D1 = f.DU1[b] * S1, D2 = f.DU2[b] * S2;
    const double mD = sqrt(dot3(D0, D1, D2, D0, D1, D2));
    const double eD0 = D0 / mD, eD1 = D1 / mD, eD2 = D2 / mD;
    const double ec0 = m.eCx[fc], ec1 = m.eCy[fc], ec2 = m.eCz[fc];
    const double den = dot3(ec0, ec1, ec2, eD0, eD1, eD2);
    const double E0 = (mD / den) * ec0, E1 = (mD / den) * ec1, E2 = (mD / den) * ec2;
    const double cn0 = m.CNx[fc], cn1 = m.CNy[fc], cn2 = m.CNz[fc];
    const double geo = sqrt(dot3(E0, E1, E2, E0, E1, E2)) / sqrt(dot3(cn0, cn1, cn2, cn0, cn1, cn2));
    const double T0 = D0 - E0, T1 = D1 - E1, T2 = D2 - E2;
    const double gb0 = f.gp0[b], gb1 = f.gp1[b], gb2 = f.gp2[b];
    const double Ub = dot3(f.U0[b], f.U1[b], f.U2[b], S0, S1, S2);
    double V = 0.0 + rb * Ub;
    const double FC = 0.0 + rb * geo;
    const double FF = 0.0 - 0.0;
    V = V - rb * dot3(gb0, gb1, gb2, T0, T1, T2);
    V = V + rb * dot3(gb0, gb1, gb2, D0, D1, D2);
    f.mdot[fc] = (FC * f.p[o] + FF * f.p[b]) + V;
    f.fC1[fc] = FC;
    f.fC2[fc] = FF;
  } else if (ty == UFVM_PATCH_WALL || ty == UFVM_PATCH_EMPTY || ty == UFVM_PATCH_SYMMETRY) {
    f.fC1[fc] = 0.0;
    f.fC2[fc] = 0.0;
  } else {
    atomicExch(bad_bc, 1);
  }
}

// cfdAssembleIntoGlobalMatrixFaceFluxes for the p equation + effective divergence residual
__global__ void __launch_bounds__(kBlock) k_assemble_p(MeshView m, FieldView f, double* ac, double* bc, double* anb,
                                                       double* part) {
  __shared__ double sh[32];
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  double e2 = 0.0, em = -INFINITY;
  if (e < m.Nc) {
    const int s = m.cfStart[e], ne = m.cfStart[e + 1], r0 = m.rowptr[e];
    double acv = 0.0, bcv = 0.0, eff = 0.0;
    for (int q = s; q < ne; ++q) {
      const int fc = m.cfFace[q];
      const double md = f.mdot[fc];
      if (fc < m.Fi) {
        const double C1 = f.fC1[fc], C2 = f.fC2[fc];
        if (m.owner[fc] == e) { acv = acv + C1; anb[r0 + q - s] = 0.0 + C2; bcv = bcv - md; eff = eff + md; }
        else { acv = acv - C2; anb[r0 + q - s] = 0.0 - C1; bcv = bcv + md; eff = eff - md; }
      } else {
        const int p = m.bPatch[fc - m.Fi];
        const int ty = m.ptype[p];
        const double T = (ty == UFVM_PATCH_INLET || ty == UFVM_PATCH_OUTLET) ? md : 0.0;
        acv = acv + f.fC1[fc];
        bcv = bcv - T;
        eff = eff + md;
      }
    }
    ac[e] = acv;
    bc[e] = bcv;
    e2 = eff * eff;
    em = eff;
  }
  e2 = block_reduce<0>(e2, sh);
  if (threadIdx.x == 0) part[2 * blockIdx.x] = e2;
  em = block_reduce<1>(em, sh);
  if (threadIdx.x == 0) part[2 * blockIdx.x + 1] = em;
}

// ---------------------------------------------------------------- corrections
__global__ void k_add(int n, double* __restrict__ x, const double* __restrict__ d) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] = x[i] + d[i];
}

// cfdCorrectScalarEquation.m:16-109 boundary part for U component comp
__global__ void k_correct_u_bc(MeshView m, FieldView f, int comp) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m.Fb) return;
  const int fc = m.Fi + k, p = m.bPatch[k], ty = m.ptype[p], tu = m.bcU[p];
  const int b = m.Nc + k, o = m.owner[fc];
  double* u = Uc(f, comp);
  if (ty == UFVM_PATCH_WALL) {
    if (tu == UFVM_BC_ZERO_GRADIENT) u[b] = u[o];
    else if (tu == UFVM_BC_SLIP) tangential(m, f, fc, b, o, comp, comp);
  } else if (ty == UFVM_PATCH_OUTLET) {
    if (tu == UFVM_BC_ZERO_GRADIENT) u[b] = u[o];
  } else if (ty == UFVM_PATCH_SYMMETRY || ty == UFVM_PATCH_EMPTY) {
    tangential(m, f, fc, b, o, comp, comp);
  }
}

// cfdCorrectPPField.m:26-52
__global__ void k_pp_cells(int Nc, int fixed, const double* __restrict__ dphi, double* PP) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= Nc) return;
  const double ppc = fixed >= 0 ? dphi[fixed] : 0.0;
  PP[e] = dphi[e] - ppc;
}

__global__ void k_pp_bc(MeshView m, FieldView f) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m.Fb) return;
  const int p = m.bPatch[k], ty = m.ptype[p], tp = m.bcP[p];
  const int b = m.Nc + k;
  if ((ty == UFVM_PATCH_INLET || ty == UFVM_PATCH_OUTLET) && tp == UFVM_BC_FIXED_VALUE) f.PP[b] = 0.0;
  else f.PP[b] = f.PP[m.owner[m.Fi + k]];
}

// cfdCorrectVelocityField.m:26-55 (interior)
__global__ void k_vel_cells(int Nc, FieldView f) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= Nc) return;
  f.U0[e] = f.U0[e] - f.DU0[e] * f.gPP0[e];
  f.U1[e] = f.U1[e] - f.DU1[e] * f.gPP1[e];
  f.U2[e] = f.U2[e] - f.DU2[e] * f.gPP2[e];
}

// velocity boundary correction of one patch: mode 1 tangential (symmetry, empty, slip),
// mode 2 gather owner velocity (outlet with fixed p), mode 3 scatter it to `row0 + j`.
__global__ void k_vel_patch(MeshView m, FieldView f, int start, int count, int mode, int row0, double* tmp) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= count) return;
  const int fc = start + j, o = m.owner[fc];
  if (mode == 1) {
    tangential(m, f, fc, m.Nc + fc - m.Fi, o, 0, 2);
  } else if (mode == 2) {
    tmp[3 * j] = f.U0[o]; tmp[3 * j + 1] = f.U1[o]; tmp[3 * j + 2] = f.U2[o];
  } else {
    const int row = row0 + j;
    f.U0[row] = tmp[3 * j]; f.U1[row] = tmp[3 * j + 1]; f.U2[row] = tmp[3 * j + 2];
  }
}

// cfdCorrectPressureEquation.m:22-54
__global__ void k_p_cells(int Nc, int fixed, double urfP, FieldView f) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= Nc) return;
  const double ppf = fixed >= 0 ? f.PP[fixed] : 0.0;
  f.p[e] = f.p[e] + urfP * (f.PP[e] - ppf);
}

__global__ void k_p_bc(MeshView m, FieldView f) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m.Fb) return;
  const int p = m.bPatch[k], ty = m.ptype[p], tp = m.bcP[p];
  if ((ty == UFVM_PATCH_INLET || ty == UFVM_PATCH_OUTLET) && tp == UFVM_BC_FIXED_VALUE) return;
  f.p[m.Nc + k] = f.p[m.owner[m.Fi + k]];
}

// cfdCorrectMdotField.m:24-50 + boundary patches
__global__ void k_mdot_correct(MeshView m, FieldView f) {
  const int fc = blockIdx.x * blockDim.x + threadIdx.x;
  if (fc >= m.F) return;
  if (fc < m.Fi) {
    f.mdot[fc] = (f.mdot[fc] + f.fC1[fc] * f.PP[m.owner[fc]]) + f.fC2[fc] * f.PP[m.neigh[fc]];
    return;
  }
  const int p = m.bPatch[fc - m.Fi], ty = m.ptype[p], tp = m.bcP[p];
  if (ty == UFVM_PATCH_SYMMETRY || ty == UFVM_PATCH_EMPTY || (ty == UFVM_PATCH_WALL && tp == UFVM_BC_SLIP)) {
    f.mdot[fc] = 0.0 * f.mdot[fc];
  } else if (ty == UFVM_PATCH_OUTLET && tp == UFVM_BC_FIXED_VALUE) {
    const int o = m.owner[fc];
    f.mdot[fc] = 1.0 * dot3(f.U0[o], f.U1[o], f.U2[o], m.Sx[fc], m.Sy[fc], m.Sz[fc]);
  }
}

// ================================================================ host orchestration
int Case::update_fields() {
  const MeshView m = mv();
  FieldView f = fv();
  k_bc_update<<<nblocks(M.Fb), kBlock, 0, stream>>>(m, f);
  UFVM_LAUNCH_CHECK();
  double* phiU[3] = {U[0].p, U[1].p, U[2].p};
  double* gUp[9];
  for (int k = 0; k < 9; ++k) gUp[k] = gU[k].p;
  UFVM_CHECK(gradient(phiU, 3, gUp, true));
  // scale over every active row of U
  const int nb = nblocks(rowsU);
  UFVM_CHECK(dalloc(part, 2 * std::max(nb, nblocks(M.F)) + 8));
  UFVM_CHECK(dalloc(red, 8));
  k_minmax<<<nb, kBlock, 0, stream>>>(rowsU, U[0].p, U[1].p, U[2].p, part.p);
  k_final2<1, 2><<<1, 1024, 0, stream>>>(nb, part.p, red.p);
  UFVM_LAUNCH_CHECK();
  double mm[2];
  UFVM_CUDA(cudaMemcpyAsync(mm, red.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, stream));
  UFVM_CUDA(cudaStreamSynchronize(stream));
  double sc = std::max(mm[0] - mm[1], std::fabs(mm[0]));
  if (sc < 1e-6) sc = 1;
  scaleU = sc;
  double* phiP[1] = {p.p};
  double* gPp[3] = {gp[0].p, gp[1].p, gp[2].p};
  UFVM_CHECK(gradient(phiP, 1, gPp, false));
  return UFVM_OK;
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
  Level& L = lev[0];
  const int nb = nblocks(M.Nc);
  UFVM_CHECK(dalloc(part, 2 * std::max(nb, nblocks(M.F)) + 8));
  UFVM_CHECK(dalloc(flags, 8));
  UFVM_CUDA(cudaMemsetAsync(flags.p, 0, 8 * sizeof(int), stream));
  AsmArgs a;
  a.comp = comp; a.quirks = S.quirks; a.nu = S.nu; a.urf = S.urf_u; a.fdt = S.false_dt; a.scale = scaleU;
  a.ac = L.ac.p; a.bc = L.bc.p; a.anb = L.anb.p; a.DUout = DU[comp].p; a.part = part.p; a.zero_diag = flags.p;
  k_assemble_u<<<nb, kBlock, 0, stream>>>(mv(), fv(), a);
  k_copy_owner<<<nblocks(M.Fb), kBlock, 0, stream>>>(M.Nc, M.Fi, M.Fb, M.owner.p, DU[comp].p);
  k_final2<0, 1><<<1, 1024, 0, stream>>>(nb, part.p, red.p);
  UFVM_LAUNCH_CHECK();
  double out[2];
  int zd = 0;
  UFVM_CUDA(cudaMemcpyAsync(out, red.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, stream));
  UFVM_CUDA(cudaMemcpyAsync(&zd, flags.p, sizeof(int), cudaMemcpyDeviceToHost, stream));
  UFVM_CUDA(cudaStreamSynchronize(stream));
  if (zd) { set_error("****** Divide by Zero ******* (ac == 0 in U equation)"); return UFVM_E_ZERO_DIAG; }
  *rms = std::sqrt(out[0] / M.Nc);
  *mx = out[1];
  return UFVM_OK;
}

int Case::assemble_p(double* rms, double* mx) {
  UFVM_CHECK(fresh_level0());
  Level& L = lev[0];
  UFVM_CHECK(dalloc(flags, 8));
  UFVM_CUDA(cudaMemsetAsync(flags.p, 0, 8 * sizeof(int), stream));
  k_rhiechow<<<nblocks(M.F), kBlock, 0, stream>>>(mv(), fv(), S.urf_u, S.quirks, flags.p + 1);
  const int nb = nblocks(M.Nc);
  UFVM_CHECK(dalloc(part, 2 * std::max(nb, nblocks(M.F)) + 8));
  k_assemble_p<<<nb, kBlock, 0, stream>>>(mv(), fv(), L.ac.p, L.bc.p, L.anb.p, part.p);
  k_final2<0, 1><<<1, 1024, 0, stream>>>(nb, part.p, red.p);
  UFVM_LAUNCH_CHECK();
  double out[2];
  int bad = 0;
  UFVM_CUDA(cudaMemcpyAsync(out, red.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, stream));
  UFVM_CUDA(cudaMemcpyAsync(&bad, flags.p + 1, sizeof(int), cudaMemcpyDeviceToHost, stream));
  UFVM_CUDA(cudaStreamSynchronize(stream));
  if (bad) { set_error("p boundary condition not implemented for this patch type"); return UFVM_E_BC_UNSUPPORTED; }
  *rms = std::sqrt(out[0] / M.Nc);
  *mx = out[1];
  return UFVM_OK;
}

int Case::correct_u(int comp) {
  Level& L = lev[0];
  k_add<<<nblocks(M.Nc), kBlock, 0, stream>>>(M.Nc, U[comp].p, L.dphi.p);
  k_correct_u_bc<<<nblocks(M.Fb), kBlock, 0, stream>>>(mv(), fv(), comp);
  UFVM_LAUNCH_CHECK();
  return UFVM_OK;
}

int Case::correct_p() {
  Level& L = lev[0];
  const MeshView m = mv();
  FieldView f = fv();
  k_pp_cells<<<nblocks(M.Nc), kBlock, 0, stream>>>(M.Nc, S.fixed_element, L.dphi.p, PP.p);
  k_pp_bc<<<nblocks(M.Fb), kBlock, 0, stream>>>(m, f);
  UFVM_LAUNCH_CHECK();
  double* phiPP[1] = {PP.p};
  double* gPPp[3] = {gPP[0].p, gPP[1].p, gPP[2].p};
  UFVM_CHECK(gradient(phiPP, 1, gPPp, false));
  k_vel_cells<<<nblocks(M.Nc), kBlock, 0, stream>>>(M.Nc, f);
  UFVM_LAUNCH_CHECK();
  // boundary velocity, patch by patch in patch order (later patches overwrite earlier ones,
  // as the reference's sequential patch loop does)
  for (int ip = 0; ip < P.n; ++ip) {
    const int ty = P.type[ip], tp = P.bcP[ip], cnt = P.count[ip];
    if (cnt == 0) continue;
    if (ty == UFVM_PATCH_OUTLET && tp == UFVM_BC_FIXED_VALUE) {
      const int row0 = (S.quirks & UFVM_Q12_OUTLET_U_FACE_ROWS) ? P.start[ip] : M.Nc + P.start[ip] - M.Fi;
      UFVM_CHECK(dalloc(tmp3, 3 * (size_t)cnt));
      k_vel_patch<<<nblocks(cnt), kBlock, 0, stream>>>(m, f, P.start[ip], cnt, 2, row0, tmp3.p);
      k_vel_patch<<<nblocks(cnt), kBlock, 0, stream>>>(m, f, P.start[ip], cnt, 3, row0, tmp3.p);
      rowsU = std::max(rowsU, row0 + cnt);
    } else if (ty == UFVM_PATCH_SYMMETRY || ty == UFVM_PATCH_EMPTY || (ty == UFVM_PATCH_WALL && tp == UFVM_BC_SLIP)) {
      k_vel_patch<<<nblocks(cnt), kBlock, 0, stream>>>(m, f, P.start[ip], cnt, 1, 0, nullptr);
    }
  }
  UFVM_LAUNCH_CHECK();
  k_p_cells<<<nblocks(M.Nc), kBlock, 0, stream>>>(M.Nc, S.fixed_element, S.urf_p, f);
  k_p_bc<<<nblocks(M.Fb), kBlock, 0, stream>>>(m, f);
  k_mdot_correct<<<nblocks(M.F), kBlock, 0, stream>>>(m, f);
  UFVM_LAUNCH_CHECK();
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
  UFVM_CHECK(dalloc(fC1, F));
  UFVM_CHECK(dalloc(fC2, F));
  UFVM_CUDA(cudaMemsetAsync(fC1.p, 0, F * sizeof(double), stream));
  UFVM_CUDA(cudaMemsetAsync(fC2.p, 0, F * sizeof(double), stream));
  const MeshView m = mv();
  FieldView f = fv();
  k_bc_init<<<nblocks(Fb), kBlock, 0, stream>>>(m, f);
  UFVM_LAUNCH_CHECK();
  double* phiU[3] = {U[0].p, U[1].p, U[2].p};
  double* gUp[9];
  for (int k = 0; k < 9; ++k) gUp[k] = gU[k].p;
  UFVM_CHECK(gradient(phiU, 3, gUp, true));
  double* phiP[1] = {p.p};
  double* gPp[3] = {gp[0].p, gp[1].p, gp[2].p};
  UFVM_CHECK(gradient(phiP, 1, gPp, false));
  if (mdot0h) {
    UFVM_CUDA(cudaMemcpyAsync(mdot.p, mdot0h, F * sizeof(double), cudaMemcpyHostToDevice, stream));
  } else {
    k_mdot_init<<<nblocks(F), kBlock, 0, stream>>>(m, f);
    UFVM_LAUNCH_CHECK();
  }
  UFVM_CHECK(fresh_level0());
  UFVM_CUDA(cudaStreamSynchronize(stream));
  return UFVM_OK;
}

}  // namespace ufvm
