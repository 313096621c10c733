// stages.cu -- batched SIMPLE stage kernels. Each kernel is launched over a (slot, block)
// work list and reads its case from the slot table; the arithmetic of every expression is
// the MATLAB source's, term by term, left to right (see simple.cu for the ordering argument).
#include "simple.cuh"

namespace ufvm {

#define SLOT_BEGIN(WORK)                                     \
  const int2 w_ = (WORK)[blockIdx.x];                        \
  const SlotDesc& S = slots[w_.x];                           \
  const MeshView& m = S.m;                                   \
  const int idx = w_.y * blockDim.x + threadIdx.x;

__device__ __forceinline__ double* Uc(const FieldView& f, int c) { return c == 0 ? f.U0 : (c == 1 ? f.U1 : f.U2); }
__device__ __forceinline__ double* DUc(const FieldView& f, int c) { return c == 0 ? f.DU0 : (c == 1 ? f.DU1 : f.DU2); }
__device__ __forceinline__ double* gpd(const FieldView& f, int d) { return d == 0 ? f.gp0 : (d == 1 ? f.gp1 : f.gp2); }

__device__ __forceinline__ void tangential(const MeshView& m, const FieldView& f, int fc, int b, int o, int c0, int c1) {
  const double S0 = m.Sx[fc], S1 = m.Sy[fc], S2 = m.Sz[fc];
  const double nS = sqrt(dot3(S0, S1, S2, S0, S1, S2));
  const double n0 = S0 / nS, n1 = S1 / nS, n2 = S2 / nS;
  const double un = dot3(f.U0[o], f.U1[o], f.U2[o], n0, n1, n2);
  for (int c = c0; c <= c1; ++c) {
    const double nc = c == 0 ? n0 : (c == 1 ? n1 : n2);
    Uc(f, c)[b] = Uc(f, c)[o] - un * nc;
  }
}

// ---------------------------------------------------------------- boundary conditions
// update/cfdUpdateBoundaryConditions.m:13-96 (per-iteration: fixed values only)
__global__ void k_bc_update(const SlotDesc* __restrict__ slots, const int2* __restrict__ work) {
  SLOT_BEGIN(work);
  const int k = idx;
  if (k >= m.Fb) return;
  const FieldView& f = S.f;
  const int p = m.bPatch[k], ty = m.ptype[p], tu = m.bcU[p], tp = m.bcP[p];
  const int b = m.Nc + k;
  if ((ty == UFVM_PATCH_WALL && (tu == UFVM_BC_FIXED_VALUE || tu == UFVM_BC_NOSLIP)) ||
      ((ty == UFVM_PATCH_INLET || ty == UFVM_PATCH_OUTLET) && tu == UFVM_BC_FIXED_VALUE)) {
    f.U0[b] = f.vU0[k]; f.U1[b] = f.vU1[k]; f.U2[b] = f.vU2[k];
  }
  if (tp == UFVM_BC_FIXED_VALUE && (ty == UFVM_PATCH_WALL || ty == UFVM_PATCH_INLET || ty == UFVM_PATCH_OUTLET))
    f.p[b] = f.vP[k];
}

// initialize/cfdInitializeBoundaryConditions.m (initial boundary values)
__global__ void k_bc_init(const SlotDesc* __restrict__ slots, const int2* __restrict__ work) {
  SLOT_BEGIN(work);
  const int k = idx;
  if (k >= m.Fb) return;
  const FieldView& f = S.f;
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
__global__ void k_mdot_init(const SlotDesc* __restrict__ slots, const int2* __restrict__ work) {
  SLOT_BEGIN(work);
  const int fc = idx;
  if (fc >= m.F) return;
  const FieldView& f = S.f;
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
enum { G_U = 0, G_P = 1, G_PP = 2 };

template <int W>
__device__ __forceinline__ void grad_ptrs(const FieldView& f, const double** phi, double** g) {
  if (W == G_U) {
    phi[0] = f.U0; phi[1] = f.U1; phi[2] = f.U2;
    for (int k = 0; k < 9; ++k) g[k] = f.gU[k];
  } else if (W == G_P) {
    phi[0] = f.p; g[0] = f.gp0; g[1] = f.gp1; g[2] = f.gp2;
  } else {
    phi[0] = f.PP; g[0] = f.gPP0; g[1] = f.gPP1; g[2] = f.gPP2;
  }
}

// compute/cfdComputeGradientGauss0.m:28-80 (Q1: boundary value of component 1)
template <int W>
__global__ void __launch_bounds__(kBlock, 3) k_grad_cells(const SlotDesc* __restrict__ slots, const int2* __restrict__ work) {
  constexpr int NC = W == G_U ? 3 : 1;
  SLOT_BEGIN(work);
  const int e = idx;
  if (e >= m.Nc) return;
  const double* phi[3];
  double* gg[9];
  grad_ptrs<W>(S.f, phi, gg);
  const bool q1 = W == G_U && (S.quirks & UFVM_Q1_VEC_BOUNDARY_COMPONENT);
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
        const double phf = w * phi[c][n] + (1 - w) * phi[c][o];
        if (own) { g[c][0] = g[c][0] + phf * S0; g[c][1] = g[c][1] + phf * S1; g[c][2] = g[c][2] + phf * S2; }
        else { g[c][0] = g[c][0] - phf * S0; g[c][1] = g[c][1] - phf * S1; g[c][2] = g[c][2] - phf * S2; }
      }
    } else {
      const int b = m.Nc + fc - m.Fi;
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const double pb = phi[q1 ? 0 : c][b];
        g[c][0] = g[c][0] + pb * S0; g[c][1] = g[c][1] + pb * S1; g[c][2] = g[c][2] + pb * S2;
      }
    }
  }
  const double v = m.vol[e];
#pragma unroll
  for (int c = 0; c < NC; ++c)
#pragma unroll
    for (int d = 0; d < 3; ++d) gg[c * 3 + d][e] = g[c][d] / v;
}

// boundary rows: owner copy, then the wall / inlet / outlet correction (cfdUpdateGradient.m:81-255)
template <int W>
__global__ void k_grad_bfix(const SlotDesc* __restrict__ slots, const int2* __restrict__ work) {
  constexpr int NC = W == G_U ? 3 : 1;
  SLOT_BEGIN(work);
  const int k = idx;
  if (k >= m.Fb) return;
  const double* phi[3];
  double* gg[9];
  grad_ptrs<W>(S.f, phi, gg);
  const bool q1 = W == G_U && (S.quirks & UFVM_Q1_VEC_BOUNDARY_COMPONENT);
  const int fc = m.Fi + k, o = m.owner[fc], b = m.Nc + k;
  const int ty = m.ptype[m.bPatch[k]];
  const bool fix = ty == UFVM_PATCH_WALL || ty == UFVM_PATCH_INLET || ty == UFVM_PATCH_OUTLET;
  const double d0 = m.CNx[fc], d1 = m.CNy[fc], d2 = m.CNz[fc];
  const double dmag = sqrt(dot3(d0, d1, d2, d0, d1, d2));
  const double e0 = d0 / dmag, e1 = d1 / dmag, e2 = d2 / dmag;
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    const double g0 = gg[c * 3][o], g1 = gg[c * 3 + 1][o], g2 = gg[c * 3 + 2][o];
    if (!fix) {
      gg[c * 3][b] = g0; gg[c * 3 + 1][b] = g1; gg[c * 3 + 2][b] = g2;
      continue;
    }
    const int pc = (q1 && ty != UFVM_PATCH_WALL) ? 0 : c;
    const double ge = dot3(g0, g1, g2, e0, e1, e2);
    const double sn = (phi[pc][b] - phi[pc][o]) / dmag;
    gg[c * 3][b] = (g0 - ge * e0) + sn * e0;
    gg[c * 3 + 1][b] = (g1 - ge * e1) + sn * e1;
    gg[c * 3 + 2][b] = (g2 - ge * e2) + sn * e2;
  }
}

template <int W>
static int gradient(const BatchLaunch& b) {
  k_grad_cells<W><<<b.nwc, kBlock, 0, b.st>>>(b.slots, b.wc);
  k_grad_bfix<W><<<b.nwb, kBlock, 0, b.st>>>(b.slots, b.wb);
  UFVM_LAUNCH_CHECK();
  return UFVM_OK;
}

// ---------------------------------------------------------------- per-slot reductions
// stage 1 writes (a, b) pairs per work block; stage 2 reduces each slot's range in a
// fixed order. MODE 0: (sum r^2, max |r|) -> (sqrt(sum / Nc), max). MODE 1: (max, min) of U
// -> scale (cfdUpdateScale.m:15-28). MODE 2: (sum e^2, max e) -> (sqrt(sum / Nc), max).
template <int MODE>
__global__ void k_slot_final(const SlotDesc* __restrict__ slots, const int* __restrict__ ws,
                             const int* __restrict__ we, const double* __restrict__ part) {
  __shared__ double sh[32];
  const int s = blockIdx.x;
  const int a0 = ws[s], a1 = we[s];
  double a = MODE == 1 ? -INFINITY : 0.0, bb = MODE == 1 ? INFINITY : -INFINITY;
  for (int k = a0 + (int)threadIdx.x; k < a1; k += blockDim.x) {
    a = MODE == 1 ? dmax(a, part[2 * k]) : a + part[2 * k];
    bb = MODE == 1 ? dmin(bb, part[2 * k + 1]) : dmax(bb, part[2 * k + 1]);
  }
  if (MODE == 1) {
    a = block_reduce<1>(a, sh);
    const double mx = a;
    bb = block_reduce<2>(bb, sh);
    if (threadIdx.x == 0) {
      double sc = dmax(mx - bb, fabs(mx));
      if (sc < 1e-6) sc = 1;
      slots[s].scal[SCAL_SCALE] = sc;
    }
  } else {
    a = block_reduce<0>(a, sh);
    const double sum = a;
    bb = block_reduce<1>(bb, sh);
    if (threadIdx.x == 0) {
      slots[s].scal[SCAL_RMS] = sqrt(sum / slots[s].m.Nc);
      slots[s].scal[SCAL_MAX] = bb;
    }
  }
}

__global__ void k_minmax_U(const SlotDesc* __restrict__ slots, const int2* __restrict__ work, double* part) {
  __shared__ double sh[32];
  SLOT_BEGIN(work);
  (void)m;
  double mx = -INFINITY, mn = INFINITY;
  if (idx < S.rowsU) {
    const FieldView& f = S.f;
    mx = dmax(dmax(f.U0[idx], f.U1[idx]), f.U2[idx]);
    mn = dmin(dmin(f.U0[idx], f.U1[idx]), f.U2[idx]);
  }
  mx = block_reduce<1>(mx, sh);
  if (threadIdx.x == 0) part[2 * blockIdx.x] = mx;
  mn = block_reduce<2>(mn, sh);
  if (threadIdx.x == 0) part[2 * blockIdx.x + 1] = mn;
}

// ---------------------------------------------------------------- momentum assembly
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

// The part of cfdAssembleEquation('U', comp) that depends on one face only: the upwind
// convection coefficients and flux (cfdAssembleConvectionTerm.m:103-232), the diffusion
// coefficients and flux (cfdAssembleDiffusionTerm.m:94-690; Q3, Q4, Q14, Q15) and the explicit
// stress flux (cfdAssembleExplicitStressTerm.m:13-49, Q2), computed once per face (each
// interior face serves two cells) into uft[comp][k][F]:
//   k = 0, 1, 2: convection C1, C2, T;  3, 4, 5: diffusion C1, C2, T;  6: stress T.
// The cell kernel below adds them exactly as the reference's scatter does.
enum { UF_C1 = 0, UF_C2 = 1, UF_T = 2, UF_D1 = 3, UF_D2 = 4, UF_TD = 5, UF_TS = 6, UF_N = 7 };
// Upwind convection coefficients of an interior face from its mass flux (sign +1): a function
// of mdot alone, so the cell kernel recomputes them instead of reading them back (the same
// operations give the same bits); uft[UF_C1] / uft[UF_C2] are written for boundary faces only.
__device__ __forceinline__ double conv_c1(double psi) { return 1.0 * dmax(psi, 0.0); }
__device__ __forceinline__ double conv_c2(double psi) { return -1.0 * dmax(-psi, 0.0); }

// Interior faces: the face terms of components c0..c1, stored at uft + comp * UF_N * F. The
// face's geometry, mass flux and cells are read once for all the components it forms. An
// interior face's terms depend only on the cells' values of the component, the gradients of
// the iteration and the mass flux, none of which the solve and correction of another component
// change (they write that component's cells and boundary values), so the service forms all
// three components' interior terms before the first component's solve.
__global__ void __launch_bounds__(kBlock, 3) k_uface_int(const SlotDesc* __restrict__ slots,
                                                         const int2* __restrict__ work, int c0, int c1) {
  SLOT_BEGIN(work);
  const int fc = idx;
  if (fc >= m.Fi) return;
  const FieldView& f = S.f;
  const int quirks = S.quirks;
  const bool q4 = (quirks & UFVM_Q4_GRAD_WEIGHTS_SWAPPED) != 0;
  const bool q2 = (quirks & UFVM_Q2_STRESS_NOT_TRANSPOSED) != 0;
  const double nu = S.nu;
  const size_t F = (size_t)m.F;
  const int o = m.owner[fc], n = m.neigh[fc];
  const double psi = f.mdot[fc];
  const double w = m.gf[fc];
  const double gD = m.gDiff[fc];
  const double d0 = m.CNx[fc], d1 = m.CNy[fc], d2 = m.CNz[fc];
  const double t0 = m.Tx[fc], t1 = m.Ty[fc], t2 = m.Tz[fc];
  const double sx = m.Sx[fc], sy = m.Sy[fc], sz = m.Sz[fc];
  const double gam = w * nu + (1 - w) * nu;
  const double dmag = sqrt(dot3(d0, d1, d2, d0, d1, d2));
  const double e0 = d0 / dmag, e1 = d1 / dmag, e2 = d2 / dmag;
#pragma unroll 1
  for (int comp = c0; comp <= c1; ++comp) {
    const double* ph = Uc(f, comp);
    const double* g0 = f.gU[comp * 3];
    const double* g1 = f.gU[comp * 3 + 1];
    const double* g2 = f.gU[comp * 3 + 2];
    const double* s0 = q2 ? f.gU[comp * 3 + 0] : f.gU[0 * 3 + comp];
    const double* s1 = q2 ? f.gU[comp * 3 + 1] : f.gU[1 * 3 + comp];
    const double* s2 = q2 ? f.gU[comp * 3 + 2] : f.gU[2 * 3 + comp];
    const double pho = ph[o], phn = ph[n];
    double Tc, D1, D2, TD, TS;
    {  // (1) convection, sign +1; C1, C2 of an interior face are recomputed from mdot by the cell kernel
      const double C1 = conv_c1(psi);
      const double C2 = conv_c2(psi);
      Tc = (C1 * pho + C2 * phn) + 0.0;
    }
    {  // (2) diffusion, sign -1, with the Average:Corrected face gradient
      // (interpolate/cfdInterpolateGradientsFromElementsToInteriorFaces.m:23-70; Q4 weights)
      double a0, a1, a2;
      if (q4) {
        a0 = (1 - w) * g0[n] + w * g0[o]; a1 = (1 - w) * g1[n] + w * g1[o]; a2 = (1 - w) * g2[n] + w * g2[o];
      } else {
        a0 = w * g0[n] + (1 - w) * g0[o]; a1 = w * g1[n] + (1 - w) * g1[o]; a2 = w * g2[n] + (1 - w) * g2[o];
      }
      const double lgm = (phn - pho) / dmag;
      const double agm = dot3(a0, a1, a2, e0, e1, e2);
      const double gf0 = (a0 - agm * e0) + lgm * e0;
      const double gf1 = (a1 - agm * e1) + lgm * e1;
      const double gf2 = (a2 - agm * e2) + lgm * e2;
      D1 = (1.0 * gam) * gD;
      D2 = (-1.0 * gam) * gD;
      const double V = (-1.0 * gam) * dot3(gf0, gf1, gf2, t0, t1, t2);
      TD = (D1 * pho + D2 * phn) + V;
    }
    {  // (3) explicit stress, sign -1
      const double x0 = w * s0[n] + (1 - w) * s0[o], x1 = w * s1[n] + (1 - w) * s1[o];
      const double x2 = w * s2[n] + (1 - w) * s2[o];
      TS = (-1.0 * gam) * ((x0 * sx + x1 * sy) + x2 * sz);
    }
    double* u = f.uft + (size_t)comp * UF_N * F;
    u[UF_T * F + fc] = Tc;
    u[UF_D1 * F + fc] = D1; u[UF_D2 * F + fc] = D2; u[UF_TD * F + fc] = TD;
    u[UF_TS * F + fc] = TS;
  }
}

// Boundary faces: the face terms of one component (they read the other components' boundary and
// owner values, which the earlier components' corrections have changed).
__global__ void __launch_bounds__(kBlock, 4) k_uface_bnd(const SlotDesc* __restrict__ slots,
                                                         const int2* __restrict__ work, int comp) {
  SLOT_BEGIN(work);
  if (idx >= m.Fb) return;
  const int fc = m.Fi + idx;
  const FieldView& f = S.f;
  const int quirks = S.quirks;
  const double* ph = Uc(f, comp);
  const double nu = S.nu;
  const double psi = f.mdot[fc];
  const double* g0 = f.gU[comp * 3];
  const double* g1 = f.gU[comp * 3 + 1];
  const double* g2 = f.gU[comp * 3 + 2];
  const bool q2 = (quirks & UFVM_Q2_STRESS_NOT_TRANSPOSED) != 0;
  const double* s0 = q2 ? f.gU[comp * 3 + 0] : f.gU[0 * 3 + comp];
  const double* s1 = q2 ? f.gU[comp * 3 + 1] : f.gU[1 * 3 + comp];
  const double* s2 = q2 ? f.gU[comp * 3 + 2] : f.gU[2 * 3 + comp];
  const size_t F = (size_t)m.F;
  double* u = f.uft + (size_t)comp * UF_N * F;
  const int e = m.owner[fc];
  const int kb = fc - m.Fi, b = m.Nc + kb, p = m.bPatch[kb];
  const int ty = m.ptype[p], tu = m.bcU[p];
  double Cc = 0.0, Tc = 0.0;  // stored with the other terms at the end, as above
  {  // (1) convection
    if (ty == UFVM_PATCH_INLET || ty == UFVM_PATCH_OUTLET) {
      Cc = 1.0 * dmax(psi, 0.0);
      const double C2 = -1.0 * dmax(-psi, 0.0);
      Tc = (Cc * ph[e] + C2 * ph[b]) + 0.0;
    }
  }
  const double gam = nu;
  {  // (2) diffusion
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
      const double TM = (quirks & UFVM_Q3_NOSLIP_GAMMA_TWICE) ? gam / dn : 1.0;
      const double fac = (quirks & UFVM_Q14_NOSLIP_PATCH_SUM) ? (1 - m.pnsum[3 * p + comp]) : (1 - nc * nc);
      const double third = (quirks & UFVM_Q15_NOSLIP_THIRD_SIGN) ? -1.0 : 1.0;
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
    // (3) explicit stress
    const double TS = (-1.0 * gam) * ((s0[b] * m.Sx[fc] + s1[b] * m.Sy[fc]) + s2[b] * m.Sz[fc]);
    u[UF_C1 * F + fc] = Cc; u[UF_T * F + fc] = Tc;
    u[UF_D1 * F + fc] = C1; u[UF_TD * F + fc] = T;
    u[UF_TS * F + fc] = TS;
  }
}

constexpr int kCellFaces = 8;  // cells with at most this many faces take the register path

// cfdAssembleEquation('U', comp): the staged face terms (k_uface_int, k_uface_bnd) added into
// the cell's row in the reference's order -- convection over the cell's faces, the convection
// divergence, diffusion, explicit stress -- then grad(p), false transient, URF, scaled
// residual, DU.
__global__ void __launch_bounds__(kBlock) k_assemble_u(const SlotDesc* __restrict__ slots,
                                                       const int2* __restrict__ work, int comp, double* part) {
  __shared__ double sh[32];
  SLOT_BEGIN(work);
  const int e = idx;
  double rr = 0.0, rm = 0.0;
  if (e < m.Nc) {
    const FieldView& f = S.f;
    const double* ph = Uc(f, comp);
    const int s = m.cfStart[e], ne = m.cfStart[e + 1];
    const int r0 = m.rowptr[e];
    double* anb = S.anb;
    const size_t F = (size_t)m.F;
    const double* u = f.uft + (size_t)comp * UF_N * F;
    double acv = 0.0, bcv = 0.0, eff = 0.0;
    const int nf = ne - s;
    if (nf <= kCellFaces) {
      // The cell's face list, its side of each face (owner, neighbour, boundary) and its row of
      // off-diagonals are read or built once and kept in registers; the three passes below add
      // the same terms in the same order as the general loops after them.
      // side of face j in bits 2j..2j+1: 1 owner, 2 neighbour, 0 boundary
      int fcs[kCellFaces];
      unsigned sides = 0;
      double an[kCellFaces];
#pragma unroll
      for (int j = 0; j < kCellFaces; ++j)
        if (j < nf) {
          fcs[j] = m.cfFace[s + j];
          sides |= (fcs[j] < m.Fi ? (m.owner[fcs[j]] == e ? 1u : 2u) : 0u) << (2 * j);
        }
#define SIDE(j) ((sides >> (2 * (j))) & 3u)
      // (1) convection, sign +1
#pragma unroll
      for (int j = 0; j < kCellFaces; ++j)
        if (j < nf) {
          const int fc = fcs[j];
          const double psi = f.mdot[fc];
          const double T = u[UF_T * F + fc];
          if (SIDE(j) == 1u) {
            const double C2 = conv_c2(psi);
            acv = acv + conv_c1(psi); an[j] = 0.0 + C2; bcv = bcv - T; eff = eff + psi;
          } else if (SIDE(j) == 2u) {
            const double C2 = conv_c2(psi);
            acv = acv - C2; an[j] = 0.0 - conv_c1(psi); bcv = bcv + T; eff = eff - psi;
          } else {
            acv = acv + u[UF_C1 * F + fc]; bcv = bcv - T; eff = eff + psi;
          }
        }
      {  // cfdAssembleConvectionDivergenceTerm
        const double fce = dmax(eff, 0.0) - eff;
        const double fve = -dmax(eff, 0.0) * ph[e];
        const double fte = fce * ph[e] + fve;
        acv = acv + fce;
        bcv = bcv - fte;
      }
      // (2) diffusion, sign -1
#pragma unroll
      for (int j = 0; j < kCellFaces; ++j)
        if (j < nf) {
          const int fc = fcs[j];
          const double C1 = u[UF_D1 * F + fc], T = u[UF_TD * F + fc];
          if (SIDE(j) == 1u) {
            const double C2 = u[UF_D2 * F + fc];
            acv = acv + C1; an[j] = an[j] + C2; bcv = bcv - T;
          } else if (SIDE(j) == 2u) {
            const double C2 = u[UF_D2 * F + fc];
            acv = acv - C2; an[j] = an[j] - C1; bcv = bcv + T;
          } else {
            acv = acv + C1; bcv = bcv - T;
          }
        }
      // (3) explicit stress, sign -1
#pragma unroll
      for (int j = 0; j < kCellFaces; ++j)
        if (j < nf) {
          const double T = u[UF_TS * F + fcs[j]];
          if (SIDE(j) == 1u) { acv = acv + 0.0; an[j] = an[j] + 0.0; bcv = bcv - T; }
          else if (SIDE(j) == 2u) { acv = acv - 0.0; an[j] = an[j] - 0.0; bcv = bcv + T; }
          else { acv = acv + 0.0; bcv = bcv - T; }
        }
#pragma unroll
      for (int j = 0; j < kCellFaces; ++j)
        if (j < nf && SIDE(j) != 0u) anb[r0 + j] = an[j];
#undef SIDE
    } else {
      // (1) convection, sign +1
      for (int q = s; q < ne; ++q) {
        const int fc = m.cfFace[q];
        const double psi = f.mdot[fc];
        const double T = u[UF_T * F + fc];
        const double C1 = fc < m.Fi ? conv_c1(psi) : u[UF_C1 * F + fc];
        if (fc < m.Fi) {
          const double C2 = conv_c2(psi);
          if (m.owner[fc] == e) { acv = acv + C1; anb[r0 + q - s] = 0.0 + C2; bcv = bcv - T; eff = eff + psi; }
          else { acv = acv - C2; anb[r0 + q - s] = 0.0 - C1; bcv = bcv + T; eff = eff - psi; }
        } else {
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
      // (2) diffusion, sign -1
      for (int q = s; q < ne; ++q) {
        const int fc = m.cfFace[q];
        const double C1 = u[UF_D1 * F + fc], T = u[UF_TD * F + fc];
        if (fc < m.Fi) {
          const double C2 = u[UF_D2 * F + fc];
          const int k = r0 + q - s;
          if (m.owner[fc] == e) { acv = acv + C1; anb[k] = anb[k] + C2; bcv = bcv - T; }
          else { acv = acv - C2; anb[k] = anb[k] - C1; bcv = bcv + T; }
        } else {
          acv = acv + C1;
          bcv = bcv - T;
        }
      }
      // (3) explicit stress, sign -1
      for (int q = s; q < ne; ++q) {
        const int fc = m.cfFace[q];
        const double T = u[UF_TS * F + fc];
        if (fc < m.Fi) {
          const int k = r0 + q - s;
          if (m.owner[fc] == e) { acv = acv + 0.0; anb[k] = anb[k] + 0.0; bcv = bcv - T; }
          else { acv = acv - 0.0; anb[k] = anb[k] - 0.0; bcv = bcv + T; }
        } else {
          acv = acv + 0.0;
          bcv = bcv - T;
        }
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
      const double fce = (V * 1.0) / S.fdt;
      const double fte = fce * ph[e];
      acv = acv + fce;
      bcv = bcv - fte;
    }
    // (6) URF (cfdApplyURF.m:13-16)
    acv = acv / S.urf_u;
    S.ac[e] = acv;
    S.bc[e] = bcv;
    S.dphi[e] = 0.0;  // fresh coefficients (cfdSetupCoefficients.m:17)
    if (acv == 0.0) atomicExch(S.flags + FLAG_ZERO_DIAG, 1);
    // (7) scaled residual terms (cfdComputeNormalizedResidual.m:55-88)
    const double r = bcv / (acv * S.scal[SCAL_SCALE]);
    rr = r * r;
    rm = fabs(r);
    // (8) DU = V / ac (cfdPostAssembleEquation.m:37-42)
    DUc(f, comp)[e] = V / acv;
  }
  rr = block_reduce<0>(rr, sh);
  if (threadIdx.x == 0) part[2 * blockIdx.x] = rr;
  rm = block_reduce<1>(rm, sh);
  if (threadIdx.x == 0) part[2 * blockIdx.x + 1] = rm;
}

// cfdPostAssembleEquation.m:75-81 boundary rows of DU
__global__ void k_du_boundary(const SlotDesc* __restrict__ slots, const int2* __restrict__ work, int comp) {
  SLOT_BEGIN(work);
  if (idx >= m.Fb) return;
  double* d = DUc(S.f, comp);
  d[m.Nc + idx] = d[m.owner[m.Fi + idx]];
}

// ---------------------------------------------------------------- Rhie-Chow (cfdAssembleMdotTerm.m)
__global__ void __launch_bounds__(kBlock, 3) k_rhiechow(const SlotDesc* __restrict__ slots, const int2* __restrict__ work) {
  SLOT_BEGIN(work);
  const int fc = idx;
  if (fc >= m.F) return;
  const FieldView& f = S.f;
  const double S0 = m.Sx[fc], S1 = m.Sy[fc], S2 = m.Sz[fc];
  const double urfU = S.urf_u;
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
    const bool q4 = (S.quirks & UFVM_Q4_GRAD_WEIGHTS_SWAPPED) != 0;
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
    atomicExch(S.flags + FLAG_BAD_BC, 1);
  }
}

// cfdAssembleIntoGlobalMatrixFaceFluxes for the p equation + effective divergence residual
__global__ void __launch_bounds__(kBlock) k_assemble_p(const SlotDesc* __restrict__ slots,
                                                       const int2* __restrict__ work, double* part) {
  __shared__ double sh[32];
  SLOT_BEGIN(work);
  const int e = idx;
  double e2 = 0.0, em = -INFINITY;
  if (e < m.Nc) {
    const FieldView& f = S.f;
    const int s = m.cfStart[e], ne = m.cfStart[e + 1], r0 = m.rowptr[e];
    double acv = 0.0, bcv = 0.0, eff = 0.0;
    for (int q = s; q < ne; ++q) {
      const int fc = m.cfFace[q];
      const double md = f.mdot[fc];
      if (fc < m.Fi) {
        const double C1 = f.fC1[fc], C2 = f.fC2[fc];
        if (m.owner[fc] == e) { acv = acv + C1; S.anb[r0 + q - s] = 0.0 + C2; bcv = bcv - md; eff = eff + md; }
        else { acv = acv - C2; S.anb[r0 + q - s] = 0.0 - C1; bcv = bcv + md; eff = eff - md; }
      } else {
        const int p = m.bPatch[fc - m.Fi];
        const int ty = m.ptype[p];
        const double T = (ty == UFVM_PATCH_INLET || ty == UFVM_PATCH_OUTLET) ? md : 0.0;
        acv = acv + f.fC1[fc];
        bcv = bcv - T;
        eff = eff + md;
      }
    }
    S.ac[e] = acv;
    S.bc[e] = bcv;
    S.dphi[e] = 0.0;
    e2 = eff * eff;
    em = eff;
  }
  e2 = block_reduce<0>(e2, sh);
  if (threadIdx.x == 0) part[2 * blockIdx.x] = e2;
  em = block_reduce<1>(em, sh);
  if (threadIdx.x == 0) part[2 * blockIdx.x + 1] = em;
}

// ---------------------------------------------------------------- corrections
// cfdCorrectScalarEquation.m:16-109, interior part for U component comp
__global__ void k_correct_u_cells(const SlotDesc* __restrict__ slots, const int2* __restrict__ work, int comp) {
  SLOT_BEGIN(work);
  if (idx >= m.Nc) return;
  double* u = Uc(S.f, comp);
  u[idx] = u[idx] + S.dphi[idx];
}

__global__ void k_correct_u_bc(const SlotDesc* __restrict__ slots, const int2* __restrict__ work, int comp) {
  SLOT_BEGIN(work);
  const int k = idx;
  if (k >= m.Fb) return;
  const FieldView& f = S.f;
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
__global__ void k_pp_cells(const SlotDesc* __restrict__ slots, const int2* __restrict__ work) {
  SLOT_BEGIN(work);
  if (idx >= m.Nc) return;
  const double ppc = S.fixed >= 0 ? S.dphi[S.fixed] : 0.0;
  S.f.PP[idx] = S.dphi[idx] - ppc;
}

__global__ void k_pp_bc(const SlotDesc* __restrict__ slots, const int2* __restrict__ work) {
  SLOT_BEGIN(work);
  const int k = idx;
  if (k >= m.Fb) return;
  const int p = m.bPatch[k], ty = m.ptype[p], tp = m.bcP[p];
  const int b = m.Nc + k;
  if ((ty == UFVM_PATCH_INLET || ty == UFVM_PATCH_OUTLET) && tp == UFVM_BC_FIXED_VALUE) S.f.PP[b] = 0.0;
  else S.f.PP[b] = S.f.PP[m.owner[m.Fi + k]];
}

// cfdCorrectVelocityField.m:26-55 (interior)
__global__ void k_vel_cells(const SlotDesc* __restrict__ slots, const int2* __restrict__ work) {
  SLOT_BEGIN(work);
  const int e = idx;
  if (e >= m.Nc) return;
  const FieldView& f = S.f;
  f.U0[e] = f.U0[e] - f.DU0[e] * f.gPP0[e];
  f.U1[e] = f.U1[e] - f.DU1[e] * f.gPP1[e];
  f.U2[e] = f.U2[e] - f.DU2[e] * f.gPP2[e];
}

// velocity boundary correction of patch index `ip` of every slot (patch order matters:
// the reference loops over patches sequentially and a later patch overwrites rows an
// earlier one wrote). mode 1: tangential (symmetry, empty, slip); mode 2: gather owner
// velocity of an outlet with fixed p; mode 3: scatter it to its rows (Q12: face-indexed).
__global__ void k_vel_patch(const SlotDesc* __restrict__ slots, const int2* __restrict__ work, int ip, int mode) {
  SLOT_BEGIN(work);
  const int k = idx;
  if (k >= m.Fb || m.bPatch[k] != ip) return;
  const FieldView& f = S.f;
  const int ty = m.ptype[ip], tp = m.bcP[ip];
  const int fc = m.Fi + k, o = m.owner[fc];
  const bool outlet_fixed = ty == UFVM_PATCH_OUTLET && tp == UFVM_BC_FIXED_VALUE;
  if (mode == 1) {
    if (ty == UFVM_PATCH_SYMMETRY || ty == UFVM_PATCH_EMPTY || (ty == UFVM_PATCH_WALL && tp == UFVM_BC_SLIP))
      tangential(m, f, fc, m.Nc + k, o, 0, 2);
  } else if (mode == 2) {
    if (!outlet_fixed) return;
    f.tmp3[3 * k] = f.U0[o]; f.tmp3[3 * k + 1] = f.U1[o]; f.tmp3[3 * k + 2] = f.U2[o];
  } else {
    if (!outlet_fixed) return;
    const int row = (S.quirks & UFVM_Q12_OUTLET_U_FACE_ROWS) ? fc : m.Nc + k;
    f.U0[row] = f.tmp3[3 * k]; f.U1[row] = f.tmp3[3 * k + 1]; f.U2[row] = f.tmp3[3 * k + 2];
  }
}

// cfdCorrectPressureEquation.m:22-54
__global__ void k_p_cells(const SlotDesc* __restrict__ slots, const int2* __restrict__ work) {
  SLOT_BEGIN(work);
  const int e = idx;
  if (e >= m.Nc) return;
  const FieldView& f = S.f;
  const double ppf = S.fixed >= 0 ? f.PP[S.fixed] : 0.0;
  f.p[e] = f.p[e] + S.urf_p * (f.PP[e] - ppf);
}

__global__ void k_p_bc(const SlotDesc* __restrict__ slots, const int2* __restrict__ work) {
  SLOT_BEGIN(work);
  const int k = idx;
  if (k >= m.Fb) return;
  const int p = m.bPatch[k], ty = m.ptype[p], tp = m.bcP[p];
  if ((ty == UFVM_PATCH_INLET || ty == UFVM_PATCH_OUTLET) && tp == UFVM_BC_FIXED_VALUE) return;
  S.f.p[m.Nc + k] = S.f.p[m.owner[m.Fi + k]];
}

// cfdCorrectMdotField.m:24-50 + boundary patches
__global__ void k_mdot_correct(const SlotDesc* __restrict__ slots, const int2* __restrict__ work) {
  SLOT_BEGIN(work);
  const int fc = idx;
  if (fc >= m.F) return;
  const FieldView& f = S.f;
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

// ================================================================ stages
int stage_init(const BatchLaunch& b, bool compute_mdot) {
  k_bc_init<<<b.nwb, kBlock, 0, b.st>>>(b.slots, b.wb);
  UFVM_LAUNCH_CHECK();
  UFVM_CHECK(gradient<G_U>(b));
  UFVM_CHECK(gradient<G_P>(b));
  if (compute_mdot) {
    k_mdot_init<<<b.nwf, kBlock, 0, b.st>>>(b.slots, b.wf);
    UFVM_LAUNCH_CHECK();
  }
  return UFVM_OK;
}

int stage_update_fields(const BatchLaunch& b) {
  k_bc_update<<<b.nwb, kBlock, 0, b.st>>>(b.slots, b.wb);
  UFVM_LAUNCH_CHECK();
  UFVM_CHECK(gradient<G_U>(b));
  k_minmax_U<<<b.nwu, kBlock, 0, b.st>>>(b.slots, b.wu, b.part);
  k_slot_final<1><<<b.nslots, 1024, 0, b.st>>>(b.slots, b.ustart, b.uend, b.part);
  UFVM_LAUNCH_CHECK();
  return gradient<G_P>(b);
}

int stage_uface_interior(const BatchLaunch& b) {
  k_uface_int<<<b.nwf, kBlock, 0, b.st>>>(b.slots, b.wf, 0, 2);
  UFVM_LAUNCH_CHECK();
  return UFVM_OK;
}

int stage_assemble_u(const BatchLaunch& b, int comp, bool interior_ready) {
  if (!interior_ready) k_uface_int<<<b.nwf, kBlock, 0, b.st>>>(b.slots, b.wf, comp, comp);
  k_uface_bnd<<<b.nwb, kBlock, 0, b.st>>>(b.slots, b.wb, comp);
  k_assemble_u<<<b.nwc, kBlock, 0, b.st>>>(b.slots, b.wc, comp, b.part);
  k_du_boundary<<<b.nwb, kBlock, 0, b.st>>>(b.slots, b.wb, comp);
  k_slot_final<0><<<b.nslots, 1024, 0, b.st>>>(b.slots, b.cstart, b.cend, b.part);
  UFVM_LAUNCH_CHECK();
  return UFVM_OK;
}

int stage_assemble_p(const BatchLaunch& b) {
  k_rhiechow<<<b.nwf, kBlock, 0, b.st>>>(b.slots, b.wf);
  k_assemble_p<<<b.nwc, kBlock, 0, b.st>>>(b.slots, b.wc, b.part);
  k_slot_final<2><<<b.nslots, 1024, 0, b.st>>>(b.slots, b.cstart, b.cend, b.part);
  UFVM_LAUNCH_CHECK();
  return UFVM_OK;
}

int stage_correct_u(const BatchLaunch& b, int comp) {
  k_correct_u_cells<<<b.nwc, kBlock, 0, b.st>>>(b.slots, b.wc, comp);
  k_correct_u_bc<<<b.nwb, kBlock, 0, b.st>>>(b.slots, b.wb, comp);
  UFVM_LAUNCH_CHECK();
  return UFVM_OK;
}

int stage_correct_p(const BatchLaunch& b, int max_patches, double*) {
  k_pp_cells<<<b.nwc, kBlock, 0, b.st>>>(b.slots, b.wc);
  k_pp_bc<<<b.nwb, kBlock, 0, b.st>>>(b.slots, b.wb);
  UFVM_LAUNCH_CHECK();
  UFVM_CHECK(gradient<G_PP>(b));
  k_vel_cells<<<b.nwc, kBlock, 0, b.st>>>(b.slots, b.wc);
  for (int ip = 0; ip < max_patches; ++ip)
    for (int mode : {2, 3, 1})
      if (!b.vel_mask || b.vel_mask[3 * ip + mode - 1])
        k_vel_patch<<<b.nwb, kBlock, 0, b.st>>>(b.slots, b.wb, ip, mode);
  UFVM_LAUNCH_CHECK();
  k_p_cells<<<b.nwc, kBlock, 0, b.st>>>(b.slots, b.wc);
  k_p_bc<<<b.nwb, kBlock, 0, b.st>>>(b.slots, b.wb);
  k_mdot_correct<<<b.nwf, kBlock, 0, b.st>>>(b.slots, b.wf);
  UFVM_LAUNCH_CHECK();
  return UFVM_OK;
}

}  // namespace ufvm
