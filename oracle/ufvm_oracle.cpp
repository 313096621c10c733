// ufvm_oracle.cpp -- TEST INFRASTRUCTURE ONLY (see ufvm_oracle.h).
//
// Single-thread FP64 restatement of the reference's steady SIMPLE path. Each routine
// names the MATLAB file:line it follows (paths relative to uFVM/src/). Indices are
// 0-based here; the MATLAB code is 1-based. Build with -ffp-contract=off.
#include "ufvm_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace {

using std::vector;

inline double dot3(const double* a, const double* b) { return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]; }
inline double mag3(const double* a) { return std::sqrt(dot3(a, a)); }

struct PatchI {
  int type, start, n;  // start = first face (0-based, global face index)
};

struct Mesh {
  int Nc = 0, F = 0, Fi = 0, Fb = 0, nP = 0, quirks = 0;
  vector<double> pts;
  vector<int> fstart, fnodes, owner, neigh;
  vector<PatchI> patches;
  vector<double> fC, Sf, area, CN, eCN, gDiff, T, gf, walldist, vol, cC;
  vector<int> cfStart, cfFaces;  // element iFaces (interior in face order, then boundary)
  vector<signed char> cfSign;
  vector<int> rowptr, col;       // cconn (iNeighbours) as CSR
  vector<int> ownSlot, neiSlot;  // iOwnerNeighbourCoef-1 / iNeighbourOwnerCoef-1 as CSR positions
};

// utilities/IO/cfdReadPolyMesh.m:153-181 (element face/neighbour lists) and
// utilities/IO/cfdProcessOpenFoamMesh.m:15-172 (geometry).
void process_mesh(Mesh& m) {
  const int F = m.F, Fi = m.Fi, Nc = m.Nc;
  // element connectivity (cfdReadPolyMesh.m:153-181)
  vector<vector<int>> ifaces(Nc), inb(Nc);
  vector<vector<signed char>> fsign(Nc);
  for (int f = 0; f < Fi; ++f) {
    int o = m.owner[f], n = m.neigh[f];
    ifaces[o].push_back(f); fsign[o].push_back(1); inb[o].push_back(n);
    ifaces[n].push_back(f); fsign[n].push_back(-1); inb[n].push_back(o);
  }
  for (int f = Fi; f < F; ++f) {
    int o = m.owner[f];
    ifaces[o].push_back(f); fsign[o].push_back(1);
  }
  m.cfStart.assign(Nc + 1, 0);
  m.rowptr.assign(Nc + 1, 0);
  for (int e = 0; e < Nc; ++e) {
    m.cfStart[e + 1] = m.cfStart[e] + (int)ifaces[e].size();
    m.rowptr[e + 1] = m.rowptr[e] + (int)inb[e].size();
  }
  m.cfFaces.clear(); m.cfSign.clear(); m.col.clear();
  for (int e = 0; e < Nc; ++e) {
    m.cfFaces.insert(m.cfFaces.end(), ifaces[e].begin(), ifaces[e].end());
    m.cfSign.insert(m.cfSign.end(), fsign[e].begin(), fsign[e].end());
    m.col.insert(m.col.end(), inb[e].begin(), inb[e].end());
  }
  // face geometry (cfdProcessOpenFoamMesh.m:21-56)
  m.fC.assign(3 * F, 0); m.Sf.assign(3 * F, 0); m.area.assign(F, 0);
  for (int f = 0; f < F; ++f) {
    const int s = m.fstart[f], nn = m.fstart[f + 1] - s;
    double centre[3] = {0, 0, 0};
    for (int q = 0; q < nn; ++q) {
      const double* p = &m.pts[3 * m.fnodes[s + q]];
      for (int k = 0; k < 3; ++k) centre[k] = centre[k] + p[k];
    }
    for (int k = 0; k < 3; ++k) centre[k] = centre[k] / nn;
    double cen[3] = {0, 0, 0}, S[3] = {0, 0, 0}, A = 0;
    for (int t = 0; t < nn; ++t) {
      const double* p1 = centre;
      const double* p2 = &m.pts[3 * m.fnodes[s + t]];
      const double* p3 = &m.pts[3 * m.fnodes[s + (t + 1 < nn ? t + 1 : 0)]];
      double lc[3], a[3], b[3], ls[3];
      for (int k = 0; k < 3; ++k) lc[k] = ((p1[k] + p2[k]) + p3[k]) / 3;
      for (int k = 0; k < 3; ++k) { a[k] = p2[k] - p1[k]; b[k] = p3[k] - p1[k]; }
      // MATLAB cross: [a2 b3 - a3 b2; a3 b1 - a1 b3; a1 b2 - a2 b1]
      ls[0] = 0.5 * (a[1] * b[2] - a[2] * b[1]);
      ls[1] = 0.5 * (a[2] * b[0] - a[0] * b[2]);
      ls[2] = 0.5 * (a[0] * b[1] - a[1] * b[0]);
      double la = mag3(ls);
      for (int k = 0; k < 3; ++k) cen[k] = cen[k] + la * lc[k];
      for (int k = 0; k < 3; ++k) S[k] = S[k] + ls[k];
      A = A + la;
    }
    for (int k = 0; k < 3; ++k) m.fC[3 * f + k] = cen[k] / A;
    for (int k = 0; k < 3; ++k) m.Sf[3 * f + k] = S[k];
    m.area[f] = A;
  }
  // element volume and centroid (cfdProcessOpenFoamMesh.m:60-104), Q5 rough centre
  m.vol.assign(Nc, 0); m.cC.assign(3 * Nc, 0);
  const bool q5 = (m.quirks & ORQ_Q5_ROUGH_CENTRE) != 0;
  for (int e = 0; e < Nc; ++e) {
    const int s = m.cfStart[e], nf = m.cfStart[e + 1] - s;
    double centre[3] = {0, 0, 0};
    for (int q = 0; q < nf; ++q) {
      const int f = q5 ? q : m.cfFaces[s + q];  // Q5: global faces 1..nf
      for (int k = 0; k < 3; ++k) centre[k] = centre[k] + m.fC[3 * f + k];
    }
    for (int k = 0; k < 3; ++k) centre[k] = centre[k] / nf;
    double svc[3] = {0, 0, 0}, sv = 0;
    for (int q = 0; q < nf; ++q) {
      const int f = m.cfFaces[s + q];
      const double sg = m.cfSign[s + q];
      double S[3], Cf[3], lc[3];
      for (int k = 0; k < 3; ++k) S[k] = m.Sf[3 * f + k] * sg;
      for (int k = 0; k < 3; ++k) Cf[k] = m.fC[3 * f + k] - centre[k];
      double lv = dot3(S, Cf) / 3;
      for (int k = 0; k < 3; ++k) lc[k] = 0.75 * m.fC[3 * f + k] + 0.25 * centre[k];
      for (int k = 0; k < 3; ++k) svc[k] = svc[k] + lc[k] * lv;
      sv = sv + lv;
    }
    for (int k = 0; k < 3; ++k) m.cC[3 * e + k] = svc[k] / sv;
    m.vol[e] = sv;
  }
  // secondary face geometry (cfdProcessOpenFoamMesh.m:108-155)
  m.CN.assign(3 * F, 0); m.eCN.assign(3 * F, 0); m.gDiff.assign(F, 0); m.T.assign(3 * F, 0);
  m.gf.assign(F, 0); m.walldist.assign(F, 0);
  for (int f = 0; f < Fi; ++f) {
    const double A = m.area[f];
    double nf[3], CN[3], e[3], E[3], Cf[3], fF[3];
    for (int k = 0; k < 3; ++k) nf[k] = m.Sf[3 * f + k] / A;
    const double* c1 = &m.cC[3 * m.owner[f]];
    const double* c2 = &m.cC[3 * m.neigh[f]];
    for (int k = 0; k < 3; ++k) CN[k] = c2[k] - c1[k];
    double mcn = mag3(CN);
    for (int k = 0; k < 3; ++k) e[k] = CN[k] / mcn;
    for (int k = 0; k < 3; ++k) E[k] = A * e[k];
    m.gDiff[f] = mag3(E) / mag3(CN);
    for (int k = 0; k < 3; ++k) {
      m.CN[3 * f + k] = CN[k]; m.eCN[3 * f + k] = e[k]; m.T[3 * f + k] = m.Sf[3 * f + k] - E[k];
      Cf[k] = m.fC[3 * f + k] - c1[k]; fF[k] = c2[k] - m.fC[3 * f + k];
    }
    m.gf[f] = dot3(Cf, nf) / (dot3(Cf, nf) + dot3(fF, nf));
    m.walldist[f] = 0;
  }
  for (int f = Fi; f < F; ++f) {
    const double A = m.area[f];
    const double* S = &m.Sf[3 * f];
    const double* c1 = &m.cC[3 * m.owner[f]];
    double CN[3], e[3], E[3];
    for (int k = 0; k < 3; ++k) CN[k] = m.fC[3 * f + k] - c1[k];
    m.gDiff[f] = (A * A) / dot3(CN, S);
    double mcn = mag3(CN);
    for (int k = 0; k < 3; ++k) e[k] = CN[k] / mcn;
    for (int k = 0; k < 3; ++k) E[k] = A * e[k];
    for (int k = 0; k < 3; ++k) { m.CN[3 * f + k] = CN[k]; m.eCN[3 * f + k] = e[k]; m.T[3 * f + k] = S[k] - E[k]; }
    m.gf[f] = 1;
    m.walldist[f] = dot3(CN, S) / mag3(S);
  }
  // coefficient slots (cfdProcessOpenFoamMesh.m:158-172)
  m.ownSlot.assign(Fi, -1); m.neiSlot.assign(Fi, -1);
  for (int e = 0; e < Nc; ++e) {
    const int s = m.cfStart[e], nl = m.rowptr[e + 1] - m.rowptr[e];
    for (int q = 0; q < nl; ++q) {
      const int f = m.cfFaces[s + q];
      if (m.owner[f] == e) m.ownSlot[f] = m.rowptr[e] + q;
      else if (m.neigh[f] == e) m.neiSlot[f] = m.rowptr[e] + q;
    }
  }
}

// ----------------------------------------------------------------------------------
// Linear algebra on the cconn-ordered CSR (setup/cfdSetupCoefficients.m:7-39 layout)

// compute/cfdComputeResidualsArray.m:9-17
void residuals(int n, const int* rp, const int* col, const double* ac, const double* anb,
               const double* bc, const double* x, double* r) {
  for (int i = 0; i < n; ++i) {
    double v = bc[i] - ac[i] * x[i];
    for (int k = rp[i]; k < rp[i + 1]; ++k) v = v - anb[k] * x[col[k]];
    r[i] = v;
  }
}

double sum_abs_res(int n, const int* rp, const int* col, const double* ac, const double* anb,
                   const double* bc, const double* x) {
  double s = 0;
  for (int i = 0; i < n; ++i) {
    double v = bc[i] - ac[i] * x[i];
    for (int k = rp[i]; k < rp[i + 1]; ++k) v = v - anb[k] * x[col[k]];
    s = s + std::fabs(v);
  }
  return s;
}

inline double gs_row(int i, const int* rp, const int* col, const double* ac, const double* anb,
                     const double* bc, const double* x) {
  double v = bc[i];
  for (int k = rp[i]; k < rp[i + 1]; ++k) v = v - anb[k] * x[col[k]];
  return v / ac[i];
}

// solve/cfdSolveSOR.m:13-29 (symmetric Gauss-Seidel, natural order)
void sor_sweep(int n, const int* rp, const int* col, const double* ac, const double* anb,
               const double* bc, double* x) {
  for (int i = 0; i < n; ++i) x[i] = gs_row(i, rp, col, ac, anb, bc, x);
  for (int i = n - 1; i >= 0; --i) x[i] = gs_row(i, rp, col, ac, anb, bc, x);
}

// Multicolour symmetric Gauss-Seidel: colours ascending then descending. Within a
// colour no two rows are adjacent, so the row order inside a colour is immaterial.
void mcgs_sweep(int n, const int* rp, const int* col, const double* ac, const double* anb,
                const double* bc, const int* color, int ncolor, double* x) {
  for (int c = 0; c < ncolor; ++c)
    for (int i = 0; i < n; ++i)
      if (color[i] == c) x[i] = gs_row(i, rp, col, ac, anb, bc, x);
  for (int c = ncolor - 1; c >= 0; --c)
    for (int i = 0; i < n; ++i)
      if (color[i] == c) x[i] = gs_row(i, rp, col, ac, anb, bc, x);
}

inline int find_pos(const int* rp, const int* col, int row, int target) {
  for (int k = rp[row]; k < rp[row + 1]; ++k)
    if (col[k] == target) return k;
  return -1;
}

// solve/cfdFactorizeILU.m:5-47 (DILU; Q7 skips row N-1 in 1-based numbering)
void ilu_factor(int n, const int* rp, const int* col, const double* ac, const double* anb,
                double* dc, int quirks) {
  for (int i = 0; i < n; ++i) dc[i] = ac[i];
  const bool q7 = (quirks & ORQ_Q7_ILU_SKIP_ROW) != 0;
  for (int i = 0; i < n; ++i) {
    dc[i] = 1.0 / dc[i];
    if (q7 && i == n - 2) continue;
    for (int k = rp[i]; k < rp[i + 1]; ++k) {
      const int j = col[k];
      if (j > i) {
        const int p = find_pos(rp, col, j, i);
        dc[j] = dc[j] - anb[p] * dc[i] * anb[k];
      }
    }
  }
}

// solve/cfdSolveILU.m:18-93
void ilu_sweep(int n, const int* rp, const int* col, const double* ac, const double* anb,
               const double* bc, const double* dc, double* x, vector<double>& rc) {
  rc.resize(n);
  for (int i = 0; i < n; ++i) {
    double res = -ac[i] * x[i] + bc[i];
    for (int k = rp[i]; k < rp[i + 1]; ++k) res = res - anb[k] * x[col[k]];
    rc[i] = res;
  }
  for (int i = 0; i < n; ++i) {
    const double mat1 = dc[i] * rc[i];
    for (int k = rp[i]; k < rp[i + 1]; ++k) {
      const int j = col[k];
      if (j > i) {
        const int p = find_pos(rp, col, j, i);
        const double mat2 = anb[p] * mat1;
        rc[j] = rc[j] - mat2;
      }
    }
  }
  for (int i = n - 1; i >= 0; --i) {
    if (i < n - 1) {
      for (int k = rp[i]; k < rp[i + 1]; ++k) {
        const int j = col[k];
        if (j > i) rc[i] = rc[i] - anb[k] * rc[j];
      }
    }
    const double mat1 = dc[i] * rc[i];
    rc[i] = mat1;
    x[i] = x[i] + mat1;
  }
}

// Greedy first-fit colouring in natural order: row i takes the smallest colour not used by
// its lower-index neighbours (2 colours on the structured 2D / 3D cavities).
int coloring(int n, const int* rp, const int* col, int* color) {
  int ncolor = 0;
  std::vector<char> used;
  for (int i = 0; i < n; ++i) {
    used.assign(rp[i + 1] - rp[i] + 2, 0);
    for (int k = rp[i]; k < rp[i + 1]; ++k) {
      const int j = col[k];
      if (j < i && color[j] < (int)used.size()) used[color[j]] = 1;
    }
    int c = 0;
    while (used[c]) ++c;
    color[i] = c;
    ncolor = std::max(ncolor, c + 1);
  }
  return ncolor;
}

struct Level {
  int n = 0;
  vector<int> rp, col, parents;
  vector<double> ac, anb, bc, dphi;
  vector<int> color;
  int ncolor = 0;
};

// solve/cfdSolveAlgebraicSystem.m:11-66
void solve_algebraic_system(Level& L, int smoother, int nIter, double rrf, int quirks,
                            double* r0out, double* r1out, int* iters) {
  const int n = L.n;
  const double r0 = sum_abs_res(n, L.rp.data(), L.col.data(), L.ac.data(), L.anb.data(), L.bc.data(), L.dphi.data()) / n;
  double r1 = r0;
  int it = 1;
  if (smoother == ORS_ILU) {
    vector<double> dc(n), rc;
    ilu_factor(n, L.rp.data(), L.col.data(), L.ac.data(), L.anb.data(), dc.data(), quirks);
    while (it <= nIter && r1 > rrf * r0) {
      ilu_sweep(n, L.rp.data(), L.col.data(), L.ac.data(), L.anb.data(), L.bc.data(), dc.data(), L.dphi.data(), rc);
      r1 = sum_abs_res(n, L.rp.data(), L.col.data(), L.ac.data(), L.anb.data(), L.bc.data(), L.dphi.data()) / n;
      ++it;
    }
  } else {
    while (it <= nIter && r1 > rrf * r0) {
      if (smoother == ORS_SOR)
        sor_sweep(n, L.rp.data(), L.col.data(), L.ac.data(), L.anb.data(), L.bc.data(), L.dphi.data());
      else
        mcgs_sweep(n, L.rp.data(), L.col.data(), L.ac.data(), L.anb.data(), L.bc.data(), L.color.data(), L.ncolor, L.dphi.data());
      r1 = sum_abs_res(n, L.rp.data(), L.col.data(), L.ac.data(), L.anb.data(), L.bc.data(), L.dphi.data()) / n;
      ++it;
    }
  }
  if (r0out) *r0out = r0;
  if (r1out) *r1out = r1;
  if (iters) *iters = it - 1;
}

// solve/AMG/cfdAgglomerateLevel.m:13-105 + assemble/assembleAgglomeratedLHS.m:16-30
int agglomerate(const Level& fine, vector<int>& parents, Level& coarse) {
  const int n = fine.n;
  const int* rp = fine.rp.data();
  const int* col = fine.col.data();
  const double* anb = fine.anb.data();
  parents.assign(n, -1);
  vector<double> maxAnb(n);
  for (int i = 0; i < n; ++i) {
    double m = -INFINITY;
    for (int k = rp[i]; k < rp[i + 1]; ++k) m = std::max(m, -anb[k]);
    maxAnb[i] = m;
  }
  int iParent = 0;
  vector<int> children, children2;
  for (int seed = 0; seed < n; ++seed) {
    if (parents[seed] != -1) continue;
    parents[seed] = iParent;
    children.assign(1, seed);
    for (int k = rp[seed]; k < rp[seed + 1]; ++k) {
      const int nb = col[k];
      if (parents[nb] == -1 && (-anb[k] / maxAnb[seed]) > 0.5) {
        parents[nb] = iParent;
        children.push_back(nb);
      }
    }
    children2.clear();
    for (size_t c = 1; c < children.size(); ++c) {
      const int ch = children[c];
      for (int k = rp[ch]; k < rp[ch + 1]; ++k) {
        const int nb = col[k];
        if (parents[nb] == -1 && (-anb[k] / maxAnb[ch]) > 0.5) {
          parents[nb] = iParent;
          children2.push_back(nb);
        }
      }
    }
    if (children.size() + children2.size() == 1) parents[seed] = -1;
    else ++iParent;
  }
  for (int o = 0; o < n; ++o) {
    if (parents[o] == -1) {
      double strength = 0;
      for (int k = rp[o]; k < rp[o + 1]; ++k) {
        const int nb = col[k];
        if (parents[nb] != -1) {
          const double s = -anb[k] / maxAnb[nb];
          if (strength < s) { strength = s; parents[o] = parents[nb]; }
        }
      }
    }
    if (parents[o] == -1) parents[o] = iParent++;
  }
  const int nc = iParent;
  // coarse connectivity in discovery order (cfdAgglomerateLevel.m:89-98)
  vector<vector<int>> cc(nc);
  for (int i = 0; i < n; ++i)
    for (int k = rp[i]; k < rp[i + 1]; ++k) {
      const int P = parents[i], Q = parents[col[k]];
      if (P != Q && std::find(cc[P].begin(), cc[P].end(), Q) == cc[P].end()) cc[P].push_back(Q);
    }
  coarse.n = nc;
  coarse.rp.assign(nc + 1, 0);
  for (int P = 0; P < nc; ++P) coarse.rp[P + 1] = coarse.rp[P] + (int)cc[P].size();
  coarse.col.clear();
  for (int P = 0; P < nc; ++P) coarse.col.insert(coarse.col.end(), cc[P].begin(), cc[P].end());
  coarse.ac.assign(nc, 0); coarse.anb.assign(coarse.col.size(), 0);
  coarse.bc.assign(nc, 0); coarse.dphi.assign(nc, 0);
  // Galerkin-by-summation (assembleAgglomeratedLHS.m:16-30)
  for (int i = 0; i < n; ++i) {
    const int P = parents[i];
    coarse.ac[P] = coarse.ac[P] + fine.ac[i];
    for (int k = rp[i]; k < rp[i + 1]; ++k) {
      const int Q = parents[col[k]];
      if (Q == P) coarse.ac[P] = coarse.ac[P] + anb[k];
      else {
        const int pos = find_pos(coarse.rp.data(), coarse.col.data(), P, Q);
        coarse.anb[pos] = coarse.anb[pos] + anb[k];
      }
    }
  }
  return nc;
}

// ----------------------------------------------------------------------------------
struct Case {
  Mesh* m = nullptr;
  int nCorr = 1, fixedEl = -1, cycle = ORC_W, maxCycles = 30, maxCoarse = 10, pre = 1, post = 3;
  int pSmoother = ORS_ILU, uSmoother = ORS_ILU, uNIter = 10, quirks = ORQ_ALL, pAMG = 1;
  double nu = 0, urfU = 0.7, urfP = 0.3, tolU = 1e-6, tolP = 1e-6, pRrf = 0.1, uRrf = 0.1, fdt = 1e9;
  vector<int> bcU, bcP;          // per patch
  vector<double> valU, valP;     // per boundary face
  // fields
  vector<double> U[3];           // rows: Nc+Fb (may grow under Q12)
  vector<double> gradU[3][3];    // [component][direction][row]
  vector<double> p, gradp[3], PP, gradPP[3], DU[3], mdot, gammaU, nuF, rho;
  vector<double> fluxC1, fluxC2;
  double scaleU = 1;
  // coefficients / hierarchy
  vector<Level> lev;
  int maxLevels = 1;
  vector<double> acOld;
};

inline bool q(const Case& c, int bit) { return (c.quirks & bit) != 0; }

// update/cfdUpdateGradient.m:11-255 via compute/cfdComputeGradientGauss0.m:28-80.
// phi: ncomp column vectors; grad[c][d] sized Nc+Fb.
void update_gradient(Case& C, vector<double>* phi, int ncomp, vector<double> (*grad)[3]) {
  Mesh& m = *C.m;
  const int Nc = m.Nc, Fi = m.Fi, F = m.F, Fb = m.Fb;
  const bool q1 = q(C, ORQ_Q1_VEC_BOUNDARY_COMPONENT);
  for (int c = 0; c < ncomp; ++c)
    for (int d = 0; d < 3; ++d) grad[c][d].assign(Nc + Fb, 0.0);
  for (int c = 0; c < ncomp; ++c) {
    const double* ph = phi[c].data();
    for (int f = 0; f < Fi; ++f) {
      const int o = m.owner[f], n = m.neigh[f];
      const double g = m.gf[f];
      const double phf = g * ph[n] + (1 - g) * ph[o];
      for (int d = 0; d < 3; ++d) {
        grad[c][d][o] = grad[c][d][o] + phf * m.Sf[3 * f + d];
        grad[c][d][n] = grad[c][d][n] - phf * m.Sf[3 * f + d];
      }
    }
  }
  for (int c = 0; c < ncomp; ++c) {
    // Q1: phi_b(k) is a linear index into the (Fb x ncomp) block -> component 1
    const double* ph = phi[q1 ? 0 : c].data();
    for (int k = 0; k < Fb; ++k) {
      const int f = Fi + k, o = m.owner[f];
      for (int d = 0; d < 3; ++d) grad[c][d][o] = grad[c][d][o] + ph[Nc + k] * m.Sf[3 * f + d];
    }
  }
  for (int c = 0; c < ncomp; ++c)
    for (int e = 0; e < Nc; ++e)
      for (int d = 0; d < 3; ++d) grad[c][d][e] = grad[c][d][e] / m.vol[e];
  for (int c = 0; c < ncomp; ++c)
    for (int k = 0; k < Fb; ++k)
      for (int d = 0; d < 3; ++d) grad[c][d][Nc + k] = grad[c][d][m.owner[Fi + k]];
  // boundary-gradient fix: wall, inlet, outlet (cfdUpdateGradient.m:81-255)
  for (const PatchI& P : m.patches) {
    if (P.type != ORP_WALL && P.type != ORP_INLET && P.type != ORP_OUTLET) continue;
    const bool comp1 = q1 && P.type != ORP_WALL;  // inlet/outlet read phi(iBElement) linearly
    for (int c = 0; c < ncomp; ++c) {
      for (int j = 0; j < P.n; ++j) {
        const int f = P.start + j, o = m.owner[f], b = Nc + (f - Fi);
        const double* dv = &m.CN[3 * f];  // face centroid - owner centroid
        const double dmag = mag3(dv);
        double e[3];
        for (int d = 0; d < 3; ++d) e[d] = dv[d] / dmag;
        double go[3] = {grad[c][0][o], grad[c][1][o], grad[c][2][o]};
        const double ge = dot3(go, e);
        const int pc = comp1 ? 0 : c;
        const double sn = (phi[pc][b] - phi[pc][o]) / dmag;
        for (int d = 0; d < 3; ++d) grad[c][d][b] = (go[d] - ge * e[d]) + sn * e[d];
      }
    }
  }
  (void)F;
}

// update/cfdUpdateBoundaryConditions.m:13-96 (per-iteration update; fixed values only)
void update_bcs_U(Case& C) {
  Mesh& m = *C.m;
  for (size_t ip = 0; ip < m.patches.size(); ++ip) {
    const PatchI& P = m.patches[ip];
    const int t = C.bcU[ip];
    bool set = false;
    if (P.type == ORP_WALL && (t == ORB_FIXED_VALUE || t == ORB_NOSLIP)) set = true;
    if ((P.type == ORP_INLET || P.type == ORP_OUTLET) && t == ORB_FIXED_VALUE) set = true;
    if (!set) continue;
    for (int j = 0; j < P.n; ++j) {
      const int k = P.start + j - m.Fi;
      for (int c = 0; c < 3; ++c) C.U[c][m.Nc + k] = C.valU[3 * k + c];
    }
  }
}

void update_bcs_p(Case& C) {
  Mesh& m = *C.m;
  for (size_t ip = 0; ip < m.patches.size(); ++ip) {
    const PatchI& P = m.patches[ip];
    const int t = C.bcP[ip];
    bool set = false;
    if (P.type == ORP_WALL && t == ORB_FIXED_VALUE) set = true;
    if ((P.type == ORP_INLET || P.type == ORP_OUTLET) && t == ORB_FIXED_VALUE) set = true;
    if (!set) continue;
    for (int j = 0; j < P.n; ++j) {
      const int k = P.start + j - m.Fi;
      C.p[m.Nc + k] = C.valP[k];
    }
  }
}

// update/cfdUpdateTermCoefficientField.m:44-70: gamma_Ueq = Average(nu) on all faces
void update_gamma(Case& C) {
  Mesh& m = *C.m;
  C.gammaU.assign(m.F, 0);
  for (int f = 0; f < m.Fi; ++f) {
    const double g = m.gf[f];
    C.gammaU[f] = g * C.nuF[m.neigh[f]] + (1 - g) * C.nuF[m.owner[f]];
  }
  for (int f = m.Fi; f < m.F; ++f) C.gammaU[f] = C.nuF[m.Nc + f - m.Fi];
}

// update/cfdUpdateScale.m:15-28 over every row of U (including Q12 extension rows)
void update_scale(Case& C) {
  double mx = -INFINITY, mn = INFINITY;
  for (int c = 0; c < 3; ++c)
    for (double v : C.U[c]) { mx = std::max(mx, v); mn = std::min(mn, v); }
  double s = std::max(mx - mn, std::fabs(mx));
  if (s < 1e-6) s = 1;
  C.scaleU = s;
}

// update/cfdUpdateFields.m:17-27 -> cfdUpdateEquations.m:14-24 (U then p)
void update_fields(Case& C) {
  update_bcs_U(C);
  update_gradient(C, C.U, 3, C.gradU);
  update_gamma(C);
  update_scale(C);
  update_bcs_p(C);
  vector<double> (*gp)[3] = reinterpret_cast<vector<double> (*)[3]>(&C.gradp);
  update_gradient(C, &C.p, 1, gp);
}

void fresh_coefficients(Case& C) {
  Mesh& m = *C.m;
  if (C.lev.empty()) C.lev.resize(1);
  Level& L = C.lev[0];
  L.n = m.Nc; L.rp = m.rowptr; L.col = m.col;
  L.ac.assign(m.Nc, 0); L.bc.assign(m.Nc, 0); L.anb.assign(m.col.size(), 0); L.dphi.assign(m.Nc, 0);
  C.acOld.assign(m.Nc, 0);
}

// assemble/cfdAssembleIntoGlobalMatrixFaceFluxes.m:25-55
void scatter_faces(Case& C, const vector<double>& C1, const vector<double>& C2, const vector<double>& T) {
  Mesh& m = *C.m;
  Level& L = C.lev[0];
  for (int f = 0; f < m.Fi; ++f) {
    const int o = m.owner[f], n = m.neigh[f];
    L.ac[o] = L.ac[o] + C1[f];
    L.anb[m.ownSlot[f]] = L.anb[m.ownSlot[f]] + C2[f];
    L.bc[o] = L.bc[o] - T[f];
    L.ac[n] = L.ac[n] - C2[f];
    L.anb[m.neiSlot[f]] = L.anb[m.neiSlot[f]] - C1[f];
    L.bc[n] = L.bc[n] + T[f];
  }
  for (int f = m.Fi; f < m.F; ++f) {
    const int o = m.owner[f];
    L.ac[o] = L.ac[o] + C1[f];
    L.bc[o] = L.bc[o] - T[f];
  }
}

// Average:Corrected face gradient of one scalar column on an interior face
// (interpolate/cfdInterpolateGradientsFromElementsToInteriorFaces.m:23-70, Q4)
inline void face_grad_corrected(const Case& C, int f, const vector<double>* g, const double* ph, double* out) {
  const Mesh& m = *C.m;
  const int o = m.owner[f], n = m.neigh[f];
  const double w = m.gf[f];
  const bool q4 = q(C, ORQ_Q4_GRAD_WEIGHTS_SWAPPED);
  double gfv[3];
  for (int d = 0; d < 3; ++d)
    gfv[d] = q4 ? (1 - w) * g[d][n] + w * g[d][o] : w * g[d][n] + (1 - w) * g[d][o];
  double dcf[3];
  for (int d = 0; d < 3; ++d) dcf[d] = m.cC[3 * n + d] - m.cC[3 * o + d];
  const double dmag = mag3(dcf);
  double e[3];
  for (int d = 0; d < 3; ++d) e[d] = dcf[d] / dmag;
  const double lgm = (ph[n] - ph[o]) / dmag;
  const double agm = dot3(gfv, e);
  for (int d = 0; d < 3; ++d) out[d] = (gfv[d] - agm * e[d]) + lgm * e[d];
}

inline void face_grad_average(const Case& C, int f, const vector<double>* g, double* out) {
  const Mesh& m = *C.m;
  const int o = m.owner[f], n = m.neigh[f];
  const double w = m.gf[f];
  const bool q4 = q(C, ORQ_Q4_GRAD_WEIGHTS_SWAPPED);
  for (int d = 0; d < 3; ++d)
    out[d] = q4 ? (1 - w) * g[d][n] + w * g[d][o] : w * g[d][n] + (1 - w) * g[d][o];
}

// Momentum component assembly: assemble/cfdAssembleEquation.m:16-27 ->
// cfdAssembleEquationTerms.m:22-55 with the U-equation terms
// div(U*U) = laplacian(nu*U) + div(nu*transp(grad(U))) - grad(p).
int assemble_u(Case& C, int comp, double* rmsOut, double* maxOut) {
  Mesh& m = *C.m;
  const int Nc = m.Nc, Fi = m.Fi, F = m.F;
  fresh_coefficients(C);
  Level& L = C.lev[0];
  const vector<double>& ph = C.U[comp];
  vector<double> C1(F, 0), C2(F, 0), T(F, 0);
  // (1) Convection, upwind, sign +1 (cfdAssembleConvectionTerm.m:103-137 and BCs)
  {
    const double s = 1;
    for (int f = 0; f < Fi; ++f) {
      const double psi = C.mdot[f];
      C1[f] = s * std::max(psi, 0.0);
      C2[f] = -s * std::max(-psi, 0.0);
      T[f] = (C1[f] * ph[m.owner[f]] + C2[f] * ph[m.neigh[f]]) + 0.0;
    }
    for (size_t ip = 0; ip < m.patches.size(); ++ip) {
      const PatchI& P = m.patches[ip];
      for (int j = 0; j < P.n; ++j) {
        const int f = P.start + j, b = Nc + f - Fi;
        if (P.type == ORP_INLET || P.type == ORP_OUTLET) {
          const double psi = C.mdot[f];
          C1[f] = s * std::max(psi, 0.0);
          C2[f] = -s * std::max(-psi, 0.0);
          T[f] = (C1[f] * ph[m.owner[f]] + C2[f] * ph[b]) + 0.0;
        } else {
          C1[f] = 0; C2[f] = 0; T[f] = 0;
        }
      }
    }
    scatter_faces(C, C1, C2, T);
    // cfdAssembleConvectionDivergenceTerm (cfdAssembleConvectionTerm.m:303-349)
    vector<double> eff(Nc, 0.0);
    for (int f = 0; f < Fi; ++f) {
      eff[m.owner[f]] = eff[m.owner[f]] + C.mdot[f];
      eff[m.neigh[f]] = eff[m.neigh[f]] - C.mdot[f];
    }
    for (int f = Fi; f < F; ++f) eff[m.owner[f]] = eff[m.owner[f]] + C.mdot[f];
    for (int e = 0; e < Nc; ++e) {
      const double fce = std::max(eff[e], 0.0) - eff[e];
      const double fve = -std::max(eff[e], 0.0) * ph[e];
      const double fte = fce * ph[e] + fve;
      L.ac[e] = L.ac[e] + fce;
      L.bc[e] = L.bc[e] - fte;
    }
  }
  // (2) Diffusion laplacian(nu*U), sign -1 (cfdAssembleDiffusionTerm.m:94-130 and BCs)
  {
    const double s = -1;
    const vector<double>* g = C.gradU[comp];
    for (int f = 0; f < Fi; ++f) {
      double gfc[3];
      face_grad_corrected(C, f, g, ph.data(), gfc);
      const double gam = C.gammaU[f];
      C1[f] = -s * gam * m.gDiff[f];
      C2[f] = s * gam * m.gDiff[f];
      const double V = s * gam * dot3(gfc, &m.T[3 * f]);
      T[f] = (C1[f] * ph[m.owner[f]] + C2[f] * ph[m.neigh[f]]) + V;
    }
    for (size_t ip = 0; ip < m.patches.size(); ++ip) {
      const PatchI& P = m.patches[ip];
      const int t = C.bcU[ip];
      if ((P.type == ORP_WALL && t == ORB_FIXED_VALUE) || (P.type == ORP_INLET && t == ORB_FIXED_VALUE)) {
        for (int j = 0; j < P.n; ++j) {
          const int f = P.start + j, b = Nc + f - Fi;
          const double gam = C.gammaU[f];
          double gb[3] = {g[0][b], g[1][b], g[2][b]};
          C1[f] = -s * gam * m.gDiff[f];
          C2[f] = s * gam * m.gDiff[f];
          const double V = s * gam * dot3(gb, &m.T[3 * f]);
          T[f] = (C1[f] * ph[m.owner[f]] + C2[f] * ph[b]) + V;
        }
      } else if (P.type == ORP_WALL && t == ORB_NOSLIP) {
        // cfdAssembleDiffusionTermWallNoslipBC (:479-562), Q3 / Q14 / Q15
        double S1 = 0;
        vector<double> nrm(3 * P.n);
        for (int j = 0; j < P.n; ++j) {
          const int f = P.start + j;
          for (int d = 0; d < 3; ++d) nrm[3 * j + d] = m.Sf[3 * f + d] / m.area[f];
        }
        if (q(C, ORQ_Q14_NOSLIP_PATCH_SUM))
          for (int j = 0; j < P.n; ++j) S1 = S1 + nrm[3 * j + comp] * nrm[3 * j + comp];
        const int c2 = comp == 0 ? 1 : 0;   // the two other components, in the MATLAB order
        const int c3 = comp == 2 ? 1 : 2;
        const double third = q(C, ORQ_Q15_NOSLIP_THIRD_SIGN) ? -1.0 : 1.0;
        for (int j = 0; j < P.n; ++j) {
          const int f = P.start + j, b = Nc + f - Fi, o = m.owner[f];
          const double gam = C.gammaU[f];
          const double A = m.area[f];
          const double dn = m.walldist[f];
          const double TM = q(C, ORQ_Q3_NOSLIP_GAMMA_TWICE) ? gam / dn : 1.0;
          const double nc = nrm[3 * j + comp], n2 = nrm[3 * j + c2], n3 = nrm[3 * j + c3];
          const double fac = q(C, ORQ_Q14_NOSLIP_PATCH_SUM) ? (1 - S1) : (1 - nc * nc);
          const double coef = ((-s * gam) * A / dn) * TM;
          const double acv = coef * fac;
          const double inner = (C.U[comp][b] * fac + (C.U[c2][o] - C.U[c2][b]) * n2 * nc)
                               + third * ((C.U[c3][o] - C.U[c3][b]) * n3 * nc);
          const double bcv = coef * inner;
          C1[f] = acv; C2[f] = 0;
          T[f] = (C1[f] * ph[o] + C2[f] * ph[b]) + bcv;
        }
      } else if (P.type == ORP_SYMMETRY || P.type == ORP_EMPTY) {
        // cfdAssembleDiffusionTermSymmetry (:567-629) / Empty (:631-690), vector branch
        for (int j = 0; j < P.n; ++j) {
          const int f = P.start + j, b = Nc + f - Fi, o = m.owner[f];
          const double gam = C.gammaU[f], A = m.area[f];
          double n[3];
          for (int d = 0; d < 3; ++d) n[d] = m.Sf[3 * f + d] / A;
          const double dd = dot3(&m.CN[3 * f], n);
          double a[3], bb[3];
          for (int d = 0; d < 3; ++d) {
            const double l = d == comp ? 0.0 : 1.0;
            a[d] = C.U[d][o] * l; bb[d] = n[d] * l;
          }
          C1[f] = ((((-s * 2) * gam) * A) * (n[comp] * n[comp])) / dd;
          C2[f] = 0;
          const double V = (((((s * 2) * gam) * A) * dot3(a, bb)) * n[comp]) / dd;
          T[f] = (C1[f] * ph[o] + C2[f] * ph[b]) + V;
        }
      } else {
        // wall zeroGradient / slip and outlet: zero flux
        for (int j = 0; j < P.n; ++j) { const int f = P.start + j; C1[f] = 0; C2[f] = 0; T[f] = 0; }
      }
    }
    scatter_faces(C, C1, C2, T);
  }
  // (3) div(nu*transp(grad(U))), sign -1 (cfdAssembleExplicitStressTerm.m:13-49, Q2)
  {
    const double s = -1;
    const bool q2 = q(C, ORQ_Q2_STRESS_NOT_TRANSPOSED);
    for (int f = 0; f < F; ++f) {
      double gf3[3];
      double gam;
      for (int d = 0; d < 3; ++d) {
        const vector<double>& gd = q2 ? C.gradU[comp][d] : C.gradU[d][comp];
        if (f < Fi) {
          const double w = m.gf[f];
          gf3[d] = w * gd[m.neigh[f]] + (1 - w) * gd[m.owner[f]];
        } else {
          gf3[d] = gd[Nc + f - Fi];
        }
      }
      if (f < Fi) {
        const double w = m.gf[f];
        gam = w * C.nuF[m.neigh[f]] + (1 - w) * C.nuF[m.owner[f]];
      } else {
        gam = C.nuF[Nc + f - Fi];
      }
      C1[f] = 0; C2[f] = 0;
      T[f] = (s * gam) * ((gf3[0] * m.Sf[3 * f] + gf3[1] * m.Sf[3 * f + 1]) + gf3[2] * m.Sf[3 * f + 2]);
    }
    scatter_faces(C, C1, C2, T);
  }
  // (4) grad(p), sign +1 (cfdAssemblePressureGradientTerm.m:11-40)
  for (int e = 0; e < Nc; ++e) {
    const double fte = (1.0 * m.vol[e]) * C.gradp[comp][e];
    L.ac[e] = L.ac[e] + 0.0;
    L.bc[e] = L.bc[e] - fte;
  }
  // (5) false transient (cfdAssembleFalseTransientTerm.m:15-49, Q11)
  for (int e = 0; e < Nc; ++e) {
    const double fce = (m.vol[e] * C.rho[e]) / C.fdt;
    const double fceold = (-m.vol[e] * C.rho[e]) / C.fdt;
    const double fte = fce * ph[e];
    L.ac[e] = L.ac[e] + fce;
    C.acOld[e] = C.acOld[e] + fceold;
    L.bc[e] = L.bc[e] - fte;
  }
  // (6) URF (extras/cfdApplyURF.m:13-16)
  for (int e = 0; e < Nc; ++e) L.ac[e] = L.ac[e] / C.urfU;
  // (7) scaled residual (compute/cfdComputeNormalizedResidual.m:55-88)
  double ss = 0, mx = 0;
  for (int e = 0; e < Nc; ++e) {
    if (L.ac[e] == 0) return -3;
    const double r = L.bc[e] / (L.ac[e] * C.scaleU);
    mx = std::max(mx, std::fabs(r));
    ss = ss + r * r;
  }
  *rmsOut = std::sqrt(ss / Nc);
  *maxOut = mx;
  // (8) post-assembly DU (assemble/cfdPostAssembleEquation.m:37-42,75-81)
  C.DU[comp].resize(Nc + m.Fb);
  for (int e = 0; e < Nc; ++e) C.DU[comp][e] = m.vol[e] / L.ac[e];
  for (int k = 0; k < m.Fb; ++k) C.DU[comp][Nc + k] = C.DU[comp][m.owner[Fi + k]];
  return 0;
}

// Pressure-correction assembly: assemble/cfdAssembleMdotTerm.m:32-905 (Rhie-Chow)
int assemble_p(Case& C, double* rmsOut, double* maxOut) {
  Mesh& m = *C.m;
  const int Nc = m.Nc, Fi = m.Fi, F = m.F;
  fresh_coefficients(C);
  vector<double> C1(F, 0), C2(F, 0), T(F, 0);
  const bool q4 = q(C, ORQ_Q4_GRAD_WEIGHTS_SWAPPED);
  for (int f = 0; f < Fi; ++f) {
    const int o = m.owner[f], n = m.neigh[f];
    const double w = m.gf[f];
    const double* S = &m.Sf[3 * f];
    double dbar[3], ub[3];
    for (int c = 0; c < 3; ++c) {
      dbar[c] = w * C.DU[c][n] + (1 - w) * C.DU[c][o];
      ub[c] = w * C.U[c][n] + (1 - w) * C.U[c][o];
    }
    const double mprev = C.mdot[f];
    const double pos = mprev > 0 ? 1.0 : 0.0;
    const double rf = C.rho[o] * pos + C.rho[n] * (1 - pos);
    // pressure gradients: 'Average' and 'Average:Corrected' (both with Q4 weights)
    double gbar[3], gcor[3];
    const vector<double>* gp = C.gradp;
    for (int d = 0; d < 3; ++d)
      gbar[d] = q4 ? (1 - w) * gp[d][n] + w * gp[d][o] : w * gp[d][n] + (1 - w) * gp[d][o];
    face_grad_corrected(C, f, gp, C.p.data(), gcor);
    const double Ub = dot3(ub, S);
    double V = 0 + rf * Ub;
    double DUS[3] = {dbar[0] * S[0], dbar[1] * S[1], dbar[2] * S[2]};
    const double mDUS = mag3(DUS);
    double eDUS[3] = {DUS[0] / mDUS, DUS[1] / mDUS, DUS[2] / mDUS};
    const double* eCF = &m.eCN[3 * f];
    const double den = dot3(eCF, eDUS);
    double DUE[3];
    for (int d = 0; d < 3; ++d) DUE[d] = (mDUS * eCF[d]) / den;
    const double geoDiff = mag3(DUE) / mag3(&m.CN[3 * f]);
    double DUT[3] = {DUS[0] - DUE[0], DUS[1] - DUE[1], DUS[2] - DUE[2]};
    const double FC = 0 + rf * geoDiff;
    const double FF = 0 - rf * geoDiff;
    V = V - rf * dot3(gcor, DUT);
    V = V + rf * dot3(gbar, DUS);
    V = V + (1 - C.urfU) * (mprev - rf * Ub);
    const double md = (FC * C.p[o] + FF * C.p[n]) + V;
    C.mdot[f] = md;
    C1[f] = FC; C2[f] = FF; T[f] = md;
  }
  for (size_t ip = 0; ip < m.patches.size(); ++ip) {
    const PatchI& P = m.patches[ip];
    const int t = C.bcP[ip];
    if (P.type == ORP_INLET && t != ORB_FIXED_VALUE) {
      // cfdAssembleMdotTermInletInletBC (:281-350)
      for (int j = 0; j < P.n; ++j) {
        const int f = P.start + j, b = Nc + f - Fi, o = m.owner[f];
        double Ubv[3] = {C.U[0][b], C.U[1][b], C.U[2][b]};
        const double Usf = dot3(&m.Sf[3 * f], Ubv);
        const double V = 0 + C.rho[b] * Usf;
        const double md = (0.0 * C.p[o] + 0.0 * C.p[b]) + V;
        C.mdot[f] = md;
        C1[f] = 0; C2[f] = 0; T[f] = md;
      }
    } else if (P.type == ORP_OUTLET && t == ORB_FIXED_VALUE) {
      // cfdAssembleMdotTermOutletFixedValueBC (:799-905)
      for (int j = 0; j < P.n; ++j) {
        const int f = P.start + j, b = Nc + f - Fi, o = m.owner[f];
        const double* S = &m.Sf[3 * f];
        const double rb = C.rho[b];
        double DUS[3] = {C.DU[0][b] * S[0], C.DU[1][b] * S[1], C.DU[2][b] * S[2]};
        const double mDUS = mag3(DUS);
        double eDUS[3] = {DUS[0] / mDUS, DUS[1] / mDUS, DUS[2] / mDUS};
        const double* eCN = &m.eCN[3 * f];
        const double den = dot3(eCN, eDUS);
        double DUE[3];
        for (int d = 0; d < 3; ++d) DUE[d] = (mDUS / den) * eCN[d];
        const double geoDiff = mag3(DUE) / mag3(&m.CN[3 * f]);
        double DUT[3] = {DUS[0] - DUE[0], DUS[1] - DUE[1], DUS[2] - DUE[2]};
        double vb[3] = {C.U[0][b], C.U[1][b], C.U[2][b]};
        double gb[3] = {C.gradp[0][b], C.gradp[1][b], C.gradp[2][b]};
        const double Ub = dot3(vb, S);
        double V = 0.0 + rb * Ub;
        const double FC = 0.0 + rb * geoDiff;
        const double FF = 0.0 - 0.0;
        V = V - rb * dot3(gb, DUT);
        V = V + rb * dot3(gb, DUS);
        const double md = (FC * C.p[o] + FF * C.p[b]) + V;
        C.mdot[f] = md;
        C1[f] = FC; C2[f] = FF; T[f] = md;
      }
    } else if (P.type == ORP_WALL || P.type == ORP_EMPTY || P.type == ORP_SYMMETRY) {
      for (int j = 0; j < P.n; ++j) { const int f = P.start + j; C1[f] = 0; C2[f] = 0; T[f] = 0; }
    } else {
      return -4;  // BC combinations the reference does not implement for this path
    }
  }
  C.fluxC1 = C1; C.fluxC2 = C2;
  scatter_faces(C, C1, C2, T);
  // residual = effective divergence (compute/cfdComputeNormalizedResidual.m:27-31,
  // compute/cfdComputeEffectiveDivergence.m:21-54)
  vector<double> eff(Nc, 0.0);
  for (int f = 0; f < Fi; ++f) {
    eff[m.owner[f]] = eff[m.owner[f]] + C.mdot[f];
    eff[m.neigh[f]] = eff[m.neigh[f]] - C.mdot[f];
  }
  for (int f = Fi; f < F; ++f) eff[m.owner[f]] = eff[m.owner[f]] + C.mdot[f];
  double mx = -INFINITY, ss = 0;
  for (int e = 0; e < Nc; ++e) { mx = std::max(mx, eff[e]); ss = ss + eff[e] * eff[e]; }
  *maxOut = mx;
  *rmsOut = std::sqrt(ss / Nc);
  return 0;
}

// ---- AMG (solve/AMG/*) ----
int build_hierarchy(Case& C) {
  // cfdAgglomerate.m:7-17
  C.lev.resize(1);
  int iLevel = 0;
  while (iLevel < C.maxCoarse) {
    ++iLevel;
    Level coarse;
    vector<int> parents;
    const int np = agglomerate(C.lev[iLevel - 1], parents, coarse);
    if (np == 1 && !q(C, ORQ_Q16_ONE_CELL_COARSEST)) {
      // repaired: a single aggregate of a pure-Neumann operator has a zero diagonal
      --iLevel;
      break;
    }
    C.lev[iLevel - 1].parents = parents;
    C.lev.push_back(coarse);
    if (np <= 5) break;
  }
  for (auto& L : C.lev) {
    if (C.pSmoother == ORS_MCGS) {
      L.color.resize(L.n);
      L.ncolor = coloring(L.n, L.rp.data(), L.col.data(), L.color.data());
    }
  }
  C.maxLevels = iLevel;  // index of the coarsest level (0-based)
  return iLevel;
}

void smooth(Case& C, int l, int nIter, double rrf) {
  solve_algebraic_system(C.lev[l], C.pSmoother, nIter, rrf, C.quirks, nullptr, nullptr, nullptr);
}

// cfdRestrict.m:5-12 + cfdUpdateRHS.m:10-17
void restrict_(Case& C, int l, int pre /* <0: no smoothing */) {
  if (pre >= 0) smooth(C, l, pre, 0.1);
  Level& F = C.lev[l];
  Level& Cc = C.lev[l + 1];
  vector<double> r(F.n);
  residuals(F.n, F.rp.data(), F.col.data(), F.ac.data(), F.anb.data(), F.bc.data(), F.dphi.data(), r.data());
  Cc.bc.assign(Cc.n, 0.0);
  for (int i = 0; i < F.n; ++i) Cc.bc[F.parents[i]] = Cc.bc[F.parents[i]] + r[i];
  if (!q(C, ORQ_Q6_COARSE_DPHI_KEPT)) std::fill(Cc.dphi.begin(), Cc.dphi.end(), 0.0);
}

// cfdProlongate.m:5-6 + cfdCorrectFinerLevelSolution.m:11-14
void prolong_(Case& C, int l, double rrf) {
  Level& Cc = C.lev[l];
  Level& F = C.lev[l - 1];
  for (int i = 0; i < F.n; ++i) F.dphi[i] = F.dphi[i] + Cc.dphi[F.parents[i]];
  smooth(C, l - 1, C.post, rrf);
}

double final_residual(Case& C) {
  Level& L = C.lev[0];
  return sum_abs_res(L.n, L.rp.data(), L.col.data(), L.ac.data(), L.anb.data(), L.bc.data(), L.dphi.data());
}

double vcycle(Case& C, double rrf) {
  const int Lm = C.maxLevels;
  for (int l = 0; l < Lm; ++l) restrict_(C, l, C.pre);
  smooth(C, Lm, C.post, 0.1);
  for (int l = Lm; l >= 1; --l) prolong_(C, l, rrf);
  return final_residual(C);
}

// cfdApplyWCycle.m:3-83 (levels written 1-based there; L = maxLevels)
int wcycle(Case& C, double rrf, double* out) {
  const int L = C.maxLevels;  // 0-based index of the coarsest level
  if (L < 3) return -5;       // the reference indexes level 0 / negative levels and errors out
  for (int l = 0; l < L; ++l) restrict_(C, l, C.pre);
  auto solve = [&]() { smooth(C, L, C.post, 0.1); };
  solve();
  prolong_(C, L, rrf);
  restrict_(C, L - 1, -1);
  solve();
  prolong_(C, L, rrf); prolong_(C, L - 1, rrf);
  restrict_(C, L - 2, -1); restrict_(C, L - 1, C.pre);
  solve();
  prolong_(C, L, rrf); prolong_(C, L - 1, rrf); prolong_(C, L - 2, rrf);
  restrict_(C, L - 3, -1); restrict_(C, L - 2, C.pre); restrict_(C, L - 1, C.pre);
  solve();
  prolong_(C, L, rrf); prolong_(C, L - 1, rrf);
  restrict_(C, L - 2, -1); restrict_(C, L - 1, C.pre);
  solve();
  prolong_(C, L, rrf);
  restrict_(C, L - 1, -1);
  solve();
  for (int l = L; l >= 1; --l) prolong_(C, l, rrf);
  *out = final_residual(C);
  return 0;
}

// cfdApplyFCycle.m
int fcycle(Case& C, double rrf, double* out) {
  const int L = C.maxLevels;
  if (L < 3) return -5;
  for (int l = 0; l < L; ++l) restrict_(C, l, C.pre);
  auto solve = [&]() { smooth(C, L, C.post, 0.1); };
  solve();
  prolong_(C, L, rrf);
  restrict_(C, L - 1, -1);
  solve();
  prolong_(C, L, rrf); prolong_(C, L - 1, rrf);
  restrict_(C, L - 2, -1); restrict_(C, L - 1, C.pre);
  solve();
  prolong_(C, L, rrf); prolong_(C, L - 1, rrf); prolong_(C, L - 2, rrf);
  restrict_(C, L - 3, -1); restrict_(C, L - 2, C.pre); restrict_(C, L - 1, C.pre);
  solve();
  for (int l = L; l >= 1; --l) prolong_(C, l, rrf);
  *out = final_residual(C);
  return 0;
}

// solve/AMG/cfdApplyAMG.m:9-57
int apply_amg(Case& C, double* r0, double* r1) {
  build_hierarchy(C);
  const double init = final_residual(C);
  double fin = init;
  int nCycle = 1;
  while (nCycle <= C.maxCycles && fin > C.pRrf * init) {
    if (C.cycle == ORC_V) fin = vcycle(C, C.pRrf);
    else {
      int rc = C.cycle == ORC_W ? wcycle(C, C.pRrf, &fin) : fcycle(C, C.pRrf, &fin);
      if (rc) return rc;
    }
    ++nCycle;
  }
  *r0 = init; *r1 = fin;
  return 0;
}

// solve/cfdSolveEquation.m:11-18
int solve(Case& C, int eq, double* r0, double* r1) {
  if (eq == 1 && C.pAMG) return apply_amg(C, r0, r1);
  C.lev.resize(1);
  const int sm = eq == 1 ? C.pSmoother : C.uSmoother;
  Level& L = C.lev[0];
  if (sm == ORS_MCGS) { L.color.resize(L.n); L.ncolor = coloring(L.n, L.rp.data(), L.col.data(), L.color.data()); }
  solve_algebraic_system(L, sm, eq == 1 ? 10 : C.uNIter, eq == 1 ? 0.1 : C.uRrf, C.quirks, r0, r1, nullptr);
  return 0;
}

inline void tangential(Case& C, int f, int b, int o, int comp_lo, int comp_hi) {
  Mesh& m = *C.m;
  const double* S = &m.Sf[3 * f];
  const double nS = mag3(S);
  double n[3] = {S[0] / nS, S[1] / nS, S[2] / nS};
  double uo[3] = {C.U[0][o], C.U[1][o], C.U[2][o]};
  const double un = dot3(uo, n);
  for (int c = comp_lo; c <= comp_hi; ++c) C.U[c][b] = C.U[c][o] - un * n[c];
}

// solve/correct/cfdCorrectScalarEquation.m:16-109 for U (via cfdCorrectVelocityEquation)
void correct_u(Case& C, int comp) {
  Mesh& m = *C.m;
  const int Nc = m.Nc, Fi = m.Fi;
  Level& L = C.lev[0];
  for (int e = 0; e < Nc; ++e) C.U[comp][e] = C.U[comp][e] + L.dphi[e];
  for (size_t ip = 0; ip < m.patches.size(); ++ip) {
    const PatchI& P = m.patches[ip];
    const int t = C.bcU[ip];
    for (int j = 0; j < P.n; ++j) {
      const int f = P.start + j, b = Nc + f - Fi, o = m.owner[f];
      if (P.type == ORP_WALL) {
        if (t == ORB_ZERO_GRADIENT) C.U[comp][b] = C.U[comp][o];
        else if (t == ORB_SLIP) tangential(C, f, b, o, comp, comp);
      } else if (P.type == ORP_OUTLET) {
        if (t == ORB_ZERO_GRADIENT) C.U[comp][b] = C.U[comp][o];
      } else if (P.type == ORP_SYMMETRY || P.type == ORP_EMPTY) {
        tangential(C, f, b, o, comp, comp);
      }
    }
  }
}

// solve/correct/cfdCorrectEquation.m:26-47 for p
void correct_p(Case& C) {
  Mesh& m = *C.m;
  const int Nc = m.Nc, Fi = m.Fi, Fb = m.Fb;
  Level& L = C.lev[0];
  // cfdCorrectPPField.m:26-52
  C.PP.resize(Nc + Fb, 0.0);
  const double ppc = C.fixedEl >= 0 ? L.dphi[C.fixedEl] : 0.0;
  for (int e = 0; e < Nc; ++e) C.PP[e] = L.dphi[e] - ppc;
  for (size_t ip = 0; ip < m.patches.size(); ++ip) {
    const PatchI& P = m.patches[ip];
    const int t = C.bcP[ip];
    for (int j = 0; j < P.n; ++j) {
      const int f = P.start + j, b = Nc + f - Fi;
      if ((P.type == ORP_INLET || P.type == ORP_OUTLET) && t == ORB_FIXED_VALUE) C.PP[b] = 0;
      else C.PP[b] = C.PP[m.owner[f]];
    }
  }
  vector<double> (*gpp)[3] = reinterpret_cast<vector<double> (*)[3]>(&C.gradPP);
  update_gradient(C, &C.PP, 1, gpp);
  // cfdCorrectVelocityField.m:26-55 + boundary patches
  for (int e = 0; e < Nc; ++e)
    for (int c = 0; c < 3; ++c) C.U[c][e] = C.U[c][e] - C.DU[c][e] * C.gradPP[c][e];
  for (size_t ip = 0; ip < m.patches.size(); ++ip) {
    const PatchI& P = m.patches[ip];
    const int t = C.bcP[ip];
    if (P.type == ORP_OUTLET && t == ORB_FIXED_VALUE) {
      // cfdCorrectMdotAndVelocityOutletFixedValueBC (:250-270), Q12
      for (int j = 0; j < P.n; ++j) {
        const int f = P.start + j, o = m.owner[f];
        const int row = q(C, ORQ_Q12_OUTLET_U_FACE_ROWS) ? f : Nc + f - Fi;
        for (int c = 0; c < 3; ++c) {
          if ((int)C.U[c].size() <= row) C.U[c].resize(row + 1, 0.0);
        }
        double uo[3] = {C.U[0][o], C.U[1][o], C.U[2][o]};
        for (int c = 0; c < 3; ++c) C.U[c][row] = uo[c];
      }
    } else if (P.type == ORP_SYMMETRY || P.type == ORP_EMPTY || (P.type == ORP_WALL && t == ORB_SLIP)) {
      for (int j = 0; j < P.n; ++j) {
        const int f = P.start + j;
        tangential(C, f, Nc + f - Fi, m.owner[f], 0, 2);
      }
    }
  }
  // cfdCorrectPressureEquation.m:22-54
  const double ppf = C.fixedEl >= 0 ? C.PP[C.fixedEl] : 0.0;
  for (int e = 0; e < Nc; ++e) C.p[e] = C.p[e] + C.urfP * (C.PP[e] - ppf);
  for (size_t ip = 0; ip < m.patches.size(); ++ip) {
    const PatchI& P = m.patches[ip];
    const int t = C.bcP[ip];
    if ((P.type == ORP_INLET || P.type == ORP_OUTLET) && t == ORB_FIXED_VALUE) continue;
    for (int j = 0; j < P.n; ++j) {
      const int f = P.start + j;
      C.p[Nc + f - Fi] = C.p[m.owner[f]];
    }
  }
  // cfdCorrectMdotField.m:24-50 + boundary patches
  for (int f = 0; f < Fi; ++f)
    C.mdot[f] = (C.mdot[f] + C.fluxC1[f] * C.PP[m.owner[f]]) + C.fluxC2[f] * C.PP[m.neigh[f]];
  for (size_t ip = 0; ip < m.patches.size(); ++ip) {
    const PatchI& P = m.patches[ip];
    const int t = C.bcP[ip];
    for (int j = 0; j < P.n; ++j) {
      const int f = P.start + j, b = Nc + f - Fi, o = m.owner[f];
      if (P.type == ORP_SYMMETRY || P.type == ORP_EMPTY || (P.type == ORP_WALL && t == ORB_SLIP)) {
        C.mdot[f] = 0.0 * C.mdot[f];
      } else if (P.type == ORP_OUTLET && t == ORB_FIXED_VALUE) {
        double uo[3] = {C.U[0][o], C.U[1][o], C.U[2][o]};
        C.mdot[f] = C.rho[b] * dot3(uo, &m.Sf[3 * f]);
      }
    }
  }
}

}  // namespace

// ====================================================================================
extern "C" {

void* orc_mesh_create(int nPoints, const double* points, int nFaces, const int* faceStart,
                      const int* faceNodes, int nInterior, const int* owner, const int* neighbour,
                      int nPatches, const int* patchType, const int* patchStart, const int* patchN,
                      int quirks) {
  Mesh* m = new Mesh();
  m->nP = nPoints; m->F = nFaces; m->Fi = nInterior; m->Fb = nFaces - nInterior; m->quirks = quirks;
  m->pts.assign(points, points + 3 * nPoints);
  m->fstart.assign(faceStart, faceStart + nFaces + 1);
  m->fnodes.assign(faceNodes, faceNodes + faceStart[nFaces]);
  m->owner.assign(owner, owner + nFaces);
  m->neigh.assign(neighbour, neighbour + nInterior);
  int nc = 0;
  for (int f = 0; f < nFaces; ++f) nc = std::max(nc, owner[f] + 1);
  for (int f = 0; f < nInterior; ++f) nc = std::max(nc, neighbour[f] + 1);
  m->Nc = nc;
  for (int p = 0; p < nPatches; ++p) m->patches.push_back({patchType[p], patchStart[p], patchN[p]});
  process_mesh(*m);
  return m;
}

void orc_mesh_destroy(void* m) { delete static_cast<Mesh*>(m); }

void orc_mesh_sizes(void* mv, int* s) {
  Mesh* m = static_cast<Mesh*>(mv);
  s[0] = m->Nc; s[1] = m->F; s[2] = m->Fi; s[3] = (int)m->col.size();
}

int orc_mesh_get(void* mv, const char* name, void* out) {
  Mesh* m = static_cast<Mesh*>(mv);
  std::string n(name);
  auto cpd = [&](const vector<double>& v) { std::memcpy(out, v.data(), v.size() * sizeof(double)); return (int)v.size(); };
  auto cpi = [&](const vector<int>& v) { std::memcpy(out, v.data(), v.size() * sizeof(int)); return (int)v.size(); };
  if (n == "Sf") return cpd(m->Sf);
  if (n == "centroid_f") return cpd(m->fC);
  if (n == "area") return cpd(m->area);
  if (n == "CN") return cpd(m->CN);
  if (n == "eCN") return cpd(m->eCN);
  if (n == "gDiff") return cpd(m->gDiff);
  if (n == "T") return cpd(m->T);
  if (n == "gf") return cpd(m->gf);
  if (n == "walldist") return cpd(m->walldist);
  if (n == "volume") return cpd(m->vol);
  if (n == "centroid_c") return cpd(m->cC);
  if (n == "rowptr") return cpi(m->rowptr);
  if (n == "col") return cpi(m->col);
  if (n == "own_slot") return cpi(m->ownSlot);
  if (n == "nei_slot") return cpi(m->neiSlot);
  if (n == "cell_face_start") return cpi(m->cfStart);
  if (n == "cell_faces") return cpi(m->cfFaces);
  return -1;
}

void* orc_case_create(void* mesh, const int* is, const double* ds, const int* bcTypeU, const int* bcTypeP,
                      const double* bcValU, const double* bcValP, const double* U0, const double* p0,
                      const double* mdot0) {
  Case* C = new Case();
  Mesh& m = *static_cast<Mesh*>(mesh);
  C->m = &m;
  C->nCorr = is[0]; C->fixedEl = is[1]; C->cycle = is[2]; C->maxCycles = is[3]; C->maxCoarse = is[4];
  C->pre = is[5]; C->post = is[6]; C->pSmoother = is[7]; C->uSmoother = is[8]; C->uNIter = is[9];
  C->quirks = is[10]; C->pAMG = is[11];
  C->nu = ds[0]; C->urfU = ds[1]; C->urfP = ds[2]; C->tolU = ds[3]; C->tolP = ds[4];
  C->pRrf = ds[5]; C->uRrf = ds[6]; C->fdt = ds[7];
  const int Nc = m.Nc, Fb = m.Fb, Fi = m.Fi, F = m.F;
  C->bcU.assign(bcTypeU, bcTypeU + m.patches.size());
  C->bcP.assign(bcTypeP, bcTypeP + m.patches.size());
  C->valU.assign(bcValU, bcValU + 3 * Fb);
  C->valP.assign(bcValP, bcValP + Fb);
  // initial fields: cfdInitializeEquation.m + cfdInitializeBoundaryConditions.m
  for (int c = 0; c < 3; ++c) {
    C->U[c].assign(Nc + Fb, 0.0);
    for (int e = 0; e < Nc; ++e) C->U[c][e] = U0 ? U0[3 * e + c] : 0.0;
  }
  C->p.assign(Nc + Fb, 0.0);
  for (int e = 0; e < Nc; ++e) C->p[e] = p0 ? p0[e] : 0.0;
  C->nuF.assign(Nc + Fb, C->nu);
  C->rho.assign(Nc + Fb, 1.0);
  C->PP.assign(Nc + Fb, 0.0);
  for (int c = 0; c < 3; ++c) C->DU[c].assign(Nc + Fb, 0.0);
  for (int d = 0; d < 3; ++d) C->gradPP[d].assign(Nc + Fb, 0.0);
  // boundary initial values (initialize/cfdInitializeBoundaryConditions.m)
  for (size_t ip = 0; ip < m.patches.size(); ++ip) {
    const PatchI& P = m.patches[ip];
    for (int j = 0; j < P.n; ++j) {
      const int f = P.start + j, k = f - Fi, b = Nc + k, o = m.owner[f];
      const int tu = C->bcU[ip], tp = C->bcP[ip];
      if (tu == ORB_FIXED_VALUE || tu == ORB_NOSLIP) {
        for (int c = 0; c < 3; ++c) C->U[c][b] = C->valU[3 * k + c];
      } else if (tu == ORB_ZERO_GRADIENT) {
        if (P.type == ORP_INLET) C->U[0][b] = C->U[0][o];  // linear index: component 1 only
        else for (int c = 0; c < 3; ++c) C->U[c][b] = C->U[c][o];
      } else if (tu == ORB_SLIP || tu == ORB_SYMMETRY || tu == ORB_EMPTY) {
        tangential(*C, f, b, o, 0, 2);
      }
      if (tp == ORB_FIXED_VALUE) C->p[b] = C->valP[k];
      else C->p[b] = C->p[o];
    }
  }
  // gradients at initialisation (cfdInitializeEquation.m:23)
  update_gradient(*C, C->U, 3, C->gradU);
  vector<double> (*gp)[3] = reinterpret_cast<vector<double> (*)[3]>(&C->gradp);
  update_gradient(*C, &C->p, 1, gp);
  update_gamma(*C);
  // mdot_f (initialize/cfdInitializeMdotField.m:72-86): rho = ones over faces, Average
  C->mdot.assign(F, 0.0);
  if (mdot0) {
    for (int f = 0; f < F; ++f) C->mdot[f] = mdot0[f];
  } else {
    for (int f = 0; f < F; ++f) {
      double uf[3], rf;
      if (f < Fi) {
        const double w = m.gf[f];
        for (int c = 0; c < 3; ++c) uf[c] = w * C->U[c][m.neigh[f]] + (1 - w) * C->U[c][m.owner[f]];
        rf = w * 1.0 + (1 - w) * 1.0;
      } else {
        for (int c = 0; c < 3; ++c) uf[c] = C->U[c][Nc + f - Fi];
        rf = 1.0;
      }
      C->mdot[f] = rf * dot3(&m.Sf[3 * f], uf);
    }
  }
  C->fluxC1.assign(F, 0.0); C->fluxC2.assign(F, 0.0);
  fresh_coefficients(*C);
  return C;
}

void orc_case_destroy(void* c) { delete static_cast<Case*>(c); }

void orc_update_fields(void* cv) { update_fields(*static_cast<Case*>(cv)); }
int orc_assemble_u(void* cv, int comp, double* rms, double* mx) { return assemble_u(*static_cast<Case*>(cv), comp, rms, mx); }
int orc_assemble_p(void* cv, double* rms, double* mx) { return assemble_p(*static_cast<Case*>(cv), rms, mx); }
int orc_solve(void* cv, int eq, double* r0, double* r1) { return solve(*static_cast<Case*>(cv), eq, r0, r1); }
void orc_correct_u(void* cv, int comp) { correct_u(*static_cast<Case*>(cv), comp); }
void orc_correct_p(void* cv) { correct_p(*static_cast<Case*>(cv)); }

int orc_case_iterate(void* cv, double* res) {
  Case& C = *static_cast<Case*>(cv);
  update_fields(C);
  for (int c = 0; c < 3; ++c) {
    int rc = assemble_u(C, c, &res[c], &res[4 + c]);
    if (rc) return rc;
    rc = solve(C, 0, &res[8 + c], &res[12 + c]);
    if (rc) return rc;
    correct_u(C, c);
  }
  for (int k = 0; k < C.nCorr; ++k) {
    int rc = assemble_p(C, &res[3], &res[7]);
    if (rc) return rc;
    rc = solve(C, 1, &res[11], &res[15]);
    if (rc) return rc;
    correct_p(C);
  }
  for (int i = 0; i < 4; ++i)
    if (std::isnan(res[i])) return -1;
  const bool conv = res[0] <= C.tolU && res[1] <= C.tolU && res[2] <= C.tolU && res[3] <= C.tolP;
  return conv ? 1 : 0;
}

int orc_case_get(void* cv, const char* name, double* out, int* n) {
  Case& C = *static_cast<Case*>(cv);
  Mesh& m = *C.m;
  std::string s(name);
  int cnt = 0;
  auto put = [&](const vector<double>& v) { if (out) std::memcpy(out + cnt, v.data(), v.size() * sizeof(double)); cnt += (int)v.size(); };
  if (s == "U") { for (int c = 0; c < 3; ++c) put(C.U[c]); }
  else if (s == "gradU") { for (int c = 0; c < 3; ++c) for (int d = 0; d < 3; ++d) put(C.gradU[c][d]); }
  else if (s == "p") put(C.p);
  else if (s == "gradp") { for (int d = 0; d < 3; ++d) put(C.gradp[d]); }
  else if (s == "PP") put(C.PP);
  else if (s == "gradPP") { for (int d = 0; d < 3; ++d) put(C.gradPP[d]); }
  else if (s == "DU") { for (int c = 0; c < 3; ++c) put(C.DU[c]); }
  else if (s == "mdot") put(C.mdot);
  else if (s == "gammaU") put(C.gammaU);
  else if (s == "fluxC1") put(C.fluxC1);
  else if (s == "fluxC2") put(C.fluxC2);
  else if (s == "ac") put(C.lev[0].ac);
  else if (s == "bc") put(C.lev[0].bc);
  else if (s == "anb") put(C.lev[0].anb);
  else if (s == "dphi") put(C.lev[0].dphi);
  else if (s == "scaleU") { if (out) out[0] = C.scaleU; cnt = 1; }
  else return -1;
  (void)m;
  if (n) *n = cnt;
  return 0;
}

int orc_case_set(void* cv, const char* name, const double* in) {
  Case& C = *static_cast<Case*>(cv);
  std::string s(name);
  auto get = [&](vector<double>& v, int off) { std::memcpy(v.data(), in + off, v.size() * sizeof(double)); return off + (int)v.size(); };
  int off = 0;
  if (s == "U") { for (int c = 0; c < 3; ++c) off = get(C.U[c], off); }
  else if (s == "p") get(C.p, 0);
  else if (s == "mdot") get(C.mdot, 0);
  else if (s == "DU") { for (int c = 0; c < 3; ++c) off = get(C.DU[c], off); }
  else if (s == "gradp") { for (int d = 0; d < 3; ++d) off = get(C.gradp[d], off); }
  else if (s == "gradU") { for (int c = 0; c < 3; ++c) for (int d = 0; d < 3; ++d) off = get(C.gradU[c][d], off); }
  else if (s == "dphi") get(C.lev[0].dphi, 0);
  else return -1;
  return 0;
}

int orc_case_nlevels(void* cv) { return (int)static_cast<Case*>(cv)->lev.size(); }

int orc_level_get(void* cv, int level, const char* name, void* out, int* n) {
  Case& C = *static_cast<Case*>(cv);
  if (level < 0 || level >= (int)C.lev.size()) return -1;
  Level& L = C.lev[level];
  std::string s(name);
  int cnt = 0;
  if (s == "parents") { cnt = (int)L.parents.size(); if (out) std::memcpy(out, L.parents.data(), cnt * sizeof(int)); }
  else if (s == "rowptr") { cnt = (int)L.rp.size(); if (out) std::memcpy(out, L.rp.data(), cnt * sizeof(int)); }
  else if (s == "col") { cnt = (int)L.col.size(); if (out) std::memcpy(out, L.col.data(), cnt * sizeof(int)); }
  else if (s == "color") { cnt = (int)L.color.size(); if (out) std::memcpy(out, L.color.data(), cnt * sizeof(int)); }
  else if (s == "ac") { cnt = L.n; if (out) std::memcpy(out, L.ac.data(), cnt * sizeof(double)); }
  else if (s == "anb") { cnt = (int)L.anb.size(); if (out) std::memcpy(out, L.anb.data(), cnt * sizeof(double)); }
  else if (s == "bc") { cnt = L.n; if (out) std::memcpy(out, L.bc.data(), cnt * sizeof(double)); }
  else if (s == "dphi") { cnt = L.n; if (out) std::memcpy(out, L.dphi.data(), cnt * sizeof(double)); }
  else return -1;
  if (n) *n = cnt;
  return 0;
}

void orc_residuals(int n, const int* rp, const int* col, const double* ac, const double* anb,
                   const double* bc, const double* x, double* r) { residuals(n, rp, col, ac, anb, bc, x, r); }
void orc_sor_sweep(int n, const int* rp, const int* col, const double* ac, const double* anb,
                   const double* bc, double* x) { sor_sweep(n, rp, col, ac, anb, bc, x); }
void orc_ilu_factor(int n, const int* rp, const int* col, const double* ac, const double* anb,
                    double* dc, int quirks) { ilu_factor(n, rp, col, ac, anb, dc, quirks); }
void orc_ilu_sweep(int n, const int* rp, const int* col, const double* ac, const double* anb,
                   const double* bc, const double* dc, double* x) {
  vector<double> rc;
  ilu_sweep(n, rp, col, ac, anb, bc, dc, x, rc);
}
void orc_mcgs_sweep(int n, const int* rp, const int* col, const double* ac, const double* anb,
                    const double* bc, const int* color, int ncolor, double* x) {
  mcgs_sweep(n, rp, col, ac, anb, bc, color, ncolor, x);
}
int orc_coloring(int n, const int* rp, const int* col, int* color) { return coloring(n, rp, col, color); }

void orc_solve_algebraic_system(int n, const int* rp, const int* col, const double* ac, const double* anb,
                                const double* bc, double* dphi, int smoother, int nIter, double rrf,
                                int quirks, double* r0, double* r1, int* iters) {
  Level L;
  L.n = n; L.rp.assign(rp, rp + n + 1); L.col.assign(col, col + rp[n]);
  L.ac.assign(ac, ac + n); L.anb.assign(anb, anb + rp[n]); L.bc.assign(bc, bc + n); L.dphi.assign(dphi, dphi + n);
  if (smoother == ORS_MCGS) { L.color.resize(n); L.ncolor = coloring(n, rp, col, L.color.data()); }
  solve_algebraic_system(L, smoother, nIter, rrf, quirks, r0, r1, iters);
  std::memcpy(dphi, L.dphi.data(), n * sizeof(double));
}

int orc_agglomerate(int n, const int* rp, const int* col, const double* ac, const double* anb,
                    int* parents, int* crowptr, int* ccol, double* cac, double* canb, int* cnnz) {
  Level F;
  F.n = n; F.rp.assign(rp, rp + n + 1); F.col.assign(col, col + rp[n]);
  F.ac.assign(ac, ac + n); F.anb.assign(anb, anb + rp[n]);
  Level Cc;
  vector<int> par;
  const int nc = agglomerate(F, par, Cc);
  std::memcpy(parents, par.data(), n * sizeof(int));
  std::memcpy(crowptr, Cc.rp.data(), (nc + 1) * sizeof(int));
  std::memcpy(ccol, Cc.col.data(), Cc.col.size() * sizeof(int));
  std::memcpy(cac, Cc.ac.data(), nc * sizeof(double));
  std::memcpy(canb, Cc.anb.data(), Cc.anb.size() * sizeof(double));
  *cnnz = (int)Cc.col.size();
  return nc;
}

}  // extern "C"
