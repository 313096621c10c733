// case.cuh -- device-resident state of one steady SIMPLE case (the GPU counterpart of
// uFVM's global `Domain` struct for this path: setup/cfdSetupDomain.m:11-63).
#pragma once
#include <algorithm>
#include <string>
#include <vector>

#include "common.cuh"

namespace ufvm {

// Processed mesh in HBM, structure of arrays (x, y, z split) so that face and cell
// passes read each component with unit-stride, 32-byte-sector-aligned accesses.
struct DMesh {
  int Nc = 0, F = 0, Fi = 0, Fb = 0, nnz = 0;
  DArr<int> owner, neigh, cfStart, cfFace, rowptr, col, ownSlot, neiSlot, bPatch;
  DArr<double> fCx, fCy, fCz, Sx, Sy, Sz, area, CNx, CNy, CNz, eCx, eCy, eCz, gDiff, Tx, Ty, Tz, gf, wd;
  DArr<double> vol, cCx, cCy, cCz;
};

struct DPatch {
  DArr<int> ptype, pstart, pcount, bcU, bcP;
  DArr<double> pnsum;  // [patch][3] sum of n_c^2 over the patch
};

struct HPatch {
  int n = 0;
  std::vector<int> type, start, count, bcU, bcP;
};

// One AMG level (level 0 = the assembled matrix), cconn-ordered CSR.
struct Level {
  int n = 0, nnz = 0;
  DArr<int> rowptr, col, parents, tpos;
  DArr<double> ac, anb, bc, dphi, r, dc, rc;
  // level schedules for the natural-order sweeps; lord lists each row's lower neighbours as
  // CSR positions in increasing column order (-1 in the row's remaining slots)
  bool sched_valid = false;
  int nfwd = 0, nbwd = 0, maxw = 0;
  DArr<int> lvl, fwdRows, fwdStart, bwdRows, bwdStart, lord;
  // dc holds the DILU factor of the current matrix while dc_epoch equals the solver's epoch
  unsigned long long dc_epoch = 0;
  int dc_quirks = 0;
  // Position-ordered ELL copies for the narrow level-scheduled sweeps, one per kind (0: GS
  // forward, all entries; 1: GS backward, all entries; 2: DILU forward, lower entries by
  // increasing column; 3: DILU backward, upper entries): entry t of schedule position p at
  // [t * n + p] (column -1 past the row's end), coefficients copied from the matrix;
  // sell_epoch as dc_epoch for the copied coefficients
  bool sell_valid[4] = {false, false, false, false};
  int sellW[4] = {0, 0, 0, 0};
  unsigned long long sell_epoch[4] = {0, 0, 0, 0};
  DArr<int> sellCol[4];
  DArr<double> sellA[4];
  // multicolour ordering
  bool color_valid = false;
  int ncolor = 0;
  DArr<int> color, colorRows, colorStart;
  std::vector<int> h_colorStart;
  // colour-major ELL copy for the plain FP64 multicolour sweep: position p holds row mcRow[p]
  // (colours ascending, rows ascending inside a colour), entry k at [k * n + p]; mc_epoch as
  // dc_epoch for the copied matrix values
  bool mc_valid = false;
  int mcW = 0;
  unsigned long long mc_epoch = 0;
  DArr<int> mcRow, mcCol;
  DArr<double> mcAnb, mcAc, mcBc;
  // children of each coarse row of the NEXT level (restriction / Galerkin)
  DArr<int> childStart, child;
  // FP32 copies for the mixed-precision smoother
  DArr<float> ac32, anb32, bc32, dphi32, r32;
  // FP64 flexible-CG vectors of the level-0 refinement (residual, search direction, A times
  // search direction)
  DArr<double> fr, fp, fq;
  // the batched service's FP32 V-cycle stores every level but the coarsest colour-permuted in
  // ELL form: position p holds row perm[p] (colour-major, natural order inside a colour), inv
  // is the inverse map, entry k of row p sits at [k * n + p] (column as a position, -1 past
  // the row's end); parentsP maps positions to the next level's storage indices, and
  // childStartP / childP list each next-level storage index's children as positions
  bool ell_valid = false;
  int ellW = 0;
  DArr<int> perm, inv, ellCol, parentsP, childP, childStartP, gpos;
  DArr<float> ellAnb;
  DArr<double> uAnb, uAc, uBc, uX;  // level 0: FP64 ELL copy of the momentum matrix (service U solve)
};

// Scratch buffers for matrix-level work (owned by a Case or by a stand-alone call).
struct LinCtx {
  cudaStream_t stream = nullptr;
  int nsm = 148;
  DArr<double> part, red;      // reduction partials / results
  DArr<int> iflag, iscan;      // flags / scan temporaries
  DArr<unsigned int> bar;      // grid barrier: count, gen
  DArr<int> berr;              // grid barrier timeout flag
  // An AMG solve keeps every level's matrix fixed, so the DILU factor computed by the first
  // smoother call on a level is reused by the later ones of the same solve (the factorisation
  // is a function of the matrix alone: same bits). factor_epoch names the solve; 0 = no reuse.
  unsigned long long factor_epoch = 0;
  int cluster_ok = 0;  // cluster sweeps: 0 not yet probed, 1 usable, -1 not usable
  int ensure(int n);
  void release();
};

struct AmgSolver;
struct Case;

// Raw pointer bundles handed to kernels by value.
struct MeshView {
  int Nc, F, Fi, Fb, nnz;
  const int *owner, *neigh, *cfStart, *cfFace, *rowptr, *col, *bPatch;
  const double *Sx, *Sy, *Sz, *area, *CNx, *CNy, *CNz, *eCx, *eCy, *eCz, *gDiff, *Tx, *Ty, *Tz, *gf, *wd, *vol;
  const int *ptype, *pstart, *pcount, *bcU, *bcP;
  const double* pnsum;
};

struct FieldView {
  int rowsU;
  double *U0, *U1, *U2;
  double* gU[9];  // gradient of U: gU[c * 3 + d] = dU_c / dx_d
  double *p, *gp0, *gp1, *gp2, *PP, *gPP0, *gPP1, *gPP2;
  double *DU0, *DU1, *DU2, *mdot, *fC1, *fC2;
  const double *vU0, *vU1, *vU2, *vP;  // boundary values (per boundary face)
  double* tmp3;                        // [Fb][3] staging for outlet velocity rows
  double* uft;                         // [3][7][F] per-face momentum terms of each component
};

// Per-case descriptor read by the batched kernels. A stage kernel is launched over a
// work list of (slot, block) pairs, so one launch advances every resident case; a single
// case is a one-slot table. Per-slot scalars that kernels produce live in `scal`.
struct SlotDesc {
  MeshView m;
  FieldView f;
  double nu, urf_u, urf_p, fdt;
  int quirks, fixed, rowsU, pad;
  double *ac, *bc, *anb, *dphi;  // level-0 system (cconn-ordered CSR over m.rowptr / m.col)
  double* scal;                  // SCAL_* entries below
  int* flags;                    // FLAG_* entries below
};
enum { SCAL_SCALE = 0, SCAL_RMS = 1, SCAL_MAX = 2, SCAL_MINMAX = 3, SCAL_N = 8 };
enum { FLAG_ZERO_DIAG = 0, FLAG_BAD_BC = 1, FLAG_N = 4 };

// (slot, block) work lists of one case, per domain
struct WorkLists {
  DArr<int2> cells, faces, bfaces, urows;
  int ncells = 0, nfaces = 0, nbfaces = 0, nurows = 0, urows_for = -1;
  DArr<int> cstart, cend, ustart, uend;  // per slot: range of its entries in `cells` / `urows`
};

// Everything a batched stage launch needs: the slot table and the work lists.
struct BatchLaunch {
  const SlotDesc* slots;
  const int2* wc; int nwc;   // cells
  const int2* wf; int nwf;   // faces
  const int2* wb; int nwb;   // boundary faces
  const int2* wu; int nwu;   // rows of U (for the scale)
  const int* cstart; const int* cend;
  const int* ustart; const int* uend;
  int nslots;
  double* part;              // block partials, >= 2 * max(nwc, nwu) entries
  cudaStream_t st;
  // optional (host): vel_mask[3 * ip + mode - 1] != 0 when some slot's patch ip has work in
  // boundary-velocity correction mode `mode`; launches without work are skipped
  const unsigned char* vel_mask = nullptr;
};

struct Case {
  ufvm_settings S{};
  DMesh M;
  DPatch D;
  HPatch P;
  cudaStream_t stream = nullptr;
  bool owns_stream = true;
  // host copies of the topology (setup only)
  std::vector<int> h_cfStart, h_cfFace, h_rowptr, h_col, h_ownSlot, h_neiSlot;
  // fields
  int rowsU = 0, rowsUcap = 0, q12_max_row = -1;
  DArr<double> U[3], gU[9], p, gp[3], PP, gPP[3], DU[3], mdot, fC1, fC2, vU[3], vP, tmp3, uft;
  double scaleU = 1.0;
  // linear systems / hierarchy
  std::vector<Level> lev;
  int n_levels = 1;      // number of levels in use (coarsest = n_levels - 1)
  int p_solves = 0;      // for hierarchy reuse
  bool hierarchy_valid = false;
  // scratch
  LinCtx lin;
  AmgSolver* amg = nullptr;
  DArr<double> part, red;
  DArr<int> flags;
  DArr<double> scal;
  DArr<SlotDesc> slot;   // one-entry table for this case
  WorkLists wl;
  int nsm = 148;
  int last_amg_cycles = 0;
  long long dev_bytes = 0;  // device memory this case holds (the service's admission accounting)

  MeshView mv() const;
  FieldView fv();
  SlotDesc desc();
  int sync_slot();
  BatchLaunch batch();

  template <typename T>
  int up(DArr<T>& a, const T* h, size_t n) {
    UFVM_CHECK(dalloc(a, std::max<size_t>(n, 1)));
    if (n) UFVM_CUDA(cudaMemcpyAsync(a.p, h, n * sizeof(T), cudaMemcpyHostToDevice, stream));
    return UFVM_OK;
  }

  int build_mesh(const ufvm_mesh_desc* d);
  int init_fields(const int32_t* bcu, const int32_t* bcp, const double* vu, const double* vp, const double* U0,
                  const double* p0, const double* mdot0);
  int update_fields();
  int assemble_u(int comp, double* rms, double* mx);
  int assemble_p(double* rms, double* mx);
  int solve(int eq, double* r0, double* r1);
  int correct_u(int comp);
  int correct_p();
  int iterate(double* res, int* converged);
  int fresh_level0();
  ~Case();
};

int create_case_into(Case& C, const ufvm_mesh_desc* mesh, const ufvm_settings& settings, const int32_t* bc_type_u,
                     const int32_t* bc_type_p, const double* bc_val_u, const double* bc_val_p, const double* U0,
                     const double* p0, const double* mdot0, cudaStream_t shared);

}  // namespace ufvm
