// ufvm_oracle.h -- TEST INFRASTRUCTURE ONLY.
//
// A single-thread FP64 C++ restatement of uFVM's steady SIMPLE + agglomeration-AMG
// path (en9apr/Matlab_uFVM, src/...), used as the parity oracle for the CUDA library.
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it.
// It is never linked into the product library and never used as a fallback.
//
// Operation order inside every floating-point expression follows the MATLAB source
// (left-to-right, no fused multiply-add: build with -ffp-contract=off) so that the
// CUDA kernels, compiled with --fmad=false and the same order, agree bit for bit.
#pragma once
#include <cstdint>

#ifdef __cplusplus
extern "C" {
#endif

// Quirk toggles: bit set = reproduce the reference's behaviour, bit clear = repaired.
enum {
  ORQ_Q1_VEC_BOUNDARY_COMPONENT = 1 << 0,  // cfdComputeGradientGauss0.m:57,62; cfdUpdateGradient.m:189,248
  ORQ_Q2_STRESS_NOT_TRANSPOSED  = 1 << 1,  // cfdAssembleExplicitStressTerm.m:15-22,47
  ORQ_Q3_NOSLIP_GAMMA_TWICE     = 1 << 2,  // cfdAssembleDiffusionTerm.m:535-551 + cfdGetUCoef.m:41-44
  ORQ_Q4_GRAD_WEIGHTS_SWAPPED   = 1 << 3,  // cfdInterpolateGradientsFromElementsToInteriorFaces.m:25-27,48-50
  ORQ_Q5_ROUGH_CENTRE           = 1 << 4,  // cfdProcessOpenFoamMesh.m:70-71
  ORQ_Q6_COARSE_DPHI_KEPT       = 1 << 5,  // cfdCorrectFinerLevelSolution.m:11-14
  ORQ_Q7_ILU_SKIP_ROW           = 1 << 6,  // cfdFactorizeILU.m:21
  ORQ_Q12_OUTLET_U_FACE_ROWS    = 1 << 7,  // cfdCorrectVelocityField.m:267-269
  ORQ_Q14_NOSLIP_PATCH_SUM      = 1 << 8,  // cfdAssembleDiffusionTerm.m:535,541,547 dot() of row vectors
  ORQ_Q15_NOSLIP_THIRD_SIGN     = 1 << 9,  // cfdAssembleDiffusionTerm.m:539,545,551 minus on 3rd term
  ORQ_Q16_ONE_CELL_COARSEST     = 1 << 10, // cfdAgglomerate.m:14 keeps a 1-parent level (singular)
  ORQ_ALL = (1 << 11) - 1
};

// Physical patch types (constant/polyMesh/boundary 'type').
enum { ORP_WALL = 0, ORP_INLET = 1, ORP_OUTLET = 2, ORP_SYMMETRY = 3, ORP_EMPTY = 4 };
// Boundary-condition types (0/<field> boundaryField 'type').
enum { ORB_FIXED_VALUE = 0, ORB_ZERO_GRADIENT = 1, ORB_NOSLIP = 2, ORB_SLIP = 3,
       ORB_EMPTY = 4, ORB_SYMMETRY = 5 };
// Smoothers / cycles.
enum { ORS_ILU = 0, ORS_SOR = 1, ORS_MCGS = 2 };
enum { ORC_V = 0, ORC_W = 1, ORC_F = 2 };

// Mesh: raw polyMesh (0-based) -> processed geometry (cfdProcessOpenFoamMesh).
void* orc_mesh_create(int nPoints, const double* points, int nFaces, const int* faceStart,
                      const int* faceNodes, int nInterior, const int* owner, const int* neighbour,
                      int nPatches, const int* patchType, const int* patchStart, const int* patchN,
                      int quirks);
void orc_mesh_destroy(void* m);
// sizes[0..3] = Nc, F, Fi, nnz
void orc_mesh_sizes(void* m, int* sizes);
// name in: Sf centroid_f area CN eCN gDiff T gf walldist volume centroid_c
// (vectors are written as [n][3]); int arrays: rowptr col own_slot nei_slot cell_face_start cell_faces
int orc_mesh_get(void* m, const char* name, void* out);

// Case settings (flat arrays so ctypes needs no struct layout).
// iset: [0]=nCorrectors [1]=fixedElement(0-based,-1 none) [2]=p cycle [3]=p maxCycles
//       [4]=p maxCoarseLevels [5]=p preSweep [6]=p postSweep [7]=p smoother [8]=U smoother
//       [9]=U nIter [10]=quirks [11]=p uses AMG (1) or plain smoother (0)
// dset: [0]=nu [1]=urfU [2]=urfP [3]=tolU [4]=tolP [5]=p termination rrf [6]=U rrf [7]=false dt
void* orc_case_create(void* mesh, const int* iset, const double* dset,
                      const int* bcTypeU, const int* bcTypeP,
                      const double* bcValU /*[Fb][3]*/, const double* bcValP /*[Fb]*/,
                      const double* U0 /*[Nc][3] or null*/, const double* p0 /*[Nc] or null*/,
                      const double* mdot0 /*[F] or null*/);
void orc_case_destroy(void* c);
// One steady SIMPLE iteration (cfdRunCase.m:92-142). res[0..3] = rms U1 U2 U3 p,
// res[4..7] = max, res[8..11] = linear-solver initial, res[12..15] = final.
// Returns 0 ok, 1 converged, -1 NaN detected, <-1 error.
int orc_case_iterate(void* c, double* res);
// Stage-level entry points for kernel parity.
void orc_update_fields(void* c);                               // cfdUpdateFields
int orc_assemble_u(void* c, int comp, double* rms, double* mx); // cfdAssembleEquation('U',comp)
int orc_assemble_p(void* c, double* rms, double* mx);           // cfdAssembleEquation('p')
int orc_solve(void* c, int eq, double* r0, double* r1);         // cfdSolveEquation (0=U,1=p)
void orc_correct_u(void* c, int comp);                         // cfdCorrectEquation('U',comp)
void orc_correct_p(void* c);                                   // cfdCorrectEquation('p')
// name: U gradU p gradp PP gradPP DU mdot gammaU fluxC1 fluxC2 ac bc anb dphi
int orc_case_get(void* c, const char* name, double* out, int* n);
int orc_case_set(void* c, const char* name, const double* in);
int orc_case_nlevels(void* c);
// level >= 1: coarse level of the last AMG build. ints: parents (0-based), rowptr, col
int orc_level_get(void* c, int level, const char* name, void* out, int* n);

// Stand-alone linear algebra on a CSR matrix in cconn order (cfdSetupCoefficients layout).
void orc_residuals(int n, const int* rowptr, const int* col, const double* ac, const double* anb,
                   const double* bc, const double* dphi, double* r);
void orc_sor_sweep(int n, const int* rowptr, const int* col, const double* ac, const double* anb,
                   const double* bc, double* dphi);
void orc_ilu_factor(int n, const int* rowptr, const int* col, const double* ac, const double* anb,
                    double* dc, int quirks);
void orc_ilu_sweep(int n, const int* rowptr, const int* col, const double* ac, const double* anb,
                   const double* bc, const double* dc, double* dphi);
void orc_mcgs_sweep(int n, const int* rowptr, const int* col, const double* ac, const double* anb,
                    const double* bc, const int* color, int ncolor, double* dphi);
int orc_coloring(int n, const int* rowptr, const int* col, int* color);
void orc_solve_algebraic_system(int n, const int* rowptr, const int* col, const double* ac,
                                const double* anb, const double* bc, double* dphi, int smoother,
                                int nIter, double rrf, int quirks, double* r0, double* r1, int* iters);
// Agglomerate one level (cfdAgglomerateLevel + assembleAgglomeratedLHS).
// Outputs parents (0-based), coarse CSR (crowptr size nc+1, ccol/canb capacity nnz), cac.
int orc_agglomerate(int n, const int* rowptr, const int* col, const double* ac, const double* anb,
                    int* parents, int* crowptr, int* ccol, double* cac, double* canb, int* cnnz);

#ifdef __cplusplus
}
#endif
