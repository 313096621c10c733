/* ufvm.h -- C ABI of libufvm.so, the CUDA (sm_100a) implementation of uFVM's steady
 * SIMPLE hot path: Gauss gradients, face-loop momentum assembly, Rhie-Chow face mass
 * flux, pressure-correction assembly, the agglomeration-AMG solve with ILU / Gauss-Seidel
 * smoothers, and the field corrections.
 *
 * Each entry point names the uFVM function (en9apr/Matlab_uFVM, uFVM/src/...) whose
 * behaviour it reproduces. uFVM binds functions by MATLAB path and keeps state in the
 * global `Domain` struct; here the state is an opaque, device-resident case handle.
 *
 * Conventions: plain C types only; indices are 0-based (MATLAB's are 1-based); host
 * pointers unless a parameter is documented as a device pointer; every function returns
 * a ufvm_status and, on error, ufvm_last_error() gives the message (the analogue of the
 * reference's error('...') strings). One GPU, one host thread per case handle.
 */
#ifndef UFVM_H
#define UFVM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  UFVM_OK = 0,
  UFVM_E_INVALID = 1,         /* bad argument / unknown field name */
  UFVM_E_CUDA = 2,            /* CUDA runtime error (message in ufvm_last_error) */
  UFVM_E_OOM = 3,             /* device allocation failed */
  UFVM_E_NAN = 4,             /* NaN residual: cfdRunCase.m:124-127 "Divergence detected!" */
  UFVM_E_ZERO_DIAG = 5,       /* ac == 0: cfdComputeNormalizedResidual.m:77-81 */
  UFVM_E_BC_UNSUPPORTED = 6,  /* BC combination the reference does not implement */
  UFVM_E_AMG_LEVELS = 7,      /* W/F cycle needs >= 4 levels: cfdApplyWCycle.m indexes level 0 */
  UFVM_E_TIMEOUT = 8,         /* a bounded device-side wait gave up */
  UFVM_E_NOT_CONVERGED = 9    /* ufvm_run_case reached max_iter */
} ufvm_status;

/* physical patch types (constant/polyMesh/boundary) */
enum { UFVM_PATCH_WALL = 0, UFVM_PATCH_INLET = 1, UFVM_PATCH_OUTLET = 2, UFVM_PATCH_SYMMETRY = 3,
       UFVM_PATCH_EMPTY = 4 };
/* boundary-condition types (0/U, 0/p boundaryField) */
enum { UFVM_BC_FIXED_VALUE = 0, UFVM_BC_ZERO_GRADIENT = 1, UFVM_BC_NOSLIP = 2, UFVM_BC_SLIP = 3,
       UFVM_BC_EMPTY = 4, UFVM_BC_SYMMETRY = 5 };
/* smoothers: 'ILU' (DILU), 'SOR' (symmetric Gauss-Seidel, natural order), multicolour GS */
enum { UFVM_SMOOTHER_ILU = 0, UFVM_SMOOTHER_SOR = 1, UFVM_SMOOTHER_MCGS = 2 };
enum { UFVM_CYCLE_V = 0, UFVM_CYCLE_W = 1, UFVM_CYCLE_F = 2 };
enum { UFVM_EQ_U = 0, UFVM_EQ_P = 1 };
/* arithmetic of the pressure-correction AMG */
enum { UFVM_PREC_FP64 = 0, UFVM_PREC_FP32_AMG = 1 };

/* Reference-defect toggles: bit set = reproduce the reference, bit clear = repaired. */
#define UFVM_Q1_VEC_BOUNDARY_COMPONENT (1 << 0)  /* cfdComputeGradientGauss0.m:57,62 */
#define UFVM_Q2_STRESS_NOT_TRANSPOSED  (1 << 1)  /* cfdAssembleExplicitStressTerm.m:15-22 */
#define UFVM_Q3_NOSLIP_GAMMA_TWICE     (1 << 2)  /* cfdAssembleDiffusionTerm.m:535-551, cfdGetUCoef.m:41-44 */
#define UFVM_Q4_GRAD_WEIGHTS_SWAPPED   (1 << 3)  /* cfdInterpolateGradientsFromElementsToInteriorFaces.m:25-27 */
#define UFVM_Q5_ROUGH_CENTRE           (1 << 4)  /* cfdProcessOpenFoamMesh.m:70-71 */
#define UFVM_Q6_COARSE_DPHI_KEPT       (1 << 5)  /* cfdCorrectFinerLevelSolution.m:11-14 */
#define UFVM_Q7_ILU_SKIP_ROW           (1 << 6)  /* cfdFactorizeILU.m:21 */
#define UFVM_Q12_OUTLET_U_FACE_ROWS    (1 << 7)  /* cfdCorrectVelocityField.m:267-269 */
#define UFVM_Q14_NOSLIP_PATCH_SUM      (1 << 8)  /* cfdAssembleDiffusionTerm.m:535,541,547 */
#define UFVM_Q15_NOSLIP_THIRD_SIGN     (1 << 9)  /* cfdAssembleDiffusionTerm.m:539,545,551 */
#define UFVM_Q16_ONE_CELL_COARSEST     (1 << 10) /* cfdAgglomerate.m:14 */
#define UFVM_QUIRKS_REFERENCE          ((1 << 11) - 1)

/* Raw OpenFOAM polyMesh (what cfdReadPolyMesh.m:17-214 reads), 0-based, host memory. */
typedef struct {
  int32_t n_points;
  const double* points;        /* [n_points][3] */
  int32_t n_faces;
  const int32_t* face_start;   /* [n_faces + 1] offsets into face_nodes */
  const int32_t* face_nodes;
  int32_t n_interior;
  const int32_t* owner;        /* [n_faces] */
  const int32_t* neighbour;    /* [n_interior] */
  int32_t n_patches;
  const int32_t* patch_type;   /* UFVM_PATCH_* */
  const int32_t* patch_start;
  const int32_t* patch_n;
} ufvm_mesh_desc;

/* Settings read by uFVM from system/fvSolution, transportProperties and run.m
 * (cfdReadSystem.m:119-252, cfdSetupAMG.m:6-20, cfdSetupSolutionMethods.m:6-14). */
typedef struct {
  int32_t n_correctors;        /* SIMPLE.nCorrectors */
  int32_t fixed_element;       /* pRefCell (0-based), -1: none */
  int32_t p_cycle;             /* UFVM_CYCLE_* */
  int32_t p_max_cycles;        /* 30 */
  int32_t p_max_coarse_levels; /* 10 */
  int32_t p_pre_sweep;         /* 1 */
  int32_t p_post_sweep;        /* 3 */
  int32_t p_smoother;          /* UFVM_SMOOTHER_* */
  int32_t u_smoother;          /* UFVM_SMOOTHER_* */
  int32_t u_n_iter;            /* 10 (cfdSolver.m:12) */
  int32_t quirks;              /* UFVM_Q* bits */
  int32_t p_amg;               /* 1: cfdApplyAMG, 0: cfdSolver */
  int32_t precision;           /* UFVM_PREC_* */
  int32_t hierarchy_reuse;     /* 0: rebuild the AMG hierarchy every p solve (reference);
                                  k > 0: rebuild the agglomeration every k solves */
  int32_t p_krylov;            /* service p solve: 0 plain iterative refinement (x += V(r));
                                  1 flexible CG (FCG(1)) with the FP32 V-cycle as preconditioner */
  int32_t service_eager;       /* service tick: 0 replays one captured CUDA graph per tick, with the
                                  solve loops ended on the device; 1 launches every kernel from the host */
  double nu;                   /* transportProperties nu */
  double urf_u, urf_p;         /* relaxationFactors */
  double tol_u, tol_p;         /* residualControl */
  double p_termination;        /* AMG termination (rrf) 0.1 */
  double u_rrf;                /* 0.1 */
  double false_dt;             /* 1e9 (cfdSetupTime.m:37) */
  double p_coarse_weight;      /* service V-cycle: the prolongated coarse-grid correction is scaled
                                  by this weight (over-correction of the piecewise-constant
                                  prolongation); 0 or 1: unscaled, as cfdCorrectFinerLevelSolution.m */
} ufvm_settings;

typedef struct ufvm_case ufvm_case;

/* Creates a device-resident case: processes the mesh on the GPU
 * (cfdProcessOpenFoamMesh.m:15-243), sets boundary values and initial fields
 * (cfdInitializeCase.m:14-83, cfdInitializeMdotField.m:72-86).
 * bc_type_*: per patch UFVM_BC_*; bc_val_u [n_bfaces][3], bc_val_p [n_bfaces];
 * U0 [n_cells][3], p0 [n_cells], mdot0 [n_faces] may be NULL (zero / computed). */
int ufvm_case_create(const ufvm_mesh_desc* mesh, const ufvm_settings* settings,
                     const int32_t* bc_type_u, const int32_t* bc_type_p,
                     const double* bc_val_u, const double* bc_val_p,
                     const double* U0, const double* p0, const double* mdot0,
                     ufvm_case** out);
int ufvm_case_destroy(ufvm_case* c);
/* sizes[0..3] = n_cells, n_faces, n_interior, nnz (2 * n_interior) */
int ufvm_case_sizes(const ufvm_case* c, int64_t* sizes);

/* cfdUpdateFields (update/cfdUpdateFields.m:17-27). */
int ufvm_update_fields(ufvm_case* c);
/* [rms, max] = cfdAssembleEquation(name, iComponent) (assemble/cfdAssembleEquation.m:1);
 * eq = UFVM_EQ_U (comp 0..2) or UFVM_EQ_P. */
int ufvm_assemble_equation(ufvm_case* c, int eq, int comp, double* rms, double* max);
/* [r0, r1] = cfdSolveEquation(name) (solve/cfdSolveEquation.m:1). */
int ufvm_solve_equation(ufvm_case* c, int eq, double* r0, double* r1);
/* cfdCorrectEquation(name, iComponent) (solve/correct/cfdCorrectEquation.m:1). */
int ufvm_correct_equation(ufvm_case* c, int eq, int comp);
/* One steady iteration of cfdRunCase (top/cfdRunCase.m:92-142). res[16]: rms U1 U2 U3 p,
 * max (4), linear-solver initial (4), final (4). Returns UFVM_OK, UFVM_E_NAN, ... and sets
 * *converged per cfdCheckConvergence.m:3-20. */
int ufvm_simple_iteration(ufvm_case* c, double* res, int* converged);
/* cfdRunCase: iterate until converged or max_iter. */
int ufvm_run_case(ufvm_case* c, int max_iter, int* iterations, double* res);

/* Field access (host copies). Names: U (3 x rows), gradU (9 x rows), p, gradp (3 x rows),
 * PP, gradPP, DU (3 x rows), mdot (n_faces), gammaU, fluxC1, fluxC2, ac, bc, anb, dphi,
 * scaleU. n = number of doubles in the buffer; the call fails if it is too small. */
int ufvm_get_field(ufvm_case* c, const char* name, double* host, int64_t n, int64_t* written);
int ufvm_set_field(ufvm_case* c, const char* name, const double* host, int64_t n);
/* Processed geometry (same names as the theMesh struct): Sf centroid_f area CN eCN gDiff T gf
 * walldist volume centroid_c (vectors as [n][3]). */
int ufvm_get_geometry(ufvm_case* c, const char* name, double* host, int64_t n);
/* AMG hierarchy of the last p solve: number of levels, per-level sizes and the
 * cell-to-coarse maps (cfdAgglomerateLevel.m `parents`, 0-based). */
int ufvm_get_levels(ufvm_case* c, int* n_levels, int64_t* sizes, int max_levels);
int ufvm_get_level_array(ufvm_case* c, int level, const char* name, void* host, int64_t n,
                         int64_t* written);  /* parents rowptr col ac anb color (int32 / double) */

/* ---- stand-alone matrix kernels on DEVICE pointers (cconn-ordered CSR: row i holds the
 * coefficients anb{i} of setup/cfdSetupCoefficients.m in cconn{i} order) ---- */
/* r = cfdComputeResidualsArray(coefficients) (compute/cfdComputeResidualsArray.m:9-17) */
int ufvm_compute_residuals_array(int32_t n, const int32_t* rowptr, const int32_t* col,
                                 const double* ac, const double* anb, const double* bc,
                                 const double* dphi, double* r, void* stream);
/* dphi = cfdSolveSOR(...) one symmetric natural-order Gauss-Seidel sweep (solve/cfdSolveSOR.m). */
int ufvm_solve_sor(int32_t n, const int32_t* rowptr, const int32_t* col, const double* ac,
                   const double* anb, const double* bc, double* dphi, void* stream);
/* ufvm_solve_sor without any device allocation. No counterpart in the reference: it exists for
 * callers that cannot allocate device memory when they call the smoother (a MEX gateway inside
 * a caller-owned device-memory budget, an application whose pool allocator owns all device
 * memory, or pipelined code that must not hit cudaMalloc's implicit synchronisation). All of
 * its scratch lives in one fixed array of about 4 MiB compiled into the library, so systems of
 * more than 262,144 rows are rejected with UFVM_E_INVALID. Every call shares that array and
 * clears what it needs; calls whose device work overlaps race on it and must be serialised.
 * The matrix must be structurally symmetric (every finite-volume matrix is), as for
 * ufvm_solve_sor: the level schedule is built from each row's lower neighbours.
 * Every call synchronises its stream (it reads the level schedule's size back to the host), so
 * it cannot be captured into a CUDA graph. Results are bit-identical to ufvm_solve_sor's. */
int ufvm_solve_sor_noalloc(int32_t n, const int32_t* rowptr, const int32_t* col, const double* ac,
                           const double* anb, const double* bc, double* dphi, void* stream);
/* [dc] = cfdFactorizeILU and dphi = cfdSolveILU (solve/cfdFactorizeILU.m, cfdSolveILU.m). */
int ufvm_factorize_ilu(int32_t n, const int32_t* rowptr, const int32_t* col, const double* ac,
                       const double* anb, double* dc, int32_t quirks, void* stream);
int ufvm_solve_ilu(int32_t n, const int32_t* rowptr, const int32_t* col, const double* ac,
                   const double* anb, const double* bc, const double* dc, double* dphi,
                   void* stream);
/* [r0, r1] = cfdSolveAlgebraicSystem(level, smoother, nIter, rrf) on one matrix
 * (solve/cfdSolveAlgebraicSystem.m:11-66); r0/r1/iters are host outputs. */
int ufvm_solve_algebraic_system(int32_t n, const int32_t* rowptr, const int32_t* col,
                                const double* ac, const double* anb, const double* bc,
                                double* dphi, int32_t smoother, int32_t n_iter, double rrf,
                                int32_t quirks, double* r0, double* r1, int32_t* iters,
                                void* stream);
/* Kernel timing of the stand-alone solver kernels on one system (no reference counterpart:
 * the measurement behind the plain form's roofline). kernel 0: residual r = b - A x;
 * 1: one symmetric natural-order Gauss-Seidel sweep (level scheduled, as ufvm_solve_sor);
 * 2: one symmetric multicolour Gauss-Seidel sweep (smoother UFVM_SMOOTHER_MCGS);
 * 3: one DILU application (as ufvm_solve_ilu, factor prepared untimed). Schedules, colourings
 * and the factor are built first and one launch is made untimed; each of the reps timed
 * launches follows a read of twice the L2 size and is bracketed by CUDA events on the stream.
 * ms_per_launch: mean time; bytes_per_launch: algorithmic bytes (36 n + 12 nnz per pass over
 * the system; 2 passes for a symmetric sweep; DILU adds 40 n + 24 nnz). Sweeps overwrite dphi;
 * the call allocates (L2-flush buffer and the schedules). */
int ufvm_profile_plain_kernel(int32_t kernel, int32_t n, const int32_t* rowptr, const int32_t* col,
                              const double* ac, const double* anb, const double* bc, double* dphi,
                              int32_t reps, double* ms_per_launch, double* bytes_per_launch,
                              void* stream);
/* One level of cfdAgglomerateLevel + assembleAgglomeratedLHS (device pointers in, host
 * count out). parents[n]; coarse rowptr[n+1], col/anb capacity rowptr[n] entries, ac[n]. */
int ufvm_agglomerate_level(int32_t n, const int32_t* rowptr, const int32_t* col,
                           const double* ac, const double* anb, int32_t* parents,
                           int32_t* c_rowptr, int32_t* c_col, double* c_ac, double* c_anb,
                           int32_t* n_coarse, int32_t* nnz_coarse, void* stream);

/* ---- batched steady-case service (continuous batching of independent cases) ----
 * Cases are admitted first-come first-served while their HBM footprint fits the memory budget
 * (ufvm_service_set_memory_budget; by default 90% of the device memory free at creation) and
 * their cells fit max_resident_cells. A queued case's footprint is estimated from its face,
 * interior-face and cell counts, scaled by the largest ratio of measured to estimated bytes the
 * service has seen; a resident case counts its measured allocations. A case that fails to
 * allocate at admission waits at the head of the queue while other cases are resident. Every
 * resident case advances one SIMPLE iteration per ufvm_service_step in one launch per stage,
 * and a case finishes when it converges (residualControl), fails, or reaches its iteration
 * limit; its result (U, p, mdot at that iteration) is kept on the device until release. Its slot
 * leaves the batch with the next admission, or when the device time spent on finished slots
 * reaches the host cost of a rebuild, or after 256 steps; its own device memory is freed when an
 * admission needs the room (or at ufvm_service_destroy). The solver settings are shared by all
 * cases of a service; nu, the boundary data and the pressure reference cell are per case (a
 * case whose boundaries are all walls, empty or symmetry planes pins p at settings->
 * fixed_element, or cell 0 if that is negative; any other case has none, cfdReadSystem.m:
 * 238-252). Linear solves: multicolour Gauss-Seidel (FP64) for U, FP32 AMG preconditioning
 * FP64 flexible CG for p (the service requires settings->precision == UFVM_PREC_FP32_AMG). Latencies are device time, summed
 * over the steps a case was resident; queue time is reported separately. */
typedef struct ufvm_service ufvm_service;
int ufvm_service_create(const ufvm_settings* settings, int64_t max_resident_cells, ufvm_service** out);
int ufvm_service_submit(ufvm_service* s, const ufvm_mesh_desc* mesh, double nu, const int32_t* bc_type_u,
                        const int32_t* bc_type_p, const double* bc_val_u, const double* bc_val_p,
                        int32_t max_iter, int64_t* ticket);
int ufvm_service_step(ufvm_service* s, int32_t* n_resident, int32_t* n_queued, int64_t* n_finished_total);
/* state: 0 queued, 1 resident, 2 converged, 3 stopped (not converged or failed; status in *status) */
int ufvm_service_status(ufvm_service* s, int64_t ticket, int32_t* state, int32_t* status, int32_t* iterations,
                        double* res16, double* latency_ms, double* queue_ms);
int ufvm_service_get_field(ufvm_service* s, int64_t ticket, const char* name, double* host, int64_t n,
                           int64_t* written);
int ufvm_service_release(ufvm_service* s, int64_t ticket);
/* Accumulated device time (ms) per phase of the eagerly launched ticks -- update fields,
 * U assembly, U solve, U correction, p assembly, AMG hierarchy builds, p solve, p correction --
 * then the number of U smoother sweeps, p V-cycles, steps, the service clock (ms), the ticks
 * replayed as a captured graph, the number of graph captures and the kernel launches executed by
 * the replayed graphs (loop bodies counted per execution), the current CTA threshold of the
 * V-cycle, the number of completed autotuning passes, the HBM bytes held by the slots and the
 * unreleased results, the memory budget, the admissions deferred for memory, the admissions
 * that failed to allocate and were re-queued, the departures of finished slots from the batch,
 * the footprint estimate's scale, the U-smoother and p-cycle loop bodies the replayed ticks
 * have run, the host time (ms) spent rebuilding slot tables, capturing tick graphs and
 * freeing departed cases, the wall time (ms) of AMG hierarchy builds, the host time (ms) summed
 * over the build threads in agglomeration, in colourings and FP32 arrays, in the ELL permutation
 * and, of these, in device allocation calls, and the host time (ms) of admissions. Writes
 * min(n, 34) values. */
int ufvm_service_stats(ufvm_service* s, double* out, int n);
/* Admits queued cases now, as far as the budgets allow, without waiting for the next step: their
 * meshes are uploaded and processed on the service stream, so a caller can have a batch resident
 * on the device before it starts timing or stepping. *n_resident: active cases afterwards. */
int ufvm_service_admit(ufvm_service* s, int32_t* n_resident);
/* Fault injection for tests (no counterpart in the reference): the next `count` admissions of
 * `ticket` fail as if a device allocation had failed (UFVM_E_OOM), without allocating. While
 * other cases are resident such a request waits at the head of the queue; on an empty service
 * it is stopped with UFVM_E_OOM. */
int ufvm_service_inject_admit_oom(ufvm_service* s, int64_t ticket, int32_t count);
/* HBM budget (bytes) of the resident cases plus the unreleased results (admission control). */
int ufvm_service_set_memory_budget(ufvm_service* s, int64_t bytes);
/* Tickets that finished (converged, stopped or failed) since the previous poll, oldest first:
 * writes min(capacity, pending) of them and their count; the rest stay for the next poll. */
int ufvm_service_poll(ufvm_service* s, int64_t* tickets, int64_t capacity, int64_t* n_out);
/* Queued cases are admitted at most every `steps` steps (default 8) unless the resident cells
 * fall to half the budget; a case's first step builds its AMG hierarchy and is launched
 * kernel by kernel, so gathering admissions keeps the other steps on the captured graph. */
int ufvm_service_set_admit_interval(ufvm_service* s, int32_t steps);
/* Launch schedule of the p solve's V-cycle: AMG levels of at most cta_rows rows are smoothed
 * by one thread block per case (all of a case's small levels in one launch), larger levels by
 * grid-wide launches over all cases. packed 1 (default) packs up to four small cases into one
 * 1024-thread block (256 threads and a named barrier each) and gives a large case a whole
 * block; 0 runs one block per case. By default an autotuner picks cta_rows by timing the
 * candidates 2048 .. 65536 on the live batch (re-tuned every 2000 steps); a positive cta_rows
 * fixes the schedule, 0 hands it back to the autotuner. The schedule changes no result. */
int ufvm_service_set_schedule(ufvm_service* s, int32_t cta_rows, int32_t packed);
/* The CUDA stream (cudaStream_t) on which the service issues all of its device work, so a
 * caller can order its own work or timing events after a step. No counterpart in the
 * reference (its solves are synchronous MATLAB calls). */
int ufvm_service_stream(ufvm_service* s, void** stream);
/* Measurement hook (no counterpart in the reference): times one kernel of the tick on the
 * current resident batch, reps times, and returns the average device time (ms) of one unit and
 * its compulsory DRAM bytes. kernel 0: one symmetric FP64 multicolour Gauss-Seidel sweep of
 * every case's level 0 (the U smoother); 1: the same sweep in FP32 on the V-cycle's level 0;
 * 2: the FP64 product q = A p of the flexible CG; 3: the momentum assembly of one component;
 * 4: the pressure-correction assembly (Rhie-Chow face flux and the p matrix); 5: the field
 * update (boundary values, Gauss gradients of U and p); 6: one pass of the per-case coarse
 * V-cycle kernel (latency-bound). The sweeps overwrite the correction vectors, which the next
 * step's assembly resets, so call it between steps; kernels 3-5 recompute matrices and fields
 * from the current state (4 also advances the face mass flux): use them on a batch kept only
 * for timing. */
int ufvm_service_profile(ufvm_service* s, int32_t kernel, int32_t reps, double* ms_per_unit,
                         double* bytes_per_unit);
int ufvm_service_destroy(ufvm_service* s);

const char* ufvm_last_error(void);
const char* ufvm_version(void);

#ifdef __cplusplus
}
#endif
#endif /* UFVM_H */
