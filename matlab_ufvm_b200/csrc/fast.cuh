// fast.cuh -- the batched service: many resident cases advance together, one launch per
// stage; U is smoothed with FP64 multicolour Gauss-Seidel and p is solved with FP32 AMG
// V-cycles inside FP64 iterative refinement (FP64 residual r = b - A x, FP64 update).
#pragma once
#include "amg.cuh"
#include "simple.cuh"

namespace ufvm {

// One (slot, AMG level) of the batched hierarchy.
struct LevDesc {
  int n, nnz, ncolor, coarsest;
  const int *rowptr, *col;
  double *ac64, *anb64;          // FP64 values (Galerkin source, coarsest direct solve)
  float *ac, *anb, *bc, *x, *r;  // FP32 smoother arrays
  const int* parents;            // this level -> next coarser level
  const int *childStart, *child; // children in this level of each next-level row
  const int *colorRows, *colorStart;
  double *fr, *fp, *fq;          // level 0 only: FP64 flexible-CG vectors
  // colour-permuted ELL storage of the FP32 arrays (pmode 1, every level but the coarsest);
  // ac, bc, x, r are then indexed by position
  int pmode, ellW;
  const int *perm, *inv, *ellCol, *parentsP, *childP, *childStartP;
  float* ellAnb;
  double *uAnb, *uAc, *uBc, *uX;  // level 0, pmode: FP64 ELL copy of the momentum matrix
  const int* gpos;                // pmode: Galerkin target of each fine entry (-1: in the aggregate)
  float pw;                       // weight of the prolongated coarse correction
};

// Packed coarse V-cycle: CTAs of kBlockPack threads; a task gives one large case the whole
// CTA or each of kPackGroups thread groups its own small case (slot -1: none).
constexpr int kBlockPack = 1024;
constexpr size_t kBuildThreads = 16;  // host threads that build new cases' AMG hierarchies
constexpr int kPackGroups = 4;
struct PackTask {
  int big;
  int slot[kPackGroups];
};

// A self-contained work item of the level-0 FP32 Gauss-Seidel (colour-permuted ELL): up to
// kBlock rows p0 .. p0 + cnt - 1 of one case's level 0, with that level's arrays.
struct L0Item {
  int slot, p0, cnt, n, W, pad0;
  float* x;
  const float *bc, *ac;
  const int* ellCol;
  const float* ellAnb;
};

// The same for the FP64 U smoother on the ELL copy of the momentum matrix.
struct U0Item {
  int slot, p0, cnt, n, W, pad0;
  double* x;
  const double *bc, *ac, *anb;
  const int* ellCol;
};

// Per-slot control state of the batched linear solves (device resident).
struct SolveCtl {
  double r0, r1;
  int iters, active;
};

enum { SCAL_U_RMS = 4, SCAL_P_RMS = 7, SCAL_U_MAX = 8, SCAL_P_MAX = 11, SCAL_U_R0 = 12, SCAL_P_R0 = 15,
       SCAL_U_R1 = 16, SCAL_P_R1 = 19, SCAL_CYC = 20, SCAL_SLOT_N = 24 };

struct Service {
  ufvm_settings S{};
  cudaStream_t stream = nullptr;
  int nsm = 148;
  std::vector<Case*> cases;        // resident slots (owned)
  std::vector<long long> tickets;  // caller ids per slot
  bool tables_dirty = true;
  int Lmax = 1;
  // device tables and work lists
  DArr<SlotDesc> slotTab;
  DArr<LevDesc> levTab;            // [Lmax][nslots]
  DArr<double> scal;               // [nslots][SCAL_SLOT_N]
  DArr<int> flags;                 // [nslots][FLAG_N]
  DArr<SolveCtl> uctl, pctl;
  DArr<double> part;
  DArr<double> fcg;                // flexible-CG block partials and per-slot sums
  DArr<int2> wc, wf, wb, wu;
  int nwc = 0, nwf = 0, nwb = 0, nwu = 0;
  DArr<int> cstart, cend, ustart, uend;
  // AMG work lists. A slot's levels 0 .. g-1 run as grid-wide launches (smoothing, residual,
  // restriction, prolongation), its levels g .. coarsest inside one CTA (k_coarse_vcycle).
  // wrows[l]: rows of level l (all slots that have level l); wsm[l]: smoothing rows of level l
  // by colour, wnc[l]: rows of level l, wrc[l]: rows of level l + 1, each for slots with l < g.
  std::vector<DArr<int2>> wrows, wsm, wnc, wrc;
  std::vector<int> nwrows, nwsm, nwnc, nwrc;
  int maxg = 0;                      // max over slots of g
  DArr<int> dcoarsest;               // per slot: index of its coarsest level
  DArr<int> dgstart;                 // per slot: g
  std::vector<int> h_gstart, h_coarsest;  // host copies of dgstart / dcoarsest
  DArr<int> dcta_order;              // slots in the CTA order of the coarse V-cycle (largest first)
  DArr<PackTask> dpk_tasks;          // packed tasks of the coarse V-cycle
  std::vector<unsigned char> vel_mask;  // boundary-velocity correction launches with work
  DArr<L0Item> wsm0;                 // level-0 smoothing items (same order as wsm[0])
  bool l0_items = false;
  DArr<U0Item> wu_items;             // U smoothing items (same order as wu_col)
  bool u_items = false;
  DArr<U0Item> wures_items;          // U residual items (same order as wc)
  bool ures_items = false;
  int npk_tasks = 0;
  DArr<double> cinv;                 // per slot: coarsest-level solution operator (64 x 64)
  std::vector<int> maxcol;           // per level: max colours over smoothing slots
  std::vector<std::vector<int>> smoff;  // [level][colour] offset into wsm[level]
  std::vector<std::vector<int>> smcnt;
  DArr<int2> wu_col;                 // level-0 colour rows, all slots, FP64 U smoother
  std::vector<int> ucol_off, ucol_cnt;
  int ucolors = 0;
  LinCtx lin;
  DArr<int> anyflag;
  // per-phase device time (ms) and counters, accumulated over iterate() calls
  enum { PH_UPDATE, PH_ASM_U, PH_SOLVE_U, PH_CORR_U, PH_ASM_P, PH_HIER, PH_SOLVE_P, PH_CORR_P, PH_N };
  double ph_ms[PH_N] = {0};
  long long n_usweeps = 0, n_pcycles = 0, n_iter_calls = 0;
  std::vector<cudaEvent_t> evpool;

  // one tick as a CUDA graph with device-side loop control (conditional WHILE nodes)
  int use_graph = 1;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  bool graph_valid = false;
  cudaStream_t bstream = nullptr;      // loop bodies are captured on this stream
  cudaStream_t main_stream = nullptr;
  long long n_graph_ticks = 0, n_captures = 0;
  // host time (ms) spent rebuilding the slot tables and capturing the tick graph, in total and
  // for the most recent change of the slot set
  double host_rebuild_ms = 0.0, host_capture_ms = 0.0, last_rebuild_ms = 0.0;
  // hierarchy builds: wall ms, and host ms summed over the build threads in agglomeration,
  // colourings and FP32 arrays, ELL permutation, and (part of those) device allocation calls
  double build_wall_ms = 0.0, build_ms[4] = {0.0, 0.0, 0.0, 0.0};
  // kernel launches: kernels of the captured tick outside the loops and per loop body, and
  // the device counters of executed U / p loop bodies
  long long static_kernels = 0, ubody_kernels = 0, pbody_kernels = 0, launches_total = 0;
  std::vector<std::pair<int, cudaGraph_t>> bodies;  // (0 U / 1 p, body graph) of the capture
  DArr<unsigned long long> loopcnt;
  unsigned long long loops_seen[2] = {0, 0};

  // schedule: levels of at most cta_rows rows are smoothed inside the per-case CTA of the coarse
  // V-cycle kernel, larger ones by grid-wide launches over all cases (the autotuner's start: the
  // threshold it kept on the cavity batches)
  int cta_rows = 4096;
  // the coarse V-cycle packs small cases kPackGroups to a CTA (1) or runs one CTA per case (0);
  // a case with more than pk_rows rows below its grid levels gets a whole CTA
  int use_packing = 1;
  int pk_rows = 1024;
  long long n_tunes = 0;

  int rebuild_tables();
  BatchLaunch batch();
  bool needs_hierarchy(const Case& c) const;
  // adds the bytes it allocates to c.dev_bytes, and its host ms (agglomeration, colourings and
  // FP32 arrays, ELL permutation, of these in allocation calls) to ms[0..3]
  int ensure_hierarchy(Case& c, cudaStream_t st, double* ms);
  int ensure_hierarchy_(Case& c, cudaStream_t st, double* ms);
  int build_hierarchies(std::vector<Case*>& need);
  int build_ell(Case& c, cudaStream_t st);
  std::vector<cudaStream_t> build_streams;  // streams of the hierarchy-build threads
  cudaEvent_t build_event = nullptr;
  int loop_begin(int kind, cudaGraphConditionalHandle* h);
  int loop_end();
  int solve_u(bool g);
  int solve_p(bool g);
  int enqueue_tick(bool g, std::vector<std::pair<int, int>>& marks);
  int capture_tick();
  int iterate(std::vector<double>& res_out, std::vector<int>& converged);
  int profile(int kernel, int reps, double* ms, double* bytes);
  ~Service();
};

}  // namespace ufvm
