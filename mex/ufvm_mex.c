/* ufvm_mex.c -- MATLAB MEX gateway to libufvm.so for uFVM's steady SIMPLE path.
 *
 * uFVM binds its functions by MATLAB path (doc/Readme.txt:5, addpath(genpath('.../uFVM/src'))):
 * the shadow functions in mex/gpu/ sit before uFVM on the path, keep the reference's names and
 * signatures, and call this gateway as ufvm_mex('<command>', ...). Every command maps to one
 * entry point of include/ufvm.h; the library's status codes become MATLAB errors with the
 * identifier uFVM:<code name> and ufvm_last_error()'s message, in place of the reference's
 * error('...') strings.
 *
 * Build (MATLAB R2018a or later, interleaved complex API; libufvm.so from
 * python -m matlab_ufvm_b200.build):
 *     mex -R2018a -I../include ufvm_mex.c -L../matlab_ufvm_b200 -lufvm
 * The gpuArray commands (solve_sor, solve_ilu, factorize_ilu, compute_residuals_array,
 * solve_algebraic_system, agglomerate_level) also need the Parallel Computing Toolbox headers:
 *     mex -R2018a -DUFVM_MEX_GPU -I../include ufvm_mex.c -L../matlab_ufvm_b200 -lufvm -lmwgpu
 *
 * Conventions at this boundary:
 *   - case handles are uint64 scalars (the library's ufvm_case pointer), kept in
 *     Domain.gpu.handle by the shadow functions and destroyed by 'case_destroy' or at exit;
 *   - mesh and cell indices arrive 0-based int32 (the shadows convert uFVM's 1-based arrays);
 *   - vector fields are 3 x n double arrays (one column per row of the field);
 *   - the settings arrive as a struct whose field names are those of ufvm_settings; missing
 *     fields take the reference's defaults (ufvm_mex('default_settings') returns them).
 */
#include <stdint.h>
#include <string.h>

#include "mex.h"
#include "ufvm.h"
#ifdef UFVM_MEX_GPU
#include "gpu/mxGPUArray.h"
#endif

#define MAX_HANDLES 4096
static ufvm_case* g_cases[MAX_HANDLES];
static ufvm_service* g_services[MAX_HANDLES];
static int g_exit_registered = 0;

static const char* status_id(int code) {
  switch (code) {
    case UFVM_E_INVALID: return "uFVM:invalid";
    case UFVM_E_CUDA: return "uFVM:cuda";
    case UFVM_E_OOM: return "uFVM:outOfMemory";
    case UFVM_E_NAN: return "uFVM:divergence";
    case UFVM_E_ZERO_DIAG: return "uFVM:zeroDiagonal";
    case UFVM_E_BC_UNSUPPORTED: return "uFVM:boundaryCondition";
    case UFVM_E_AMG_LEVELS: return "uFVM:amgLevels";
    case UFVM_E_TIMEOUT: return "uFVM:timeout";
    case UFVM_E_NOT_CONVERGED: return "uFVM:notConverged";
    default: return "uFVM:error";
  }
}

static void check(int code) {
  if (code != UFVM_OK) mexErrMsgIdAndTxt(status_id(code), "%s", ufvm_last_error());
}

static void at_exit(void) {
  int i;
  for (i = 0; i < MAX_HANDLES; ++i) {
    if (g_cases[i]) { ufvm_case_destroy(g_cases[i]); g_cases[i] = NULL; }
    if (g_services[i]) { ufvm_service_destroy(g_services[i]); g_services[i] = NULL; }
  }
}

static void need_args(int nrhs, int n, const char* cmd) {
  if (nrhs < n) mexErrMsgIdAndTxt("uFVM:invalid", "ufvm_mex('%s'): expected %d arguments", cmd, n - 1);
}

/* ---- argument helpers ---- */
static const double* in_double(const mxArray* a, const char* what, size_t* n) {
  if (!mxIsDouble(a) || mxIsComplex(a)) mexErrMsgIdAndTxt("uFVM:invalid", "%s must be a real double array", what);
  if (n) *n = mxGetNumberOfElements(a);
  return mxGetDoubles(a);
}

static const int32_t* in_int32(const mxArray* a, const char* what, size_t* n) {
  if (!mxIsInt32(a)) mexErrMsgIdAndTxt("uFVM:invalid", "%s must be an int32 array (0-based indices)", what);
  if (n) *n = mxGetNumberOfElements(a);
  return (const int32_t*)mxGetInt32s(a);
}

static const double* opt_double(int nrhs, const mxArray* prhs[], int k) {
  if (k >= nrhs || mxIsEmpty(prhs[k])) return NULL;
  return in_double(prhs[k], "initial field", NULL);
}

static int slot_of(const mxArray* a, void** table, const char* what) {
  uint64_t h;
  int i;
  if (!mxIsUint64(a) || mxGetNumberOfElements(a) != 1) mexErrMsgIdAndTxt("uFVM:invalid", "%s handle must be a uint64 scalar", what);
  h = *(const uint64_t*)mxGetUint64s(a);
  for (i = 0; i < MAX_HANDLES; ++i)
    if (table[i] && (uint64_t)(uintptr_t)table[i] == h) return i;
  mexErrMsgIdAndTxt("uFVM:invalid", "unknown %s handle", what);
  return -1;
}

static ufvm_case* case_of(const mxArray* a) { return g_cases[slot_of(a, (void**)g_cases, "case")]; }
static ufvm_service* service_of(const mxArray* a) { return g_services[slot_of(a, (void**)g_services, "service")]; }

static mxArray* handle_out(void* p) {
  mxArray* o = mxCreateNumericMatrix(1, 1, mxUINT64_CLASS, mxREAL);
  *(uint64_t*)mxGetUint64s(o) = (uint64_t)(uintptr_t)p;
  return o;
}

static void keep(void** table, void* p) {
  int i;
  for (i = 0; i < MAX_HANDLES; ++i)
    if (!table[i]) { table[i] = p; return; }
  mexErrMsgIdAndTxt("uFVM:invalid", "too many open handles");
}

static void forget(void** table, void* p) {
  int i;
  for (i = 0; i < MAX_HANDLES; ++i)
    if (table[i] == p) table[i] = NULL;
}

static int equation_of(const mxArray* a) {
  char name[16];
  mxGetString(a, name, sizeof name);
  if (!strcmp(name, "U")) return UFVM_EQ_U;
  if (!strcmp(name, "p")) return UFVM_EQ_P;
  mexErrMsgIdAndTxt("uFVM:invalid", "unknown equation '%s' (this path solves U and p)", name);
  return -1;
}

/* The reference's defaults (cfdReadSystem.m:119-252, cfdSetupAMG.m:6-20,
 * cfdSetupSolutionMethods.m:6-14, cfdSetupTime.m:37). */
static void default_settings(ufvm_settings* s) {
  memset(s, 0, sizeof *s);
  s->n_correctors = 1; s->fixed_element = -1; s->p_cycle = UFVM_CYCLE_W; s->p_max_cycles = 30;
  s->p_max_coarse_levels = 10; s->p_pre_sweep = 1; s->p_post_sweep = 3; s->p_smoother = UFVM_SMOOTHER_ILU;
  s->u_smoother = UFVM_SMOOTHER_ILU; s->u_n_iter = 10; s->quirks = UFVM_QUIRKS_REFERENCE; s->p_amg = 1;
  s->precision = UFVM_PREC_FP64; s->nu = 1.0; s->urf_u = 0.7; s->urf_p = 0.3; s->tol_u = 1e-6;
  s->tol_p = 1e-6; s->p_termination = 0.1; s->u_rrf = 0.1; s->false_dt = 1e9; s->p_coarse_weight = 1.0;
}

#define INT_FIELDS(X) X(n_correctors) X(fixed_element) X(p_cycle) X(p_max_cycles) X(p_max_coarse_levels) \
  X(p_pre_sweep) X(p_post_sweep) X(p_smoother) X(u_smoother) X(u_n_iter) X(quirks) X(p_amg) X(precision) \
  X(hierarchy_reuse) X(p_krylov) X(service_eager)
#define DBL_FIELDS(X) X(nu) X(urf_u) X(urf_p) X(tol_u) X(tol_p) X(p_termination) X(u_rrf) X(false_dt) \
  X(p_coarse_weight)

static void settings_of(const mxArray* a, ufvm_settings* s) {
  mxArray* f;
  default_settings(s);
  if (!a || mxIsEmpty(a)) return;
  if (!mxIsStruct(a)) mexErrMsgIdAndTxt("uFVM:invalid", "settings must be a struct");
#define GET_INT(name) if ((f = mxGetField(a, 0, #name)) != NULL) s->name = (int32_t)mxGetScalar(f);
#define GET_DBL(name) if ((f = mxGetField(a, 0, #name)) != NULL) s->name = mxGetScalar(f);
  INT_FIELDS(GET_INT)
  DBL_FIELDS(GET_DBL)
#undef GET_INT
#undef GET_DBL
}

static mxArray* settings_out(const ufvm_settings* s) {
#define NAME(name) #name,
  static const char* names[] = {INT_FIELDS(NAME) DBL_FIELDS(NAME)};
#undef NAME
  mxArray* o = mxCreateStructMatrix(1, 1, (int)(sizeof names / sizeof names[0]), names);
#define PUT_INT(name) mxSetField(o, 0, #name, mxCreateDoubleScalar((double)s->name));
#define PUT_DBL(name) mxSetField(o, 0, #name, mxCreateDoubleScalar(s->name));
  INT_FIELDS(PUT_INT)
  DBL_FIELDS(PUT_DBL)
#undef PUT_INT
#undef PUT_DBL
  return o;
}

/* polyMesh arrays: points (3 x np double), face_start, face_nodes, owner, neighbour (int32,
 * 0-based), patch_type, patch_start, patch_n (int32). */
static void mesh_of(const mxArray* prhs[], int k, ufvm_mesh_desc* m) {
  size_t n;
  m->points = in_double(prhs[k], "points", &n);
  m->n_points = (int32_t)(n / 3);
  m->face_start = in_int32(prhs[k + 1], "face_start", &n);
  m->n_faces = (int32_t)n - 1;
  m->face_nodes = in_int32(prhs[k + 2], "face_nodes", NULL);
  m->owner = in_int32(prhs[k + 3], "owner", NULL);
  m->neighbour = in_int32(prhs[k + 4], "neighbour", &n);
  m->n_interior = (int32_t)n;
  m->patch_type = in_int32(prhs[k + 5], "patch_type", &n);
  m->n_patches = (int32_t)n;
  m->patch_start = in_int32(prhs[k + 6], "patch_start", NULL);
  m->patch_n = in_int32(prhs[k + 7], "patch_n", NULL);
}

static mxArray* residuals_out(const double* res16) {
  mxArray* o = mxCreateDoubleMatrix(1, 16, mxREAL);
  memcpy(mxGetDoubles(o), res16, 16 * sizeof(double));
  return o;
}

static mxArray* field_out(ufvm_case* c, const char* name) {
  int64_t n = 0;
  mxArray* o;
  check(ufvm_get_field(c, name, NULL, 0, &n));
  o = mxCreateDoubleMatrix((mwSize)n, 1, mxREAL);
  check(ufvm_get_field(c, name, mxGetDoubles(o), n, &n));
  return o;
}

#ifdef UFVM_MEX_GPU
/* ---- stand-alone matrix functions on gpuArrays (cconn-ordered CSR, 0-based) ---- */
typedef struct {
  const mxGPUArray *rp, *col, *ac, *anb, *bc;
} GpuSystem;

static GpuSystem gpu_system(const mxArray* prhs[], int k, int with_bc) {
  GpuSystem s;
  s.rp = mxGPUCreateFromMxArray(prhs[k]);
  s.col = mxGPUCreateFromMxArray(prhs[k + 1]);
  s.ac = mxGPUCreateFromMxArray(prhs[k + 2]);
  s.anb = mxGPUCreateFromMxArray(prhs[k + 3]);
  s.bc = with_bc ? mxGPUCreateFromMxArray(prhs[k + 4]) : NULL;
  if (mxGPUGetClassID(s.rp) != mxINT32_CLASS || mxGPUGetClassID(s.col) != mxINT32_CLASS ||
      mxGPUGetClassID(s.ac) != mxDOUBLE_CLASS || mxGPUGetClassID(s.anb) != mxDOUBLE_CLASS)
    mexErrMsgIdAndTxt("uFVM:invalid", "rowptr/col must be int32 and ac/anb double gpuArrays");
  return s;
}

static void gpu_system_free(GpuSystem* s) {
  mxGPUDestroyGPUArray(s->rp); mxGPUDestroyGPUArray(s->col); mxGPUDestroyGPUArray(s->ac);
  mxGPUDestroyGPUArray(s->anb);
  if (s->bc) mxGPUDestroyGPUArray(s->bc);
}

#define RO(a) ((const void*)mxGPUGetDataReadOnly(a))
#endif

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  char cmd[48];
  (void)nlhs;
  if (nrhs < 1 || !mxIsChar(prhs[0])) mexErrMsgIdAndTxt("uFVM:invalid", "usage: ufvm_mex('<command>', ...)");
  mxGetString(prhs[0], cmd, sizeof cmd);
  if (!g_exit_registered) {
    mexAtExit(at_exit);
    g_exit_registered = 1;
  }

  if (!strcmp(cmd, "version")) {
    plhs[0] = mxCreateString(ufvm_version());
  } else if (!strcmp(cmd, "default_settings")) {
    ufvm_settings s;
    default_settings(&s);
    plhs[0] = settings_out(&s);

  /* ---- the case API (device-resident Domain state) ---- */
  } else if (!strcmp(cmd, "case_create")) {
    /* h = ufvm_mex('case_create', points, face_start, face_nodes, owner, neighbour, patch_type,
     *              patch_start, patch_n, settings, bc_type_u, bc_type_p, bc_val_u, bc_val_p,
     *              [U0, p0, mdot0])          -- cfdInitializeCase.m:14-83 */
    ufvm_mesh_desc m;
    ufvm_settings s;
    ufvm_case* c = NULL;
    need_args(nrhs, 14, cmd);
    mesh_of(prhs, 1, &m);
    settings_of(prhs[9], &s);
    check(ufvm_case_create(&m, &s, in_int32(prhs[10], "bc_type_u", NULL), in_int32(prhs[11], "bc_type_p", NULL),
                           in_double(prhs[12], "bc_val_u", NULL), in_double(prhs[13], "bc_val_p", NULL),
                           opt_double(nrhs, prhs, 14), opt_double(nrhs, prhs, 15), opt_double(nrhs, prhs, 16), &c));
    keep((void**)g_cases, c);
    plhs[0] = handle_out(c);
  } else if (!strcmp(cmd, "case_destroy")) {
    ufvm_case* c;
    need_args(nrhs, 2, cmd);
    c = case_of(prhs[1]);
    forget((void**)g_cases, c);
    check(ufvm_case_destroy(c));
  } else if (!strcmp(cmd, "case_sizes")) {
    int64_t sz[4];
    int i;
    need_args(nrhs, 2, cmd);
    check(ufvm_case_sizes(case_of(prhs[1]), sz));
    plhs[0] = mxCreateDoubleMatrix(1, 4, mxREAL);
    for (i = 0; i < 4; ++i) mxGetDoubles(plhs[0])[i] = (double)sz[i];
  } else if (!strcmp(cmd, "update_fields")) {            /* cfdUpdateFields */
    need_args(nrhs, 2, cmd);
    check(ufvm_update_fields(case_of(prhs[1])));
  } else if (!strcmp(cmd, "assemble_equation")) {        /* [rms, max] = cfdAssembleEquation(name, iComponent) */
    double rms = 0, mx = 0;
    need_args(nrhs, 4, cmd);
    check(ufvm_assemble_equation(case_of(prhs[1]), equation_of(prhs[2]), (int)mxGetScalar(prhs[3]) - 1, &rms, &mx));
    plhs[0] = mxCreateDoubleScalar(rms);
    plhs[1] = mxCreateDoubleScalar(mx);
  } else if (!strcmp(cmd, "solve_equation")) {           /* [r0, r1] = cfdSolveEquation(name) */
    double r0 = 0, r1 = 0;
    need_args(nrhs, 3, cmd);
    check(ufvm_solve_equation(case_of(prhs[1]), equation_of(prhs[2]), &r0, &r1));
    plhs[0] = mxCreateDoubleScalar(r0);
    plhs[1] = mxCreateDoubleScalar(r1);
  } else if (!strcmp(cmd, "correct_equation")) {         /* cfdCorrectEquation(name, iComponent) */
    need_args(nrhs, 4, cmd);
    check(ufvm_correct_equation(case_of(prhs[1]), equation_of(prhs[2]), (int)mxGetScalar(prhs[3]) - 1));
  } else if (!strcmp(cmd, "simple_iteration")) {         /* one pass of cfdRunCase.m:92-142 */
    double res[16];
    int conv = 0;
    need_args(nrhs, 2, cmd);
    check(ufvm_simple_iteration(case_of(prhs[1]), res, &conv));
    plhs[0] = residuals_out(res);
    plhs[1] = mxCreateLogicalScalar(conv != 0);
  } else if (!strcmp(cmd, "run_case")) {                 /* cfdRunCase */
    double res[16];
    int it = 0, code;
    need_args(nrhs, 3, cmd);
    code = ufvm_run_case(case_of(prhs[1]), (int)mxGetScalar(prhs[2]), &it, res);
    if (code != UFVM_OK && code != UFVM_E_NOT_CONVERGED) check(code);
    plhs[0] = mxCreateDoubleScalar((double)it);
    plhs[1] = residuals_out(res);
    plhs[2] = mxCreateLogicalScalar(code == UFVM_OK);
  } else if (!strcmp(cmd, "get_field")) {
    char name[32];
    need_args(nrhs, 3, cmd);
    mxGetString(prhs[2], name, sizeof name);
    plhs[0] = field_out(case_of(prhs[1]), name);
  } else if (!strcmp(cmd, "set_field")) {
    char name[32];
    size_t n;
    const double* v;
    need_args(nrhs, 4, cmd);
    mxGetString(prhs[2], name, sizeof name);
    v = in_double(prhs[3], "field values", &n);
    check(ufvm_set_field(case_of(prhs[1]), name, v, (int64_t)n));
  } else if (!strcmp(cmd, "get_geometry")) {
    char name[32];
    int64_t sz[4];
    size_t rows;
    need_args(nrhs, 3, cmd);
    mxGetString(prhs[2], name, sizeof name);
    check(ufvm_case_sizes(case_of(prhs[1]), sz));
    rows = (!strcmp(name, "volume") || !strcmp(name, "centroid_c")) ? (size_t)sz[0] : (size_t)sz[1];
    if (!strcmp(name, "Sf") || !strcmp(name, "centroid_f") || !strcmp(name, "CN") || !strcmp(name, "eCN") ||
        !strcmp(name, "T") || !strcmp(name, "centroid_c"))
      rows *= 3;
    plhs[0] = mxCreateDoubleMatrix((mwSize)rows, 1, mxREAL);
    check(ufvm_get_geometry(case_of(prhs[1]), name, mxGetDoubles(plhs[0]), (int64_t)rows));
  } else if (!strcmp(cmd, "get_levels")) {               /* iLevel = cfdAgglomerate(maxCoarseLevels) */
    int nl = 0, i;
    int64_t sizes[16];
    need_args(nrhs, 2, cmd);
    check(ufvm_get_levels(case_of(prhs[1]), &nl, sizes, 16));
    plhs[0] = mxCreateDoubleMatrix(1, (mwSize)nl, mxREAL);
    for (i = 0; i < nl; ++i) mxGetDoubles(plhs[0])[i] = (double)sizes[i];
  } else if (!strcmp(cmd, "get_level_array")) {          /* parents of cfdAgglomerateLevel.m (0-based) */
    char name[16];
    int64_t n = 0;
    int isint;
    need_args(nrhs, 4, cmd);
    mxGetString(prhs[3], name, sizeof name);
    isint = strcmp(name, "ac") && strcmp(name, "anb");
    check(ufvm_get_level_array(case_of(prhs[1]), (int)mxGetScalar(prhs[2]), name, NULL, 0, &n));
    plhs[0] = isint ? mxCreateNumericMatrix((mwSize)n, 1, mxINT32_CLASS, mxREAL)
                    : mxCreateDoubleMatrix((mwSize)n, 1, mxREAL);
    check(ufvm_get_level_array(case_of(prhs[1]), (int)mxGetScalar(prhs[2]), name,
                               isint ? (void*)mxGetInt32s(plhs[0]) : (void*)mxGetDoubles(plhs[0]), n, &n));

  /* ---- the batched service ---- */
  } else if (!strcmp(cmd, "service_create")) {
    ufvm_settings s;
    ufvm_service* v = NULL;
    need_args(nrhs, 3, cmd);
    settings_of(prhs[1], &s);
    check(ufvm_service_create(&s, (int64_t)mxGetScalar(prhs[2]), &v));
    keep((void**)g_services, v);
    plhs[0] = handle_out(v);
  } else if (!strcmp(cmd, "service_submit")) {
    /* ticket = ufvm_mex('service_submit', h, <8 polyMesh arrays>, nu, bc_type_u, bc_type_p,
     *                   bc_val_u, bc_val_p, max_iter) */
    ufvm_mesh_desc m;
    int64_t t = 0;
    need_args(nrhs, 16, cmd);
    mesh_of(prhs, 2, &m);
    check(ufvm_service_submit(service_of(prhs[1]), &m, mxGetScalar(prhs[10]), in_int32(prhs[11], "bc_type_u", NULL),
                              in_int32(prhs[12], "bc_type_p", NULL), in_double(prhs[13], "bc_val_u", NULL),
                              in_double(prhs[14], "bc_val_p", NULL), (int32_t)mxGetScalar(prhs[15]), &t));
    plhs[0] = mxCreateDoubleScalar((double)t);
  } else if (!strcmp(cmd, "service_step")) {
    int32_t nr = 0, nq = 0;
    int64_t nf = 0;
    need_args(nrhs, 2, cmd);
    check(ufvm_service_step(service_of(prhs[1]), &nr, &nq, &nf));
    plhs[0] = mxCreateDoubleScalar(nr);
    plhs[1] = mxCreateDoubleScalar(nq);
    plhs[2] = mxCreateDoubleScalar((double)nf);
  } else if (!strcmp(cmd, "service_poll")) {
    int64_t buf[1024], n = 0;
    int64_t i;
    need_args(nrhs, 2, cmd);
    check(ufvm_service_poll(service_of(prhs[1]), buf, 1024, &n));
    plhs[0] = mxCreateDoubleMatrix(1, (mwSize)n, mxREAL);
    for (i = 0; i < n; ++i) mxGetDoubles(plhs[0])[i] = (double)buf[i];
  } else if (!strcmp(cmd, "service_status")) {
    int32_t state = 0, status = 0, it = 0;
    double res[16], lat = 0, queue = 0;
    need_args(nrhs, 3, cmd);
    check(ufvm_service_status(service_of(prhs[1]), (int64_t)mxGetScalar(prhs[2]), &state, &status, &it, res, &lat,
                              &queue));
    plhs[0] = mxCreateDoubleScalar(state);
    plhs[1] = mxCreateDoubleScalar(status);
    plhs[2] = mxCreateDoubleScalar(it);
    plhs[3] = residuals_out(res);
    plhs[4] = mxCreateDoubleScalar(lat);
    plhs[5] = mxCreateDoubleScalar(queue);
  } else if (!strcmp(cmd, "service_get_field")) {
    char name[16];
    int64_t n = 0;
    ufvm_service* v;
    int64_t t;
    need_args(nrhs, 4, cmd);
    v = service_of(prhs[1]);
    t = (int64_t)mxGetScalar(prhs[2]);
    mxGetString(prhs[3], name, sizeof name);
    check(ufvm_service_get_field(v, t, name, NULL, 0, &n));
    plhs[0] = mxCreateDoubleMatrix((mwSize)n, 1, mxREAL);
    check(ufvm_service_get_field(v, t, name, mxGetDoubles(plhs[0]), n, &n));
  } else if (!strcmp(cmd, "service_release")) {
    need_args(nrhs, 3, cmd);
    check(ufvm_service_release(service_of(prhs[1]), (int64_t)mxGetScalar(prhs[2])));
  } else if (!strcmp(cmd, "service_admit")) {
    int32_t nr = 0;
    need_args(nrhs, 2, cmd);
    check(ufvm_service_admit(service_of(prhs[1]), &nr));
    plhs[0] = mxCreateDoubleScalar(nr);
  } else if (!strcmp(cmd, "service_set_memory_budget")) {
    need_args(nrhs, 3, cmd);
    check(ufvm_service_set_memory_budget(service_of(prhs[1]), (int64_t)mxGetScalar(prhs[2])));
  } else if (!strcmp(cmd, "service_set_admit_interval")) {
    need_args(nrhs, 3, cmd);
    check(ufvm_service_set_admit_interval(service_of(prhs[1]), (int32_t)mxGetScalar(prhs[2])));
  } else if (!strcmp(cmd, "service_set_schedule")) {
    need_args(nrhs, 4, cmd);
    check(ufvm_service_set_schedule(service_of(prhs[1]), (int32_t)mxGetScalar(prhs[2]), (int32_t)mxGetScalar(prhs[3])));
  } else if (!strcmp(cmd, "service_stats")) {
    need_args(nrhs, 2, cmd);
    plhs[0] = mxCreateDoubleMatrix(1, 34, mxREAL);
    check(ufvm_service_stats(service_of(prhs[1]), mxGetDoubles(plhs[0]), 34));
  } else if (!strcmp(cmd, "service_destroy")) {
    ufvm_service* v;
    need_args(nrhs, 2, cmd);
    v = service_of(prhs[1]);
    forget((void**)g_services, v);
    check(ufvm_service_destroy(v));

#ifdef UFVM_MEX_GPU
  /* ---- matrix functions on gpuArrays (rowptr, col int32 0-based; ac, anb, bc, dphi double) ---- */
  } else if (!strcmp(cmd, "compute_residuals_array")) {  /* r = cfdComputeResidualsArray(coeffs) */
    GpuSystem s;
    const mxGPUArray* x;
    mxGPUArray* r;
    int32_t n;
    need_args(nrhs, 7, cmd);
    mxInitGPU();
    s = gpu_system(prhs, 1, 1);
    x = mxGPUCreateFromMxArray(prhs[6]);
    n = (int32_t)mxGPUGetNumberOfElements(s.ac);
    r = mxGPUCreateGPUArray(1, (const mwSize[]){(mwSize)n}, mxDOUBLE_CLASS, mxREAL, MX_GPU_DO_NOT_INITIALIZE);
    check(ufvm_compute_residuals_array(n, RO(s.rp), RO(s.col), RO(s.ac), RO(s.anb), RO(s.bc), RO(x),
                                       mxGPUGetData(r), NULL));
    plhs[0] = mxGPUCreateMxArrayOnGPU(r);
    mxGPUDestroyGPUArray(r); mxGPUDestroyGPUArray(x); gpu_system_free(&s);
  } else if (!strcmp(cmd, "solve_sor") || !strcmp(cmd, "solve_sor_noalloc")) {  /* dphi = cfdSolveSOR(...) */
    GpuSystem s;
    mxGPUArray* x;
    int32_t n;
    need_args(nrhs, 7, cmd);
    mxInitGPU();
    s = gpu_system(prhs, 1, 1);
    x = mxGPUCopyFromMxArray(prhs[6]);
    n = (int32_t)mxGPUGetNumberOfElements(s.ac);
    check((!strcmp(cmd, "solve_sor") ? ufvm_solve_sor : ufvm_solve_sor_noalloc)(
        n, RO(s.rp), RO(s.col), RO(s.ac), RO(s.anb), RO(s.bc), mxGPUGetData(x), NULL));
    plhs[0] = mxGPUCreateMxArrayOnGPU(x);
    mxGPUDestroyGPUArray(x); gpu_system_free(&s);
  } else if (!strcmp(cmd, "factorize_ilu")) {            /* dc = cfdFactorizeILU(ac, anb, bc, cconn) */
    GpuSystem s;
    mxGPUArray* dc;
    int32_t n;
    need_args(nrhs, 6, cmd);
    mxInitGPU();
    s = gpu_system(prhs, 1, 0);
    n = (int32_t)mxGPUGetNumberOfElements(s.ac);
    dc = mxGPUCreateGPUArray(1, (const mwSize[]){(mwSize)n}, mxDOUBLE_CLASS, mxREAL, MX_GPU_DO_NOT_INITIALIZE);
    check(ufvm_factorize_ilu(n, RO(s.rp), RO(s.col), RO(s.ac), RO(s.anb), mxGPUGetData(dc),
                             (int32_t)mxGetScalar(prhs[5]), NULL));
    plhs[0] = mxGPUCreateMxArrayOnGPU(dc);
    mxGPUDestroyGPUArray(dc); gpu_system_free(&s);
  } else if (!strcmp(cmd, "solve_ilu")) {                /* dphi = cfdSolveILU(ac, anb, bc, dc, rc, cconn, dphi) */
    GpuSystem s;
    const mxGPUArray* dc;
    mxGPUArray* x;
    int32_t n;
    need_args(nrhs, 8, cmd);
    mxInitGPU();
    s = gpu_system(prhs, 1, 1);
    dc = mxGPUCreateFromMxArray(prhs[6]);
    x = mxGPUCopyFromMxArray(prhs[7]);
    n = (int32_t)mxGPUGetNumberOfElements(s.ac);
    check(ufvm_solve_ilu(n, RO(s.rp), RO(s.col), RO(s.ac), RO(s.anb), RO(s.bc), RO(dc), mxGPUGetData(x), NULL));
    plhs[0] = mxGPUCreateMxArrayOnGPU(x);
    mxGPUDestroyGPUArray(x); mxGPUDestroyGPUArray(dc); gpu_system_free(&s);
  } else if (!strcmp(cmd, "solve_algebraic_system")) {
    /* [dphi, r0, r1, iters] = cfdSolveAlgebraicSystem(level, smoother, nIter, rrf) on one matrix */
    GpuSystem s;
    mxGPUArray* x;
    int32_t n, iters = 0;
    double r0 = 0, r1 = 0;
    need_args(nrhs, 11, cmd);
    mxInitGPU();
    s = gpu_system(prhs, 1, 1);
    x = mxGPUCopyFromMxArray(prhs[6]);
    n = (int32_t)mxGPUGetNumberOfElements(s.ac);
    check(ufvm_solve_algebraic_system(n, RO(s.rp), RO(s.col), RO(s.ac), RO(s.anb), RO(s.bc), mxGPUGetData(x),
                                      (int32_t)mxGetScalar(prhs[7]), (int32_t)mxGetScalar(prhs[8]),
                                      mxGetScalar(prhs[9]), (int32_t)mxGetScalar(prhs[10]), &r0, &r1, &iters, NULL));
    plhs[0] = mxGPUCreateMxArrayOnGPU(x);
    plhs[1] = mxCreateDoubleScalar(r0);
    plhs[2] = mxCreateDoubleScalar(r1);
    plhs[3] = mxCreateDoubleScalar(iters);
    mxGPUDestroyGPUArray(x); gpu_system_free(&s);
  } else if (!strcmp(cmd, "agglomerate_level")) {
    /* [parents, c_rowptr, c_col, c_ac, c_anb] = one level of cfdAgglomerateLevel + assembleAgglomeratedLHS */
    GpuSystem s;
    mxGPUArray *par, *crp, *ccol, *cac, *canb;
    int32_t n, nnz, nc = 0, cnnz = 0;
    need_args(nrhs, 5, cmd);
    mxInitGPU();
    s = gpu_system(prhs, 1, 0);
    n = (int32_t)mxGPUGetNumberOfElements(s.ac);
    nnz = (int32_t)mxGPUGetNumberOfElements(s.anb);
    par = mxGPUCreateGPUArray(1, (const mwSize[]){(mwSize)n}, mxINT32_CLASS, mxREAL, MX_GPU_DO_NOT_INITIALIZE);
    crp = mxGPUCreateGPUArray(1, (const mwSize[]){(mwSize)n + 1}, mxINT32_CLASS, mxREAL, MX_GPU_DO_NOT_INITIALIZE);
    ccol = mxGPUCreateGPUArray(1, (const mwSize[]){(mwSize)(nnz > 0 ? nnz : 1)}, mxINT32_CLASS, mxREAL,
                               MX_GPU_DO_NOT_INITIALIZE);
    cac = mxGPUCreateGPUArray(1, (const mwSize[]){(mwSize)n}, mxDOUBLE_CLASS, mxREAL, MX_GPU_DO_NOT_INITIALIZE);
    canb = mxGPUCreateGPUArray(1, (const mwSize[]){(mwSize)(nnz > 0 ? nnz : 1)}, mxDOUBLE_CLASS, mxREAL,
                               MX_GPU_DO_NOT_INITIALIZE);
    check(ufvm_agglomerate_level(n, RO(s.rp), RO(s.col), RO(s.ac), RO(s.anb), mxGPUGetData(par), mxGPUGetData(crp),
                                 mxGPUGetData(ccol), mxGPUGetData(cac), mxGPUGetData(canb), &nc, &cnnz, NULL));
    plhs[0] = mxGPUCreateMxArrayOnGPU(par);
    plhs[1] = mxGPUCreateMxArrayOnGPU(crp);
    plhs[2] = mxGPUCreateMxArrayOnGPU(ccol);
    plhs[3] = mxGPUCreateMxArrayOnGPU(cac);
    plhs[4] = mxGPUCreateMxArrayOnGPU(canb);
    plhs[5] = mxCreateDoubleScalar(nc);
    plhs[6] = mxCreateDoubleScalar(cnnz);
    mxGPUDestroyGPUArray(par); mxGPUDestroyGPUArray(crp); mxGPUDestroyGPUArray(ccol);
    mxGPUDestroyGPUArray(cac); mxGPUDestroyGPUArray(canb); gpu_system_free(&s);
#endif
  } else {
    mexErrMsgIdAndTxt("uFVM:invalid", "ufvm_mex: unknown command '%s'", cmd);
  }
}
