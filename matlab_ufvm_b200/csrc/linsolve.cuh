// linsolve.cuh -- matrix-level operations on cconn-ordered CSR levels.
#pragma once
#include "case.cuh"

namespace ufvm {

int scan_exclusive(LinCtx& c, const int* in, int* out, int n, int* total_host);
int residual(LinCtx& c, const Level& L, const double* x, double* r);
int sum_abs_residual(LinCtx& c, const Level& L, const double* x, double* out_host);
int build_schedule(LinCtx& c, Level& L);
int build_tpos(LinCtx& c, Level& L);
int build_coloring(LinCtx& c, Level& L);
int check_barrier(LinCtx& c);                        // error if a grid-barrier sweep timed out
int gs_sweep(LinCtx& c, Level& L);                   // natural-order symmetric GS (level scheduled)
int mcgs_prepare(LinCtx& c, Level& L);               // colour-major copy of the matrix and rhs
int mcgs_sweep(LinCtx& c, Level& L);                 // multicolour symmetric GS (after mcgs_prepare)
int ilu_factor(LinCtx& c, Level& L, int quirks);     // dc = DILU diagonal inverse
int ilu_sweep(LinCtx& c, Level& L);                  // one cfdSolveILU application
int solve_algebraic_system(LinCtx& c, Level& L, int smoother, int n_iter, double rrf, int quirks,
                           double* r0, double* r1, int* iters);
int restrict_residual(LinCtx& c, Level& F, Level& C);  // C.bc[P] = sum over F's children of P of r_F
int prolong(LinCtx& c, Level& F, const Level& C);      // F.dphi += C.dphi[parents]

}  // namespace ufvm
