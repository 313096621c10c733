// amg.cuh -- agglomeration AMG (cfdApplyAMG and friends).
#pragma once
#include "linsolve.cuh"

namespace ufvm {

struct AggScratch {
  DArr<double> maxAnb;
  DArr<signed char> strong;
  DArr<int> status, win, seedflag, newflag, seedRank, orphRank, res0, res1, cnt, estart, lists;
  DArr<unsigned long long> resv;
  void release();
};

int agglomerate_level(LinCtx& c, AggScratch& w, Level& F, Level& C, int* nCoarse);
int galerkin(LinCtx& c, Level& F, Level& C);
int galerkin32(LinCtx& c, Level& F, Level& C);
void free_level(Level& L, bool keep_matrix = false);

struct AmgSolver {
  LinCtx& ctx;
  AggScratch agg;
  int smoother = UFVM_SMOOTHER_SOR, quirks = UFVM_QUIRKS_REFERENCE, pre = 1, post = 3, max_cycles = 30;
  int max_coarse = 10, cycle_type = UFVM_CYCLE_V, cycles_used = 0;
  double rrf = 0.1;
  explicit AmgSolver(LinCtx& c) : ctx(c) {}
  int build(std::vector<Level>& lev, int max_coarse, int quirks, int* n_levels);
  int smooth(std::vector<Level>& lev, int l, int n_iter, double rrf);
  int restrict_(std::vector<Level>& lev, int l, int pre);
  int prolong_(std::vector<Level>& lev, int l, double rrf);
  int cycle(std::vector<Level>& lev, int L, double rrf, double* fin);
  int apply(std::vector<Level>& lev, bool rebuild, int* n_levels, double* r0, double* r1);
};

}  // namespace ufvm
