function [initialResidual, finalResidual] = cfdSolveAlgebraicSystem(gridLevel, smootherType, numberOfIterations, rrf)
% CFDSOLVEALGEBRAICSYSTEM  Shadows fvm/solve/cfdSolveAlgebraicSystem.m:1 (the smoother loop with
% the reference's stopping rule) on the level's coefficients held as gpuArrays in
% Domain.coefficients{gridLevel}.gpu (rowptr, col: int32 0-based; ac, anb, bc, dphi: double).
global Domain
codes = struct('ILU', 0, 'SOR', 1, 'MCGS', 2);
g = Domain.coefficients{gridLevel}.gpu;
[g.dphi, initialResidual, finalResidual] = ufvm_mex('solve_algebraic_system', g.rowptr, g.col, g.ac, g.anb, ...
    g.bc, g.dphi, int32(codes.(smootherType)), int32(numberOfIterations), rrf, int32(Domain.gpu.settings.quirks));
Domain.coefficients{gridLevel}.gpu = g;
end
