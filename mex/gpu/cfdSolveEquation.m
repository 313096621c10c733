function [initialResidual, finalResidual] = cfdSolveEquation(theEquationName)
% CFDSOLVEEQUATION  Shadows fvm/solve/cfdSolveEquation.m:1: the equation's linear solver (the
% smoother loop for U, cfdApplyAMG for p) on the device-resident system.
[initialResidual, finalResidual] = ufvm_mex('solve_equation', ufvm_handle(), theEquationName);
end
