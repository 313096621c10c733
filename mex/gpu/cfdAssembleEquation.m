function [rmsResidual, maxResidual] = cfdAssembleEquation(theEquationName, iComponent)
% CFDASSEMBLEEQUATION  Shadows assemble/cfdAssembleEquation.m:1 (momentum component or the
% pressure-correction equation, assembled on the GPU into the device-resident coefficients).
if nargin < 2, iComponent = 1; end
[rmsResidual, maxResidual] = ufvm_mex('assemble_equation', ufvm_handle(), theEquationName, iComponent);
end
