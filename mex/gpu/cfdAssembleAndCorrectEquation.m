function [rmsResidual, maxResidual, initRes, finalRes] = cfdAssembleAndCorrectEquation(theEquationName)
% CFDASSEMBLEANDCORRECTEQUATION  Shadows assemble/cfdAssembleAndCorrectEquation.m:35-49: for U
% the three components are assembled, solved and corrected in turn; for p the nCorrectors
% assemble/solve/correct passes run. Residuals as the reference returns them.
h = ufvm_handle();
if strcmp(theEquationName, 'U')
    comps = 1:3;
else
    comps = 1;
end
rmsResidual = zeros(1, numel(comps)); maxResidual = rmsResidual; initRes = rmsResidual; finalRes = rmsResidual;
for k = comps
    [rmsResidual(k), maxResidual(k)] = ufvm_mex('assemble_equation', h, theEquationName, k);
    [initRes(k), finalRes(k)] = ufvm_mex('solve_equation', h, theEquationName);
    ufvm_mex('correct_equation', h, theEquationName, k);
end
end
