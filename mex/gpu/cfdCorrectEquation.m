function cfdCorrectEquation(theEquationName, iComponent)
% CFDCORRECTEQUATION  Shadows solve/correct/cfdCorrectEquation.m:1 (U component update, or the
% PP / velocity / pressure / mass-flux corrections for p).
if nargin < 2, iComponent = 1; end
ufvm_mex('correct_equation', ufvm_handle(), theEquationName, iComponent);
end
