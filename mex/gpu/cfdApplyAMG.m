function [initRes, finalRes] = cfdApplyAMG(theEquation)
% CFDAPPLYAMG  Shadows solve/AMG/cfdApplyAMG.m:1 for the pressure-correction equation: the
% agglomeration and the V/W/F cycles run on the device-resident p system.
[initRes, finalRes] = ufvm_mex('solve_equation', ufvm_handle(), 'p');
end
