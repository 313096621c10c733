function [dc, rc] = cfdFactorizeILU(ac, anb, bc, cconn)
% CFDFACTORIZEILU  Shadows solve/cfdFactorizeILU.m (the DILU diagonal, level scheduled).
global Domain
[rowptr, col, anbv] = ufvm_cconn_to_csr(cconn, anb);
quirks = Domain.gpu.settings.quirks;
dc = ufvm_mex('factorize_ilu', rowptr, col, gpuArray(ac), anbv, int32(quirks));
rc = zeros(size(ac));
end
