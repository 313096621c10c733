function dphi = cfdSolveILU(ac, anb, bc, dc, rc, cconn, dphi)
% CFDSOLVEILU  Shadows solve/cfdSolveILU.m:18-93 (DILU forward and backward substitution,
% level scheduled on the GPU).
[rowptr, col, anbv] = ufvm_cconn_to_csr(cconn, anb);
dphi = ufvm_mex('solve_ilu', rowptr, col, gpuArray(ac), anbv, gpuArray(bc), gpuArray(dc), gpuArray(dphi));
end
