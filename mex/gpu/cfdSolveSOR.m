function dphi = cfdSolveSOR(ac, anb, bc, cconn, dphi)
% CFDSOLVESOR  Shadows solve/cfdSolveSOR.m (one symmetric Gauss-Seidel sweep in natural order,
% level scheduled on the GPU, bit-identical to the sequential sweep).
[rowptr, col, anbv] = ufvm_cconn_to_csr(cconn, anb);
dphi = ufvm_mex('solve_sor', rowptr, col, gpuArray(ac), anbv, gpuArray(bc), gpuArray(dphi));
end
