function residualsArray = cfdComputeResidualsArray(theCoefficients)
% CFDCOMPUTERESIDUALSARRAY  Shadows compute/cfdComputeResidualsArray.m:1 on gpuArrays:
% theCoefficients.gpu holds the cconn-ordered CSR (rowptr, col: int32 0-based; ac, anb, bc,
% dphi: double) that ufvm_coefficients_to_gpu builds once per mesh.
g = theCoefficients.gpu;
residualsArray = ufvm_mex('compute_residuals_array', g.rowptr, g.col, g.ac, g.anb, g.bc, g.dphi);
end
