function cfdRunCase
% CFDRUNCASE  Shadows top/cfdRunCase.m for steady cases: the SIMPLE loop of cfdRunCase.m:92-142
% runs on the GPU until cfdCheckConvergence.m:3-20 passes or the iteration limit is reached.
global Domain
h = ufvm_handle();
maxIter = Domain.gpu.maxIterations;
[it, res, converged] = ufvm_mex('run_case', h, maxIter);
Domain.gpu.iterations = it;
Domain.gpu.lastResiduals = res;   % rms U1 U2 U3 p, max (4), solver initial (4), final (4)
if ~converged
    warning('uFVM:notConverged', 'not converged in %d iterations', it);
end
end
