function iLevel = cfdAgglomerate(maxCoarseLevels)
% CFDAGGLOMERATE  Shadows solve/AMG/cfdAgglomerate.m:1: the levels of the hierarchy the last p
% solve built on the device (their sizes are in Domain.gpu.levelSizes, the cell-to-coarse maps
% via ufvm_mex('get_level_array', h, level, 'parents'), 0-based).
global Domain
sizes = ufvm_mex('get_levels', ufvm_handle());
Domain.gpu.levelSizes = sizes;
iLevel = min(numel(sizes), maxCoarseLevels + 1);
end
