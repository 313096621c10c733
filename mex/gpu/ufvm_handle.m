function h = ufvm_handle()
% UFVM_HANDLE  The device-resident case behind the global Domain, created on first use.
% The case holds uFVM's Domain state for this path on the GPU (mesh geometry, fields, the
% coefficient matrices and the AMG hierarchy); Domain.gpu.handle refers to it.
% Domain.gpu.settings (fields of ufvm_settings, defaults from ufvm_mex('default_settings')) and
% Domain.gpu.bc (bc_type_u, bc_type_p: UFVM_BC_* per patch; bc_val_u: 3 x Fb; bc_val_p: 1 x Fb)
% are set by the case script before the first call, from the same system/ and 0/ entries the
% reference reads.
global Domain
if isfield(Domain, 'gpu') && isfield(Domain.gpu, 'handle') && ~isempty(Domain.gpu.handle)
    h = Domain.gpu.handle;
    return
end
m = ufvm_mesh_arrays(Domain.mesh);
bc = Domain.gpu.bc;
h = ufvm_mex('case_create', m.points, m.face_start, m.face_nodes, m.owner, m.neighbour, ...
             m.patch_type, m.patch_start, m.patch_n, Domain.gpu.settings, ...
             int32(bc.bc_type_u), int32(bc.bc_type_p), bc.bc_val_u, bc.bc_val_p);
Domain.gpu.handle = h;
end
