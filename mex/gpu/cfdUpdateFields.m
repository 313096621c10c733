function cfdUpdateFields
% CFDUPDATEFIELDS  Shadows update/cfdUpdateFields.m:2 (boundary values, gradients, scales).
ufvm_mex('update_fields', ufvm_handle());
end
