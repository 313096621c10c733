function [rowptr, col, anbv] = ufvm_cconn_to_csr(cconn, anb)
% UFVM_CCONN_TO_CSR  uFVM's cell arrays cconn{i} (1-based neighbour lists) and anb{i} as the
% cconn-ordered CSR the library takes: rowptr and col int32 0-based, anb values in cconn order,
% on the GPU. The index arrays are cached per mesh (they do not change between calls).
persistent key cached_rowptr cached_col
n = numel(cconn);
counts = cellfun(@numel, cconn);
k = [n, sum(counts)];
if isempty(key) || ~isequal(key, k)
    cached_rowptr = gpuArray(int32([0; cumsum(counts(:))]));
    cached_col = gpuArray(int32(vertcat(cconn{:}) - 1));
    key = k;
end
rowptr = cached_rowptr;
col = cached_col;
anbv = gpuArray(vertcat(anb{:}));
end
