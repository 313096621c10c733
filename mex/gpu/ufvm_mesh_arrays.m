function m = ufvm_mesh_arrays(theMesh)
% UFVM_MESH_ARRAYS  The raw polyMesh arrays ufvm_mex takes, from uFVM's mesh struct
% (utilities/IO/cfdReadPolyMesh.m: nodes(n).centroid, faces(n).iNodes / iOwner / iNeighbour,
% numberOfInteriorFaces, boundaries(n).type / startFace / numberOfBFaces), 0-based int32.
nF = numel(theMesh.faces);
m.points = reshape([theMesh.nodes.centroid], 3, []);
counts = arrayfun(@(f) numel(f.iNodes), theMesh.faces);
m.face_start = int32([0, cumsum(counts)]);
m.face_nodes = int32([theMesh.faces.iNodes] - 1);
m.owner = int32([theMesh.faces.iOwner] - 1);
m.neighbour = int32([theMesh.faces(1:theMesh.numberOfInteriorFaces).iNeighbour] - 1);
types = {'wall', 'inlet', 'outlet', 'symmetry', 'empty'};
nP = numel(theMesh.boundaries);
m.patch_type = zeros(1, nP, 'int32');
m.patch_start = zeros(1, nP, 'int32');
m.patch_n = zeros(1, nP, 'int32');
for k = 1:nP
    b = theMesh.boundaries(k);
    t = find(strcmp(types, b.type), 1);
    if isempty(t)
        error('uFVM:boundaryCondition', 'patch type %s is not on this path', b.type);
    end
    m.patch_type(k) = int32(t - 1);
    m.patch_start(k) = int32(b.startFace - 1);
    m.patch_n(k) = int32(b.numberOfBFaces);
end
assert(double(m.face_start(end)) == numel(m.face_nodes) && numel(m.owner) == nF);
end
