function campoVett = ebem_cells(u, xSize, tSize)
% 3 x npts x ntimes displacement of ebem_mex -> the reference's campoVett,
% an xSize x tSize cell array of 3 x 1 vectors.
campoVett = reshape(num2cell(reshape(u, 3, []), 1), [xSize, tSize]);
end
