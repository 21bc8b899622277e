function campoVett = BEMenerg_postProcGPU_setupLayer(pbParam, domainMesh, density, xVal, tVal, methodInfo, PPn, PPw)
% Replacement body (reference: .../BEMenerg_postProcGPU/BEMenerg_postProcGPU_setupLayer.m):
% kernelLayer's numerical post-processing of all points at every time in one
% call (ebem_pp_gpu, variant EBEM_PP_LAYER = 1).
u = ebem_mex('pp_gpu', domainMesh.coordinates, domainMesh.triangles(:, 1:3), ebem_problem(pbParam), ...
             density, xVal, tVal, methodInfo.numSubRegionPP, methodInfo.numNodiSingPP, 1);
campoVett = ebem_cells(u, size(xVal, 1), length(tVal));
filePath = strcat("./outputData/", pbParam.domainType, num2str(pbParam.lev), "_GPU_campoVett");
save(filePath, 'campoVett');
end
