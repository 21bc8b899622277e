function campoVett = BEMenerg_postProcGPU_setupSP(pbParam, domainMesh, density, numPoints, xVal, tVal, methodInfo, PPn, PPw)
% Replacement body (reference: .../BEMenerg_postProcGPU/BEMenerg_postProcGPU_setupSP.m):
% kernelSP's numerical post-processing for every (point, time) in one call
% (ebem_pp_gpu, variant EBEM_PP_POINT = 0, the reference's node stride kept).
u = ebem_mex('pp_gpu', domainMesh.coordinates, domainMesh.triangles(:, 1:3), ebem_problem(pbParam), ...
             density, xVal, tVal, methodInfo.numSubRegionPP, methodInfo.numNodiSingPP, 0);
campoVett = ebem_cells(u, size(xVal, 1), length(tVal));
filePath = strcat("./outputData/", pbParam.domainType, num2str(pbParam.lev), "_GPU_campoVett");
save(filePath, 'campoVett');
end
