function density = BEMenerg_coreGPU_timeMarching(pbParam, domainMesh, methodInfo, GHn, GHw, GHCn, GHCw)
% Replacement body (reference: .../BEMenerg_coreGPU/BEMenerg_coreGPU_timeMarching.m):
% numerical-inner blocks off the diagonal (kernelGHC's method), semi-analytic
% diagonal, right-hand side and LU marching in libebem.  The reference's
% reset(gpuDevice) at entry and exit (:7,170) is gone: the library keeps its
% workspace pool and solver handles between calls, and a reset would leave
% them dangling (call ebem_mex('release', device - 1) before any reset).
density = ebem_mex('timemarch_ghc', domainMesh.coordinates, domainMesh.triangles(:, 1:3), ...
                   ebem_problem(pbParam), methodInfo.numNodiExt, methodInfo.numSubRegion, ...
                   methodInfo.numNodiSing, ebem_datum(pbParam));
outPath = strcat("./outputData/", pbParam.domainType, num2str(pbParam.lev), "_GPU_", ...
    num2str(methodInfo.numNodiExt), "_", num2str(methodInfo.numSubRegion), "_", num2str(methodInfo.numNodiSing));
save(strcat(outPath, "_density"), 'density');
end
