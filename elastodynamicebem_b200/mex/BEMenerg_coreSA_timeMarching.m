function density = BEMenerg_coreSA_timeMarching(pbParam, domainMesh, methodInfo, GHn, GHw)
% Replacement body (same signature as the reference's, functions/
% BEMenerg_indir/BEMenerg_core/BEMenerg_coreSA/BEMenerg_coreSA_timeMarching.m):
% assembly of E_0..E_{L-1}, right-hand side and LU marching in libebem
% (ebem_timemarch_sa).  GHn/GHw are the rule of methodInfo.numNodiExt, which
% the library builds itself.  The blocks are not written to ./tempData: they
% stay on the device.
density = ebem_mex('timemarch_sa', domainMesh.coordinates, domainMesh.triangles(:, 1:3), ...
                   ebem_problem(pbParam), methodInfo.numNodiExt, ebem_datum(pbParam));
outPath = strcat("./outputData/", pbParam.domainType, num2str(pbParam.lev), "_SA_", num2str(methodInfo.numNodiExt));
save(strcat(outPath, "_density"), 'density');
end
