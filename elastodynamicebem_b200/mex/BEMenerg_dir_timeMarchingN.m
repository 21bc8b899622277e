function density = BEMenerg_dir_timeMarchingN(pbParam, domainMesh, methodInfo, GHn, GHw, GHCn, GHCw, DIAGn, DIAGw)
% Replacement body (reference: functions/BEMenerg_dir/BEMenerg_dir_timeMarchingN.m):
% V_l (kernelV + DIAG-rule diagonal), K_l (kernelK + singular parts), the
% beta_V convolution and the least-squares marching of (K_0 + I_Gamma) in
% libebem.  The Neumann datum is the reference's own
% BEMenerg_dir_calcBoundDataNeumann.  No reset(gpuDevice) (see ebem_mex('release')).
deltaT = pbParam.Tfin / pbParam.nT;
gV = BEMenerg_dir_calcBoundDataNeumann(deltaT, pbParam, domainMesh);
rules = [methodInfo.numNodiExt, methodInfo.numSubRegion, methodInfo.numNodiSing, methodInfo.numNodiDiag];
density = ebem_mex('march_dn', domainMesh.coordinates, domainMesh.triangles(:, 1:3), ...
                   ebem_problem(pbParam), rules, cell2mat(gV'));
outPath = strcat("./outputData/", pbParam.domainType, num2str(pbParam.lev), "_NEW_", ...
    num2str(methodInfo.numNodiExt), "_", num2str(methodInfo.numSubRegion), "_", num2str(methodInfo.numNodiSing), "_", ...
    num2str(methodInfo.numNodiDiag));
save(strcat(outPath, "_density"), 'density');
end
