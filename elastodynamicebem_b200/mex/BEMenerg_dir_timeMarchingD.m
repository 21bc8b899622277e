function density = BEMenerg_dir_timeMarchingD(pbParam, domainMesh, methodInfo, GHn, GHw, GHCn, GHCw, DIAGn, DIAGw)
% Replacement body (reference: functions/BEMenerg_dir/BEMenerg_dir_timeMarchingD.m):
% V_l, K_l, the right-hand side of BEMenerg_core_calcTnBlock, the beta_K
% convolution and the LU marching of V_0 in libebem.  The Dirichlet datum is
% the reference's own BEMenerg_dir_calcBoundDataDirichlet.
deltaT = pbParam.Tfin / pbParam.nT;
gK = BEMenerg_dir_calcBoundDataDirichlet(deltaT, pbParam, domainMesh);
P = domainMesh.coordinates;
T = domainMesh.triangles(:, 1:3);
q = ebem_problem(pbParam);
rhs = ebem_mex('rhs', P, T, q, methodInfo.numNodiExt, ebem_datum(pbParam));
rules = [methodInfo.numNodiExt, methodInfo.numSubRegion, methodInfo.numNodiSing, methodInfo.numNodiDiag];
density = ebem_mex('march_dd', P, T, q, rules, rhs, cell2mat(gK'));
outPath = strcat("./outputData/", pbParam.domainType, num2str(pbParam.lev), "_NEW_", ...
    num2str(methodInfo.numNodiExt), "_", num2str(methodInfo.numSubRegion), "_", num2str(methodInfo.numNodiSing), "_", ...
    num2str(methodInfo.numNodiDiag));
save(strcat(outPath, "_density"), 'density');
end
