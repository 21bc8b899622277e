function campoVett = BEMenerg_ppN_setup(pbParam, domainMesh, density, numPoints, xVal, tVal, methodInfo, PPn, PPw)
% Replacement body (reference: functions/BEMenerg_dirPP/BEMenerg_ppN_setup.m):
% u(x, t) = sum_n G_n gV_n - P_n u_n at every (point, time) with kernelG /
% kernelP's rules (methodInfo.numSubRegionPP x methodInfo.numNodiSingPP),
% contracted on the device (ebem_pp_dir).
deltaT = pbParam.Tfin / pbParam.nT;
gV = BEMenerg_dir_calcBoundDataNeumann(deltaT, pbParam, domainMesh);
u = ebem_mex('pp_dir', domainMesh.coordinates, domainMesh.triangles(:, 1:3), ebem_problem(pbParam), ...
             methodInfo.numSubRegionPP, methodInfo.numNodiSingPP, cell2mat(gV'), density, xVal, tVal);
campoVett = ebem_cells(u, size(xVal, 1), length(tVal));
filePath = strcat("./outputData/", pbParam.domainType, num2str(pbParam.lev), "_NEW_campoVett");
save(filePath, 'campoVett');
end
