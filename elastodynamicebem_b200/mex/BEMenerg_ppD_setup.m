function campoVett = BEMenerg_ppD_setup(pbParam, domainMesh, density, numPoints, xVal, tVal, methodInfo, PPn, PPw)
% Replacement body (reference: functions/BEMenerg_dirPP/BEMenerg_ppD_setup.m):
% u(x, t) = sum_n G_n phi_n - P_n gK_n (ebem_pp_dir with a = density, b = gK).
deltaT = pbParam.Tfin / pbParam.nT;
gK = BEMenerg_dir_calcBoundDataDirichlet(deltaT, pbParam, domainMesh);
u = ebem_mex('pp_dir', domainMesh.coordinates, domainMesh.triangles(:, 1:3), ebem_problem(pbParam), ...
             methodInfo.numSubRegionPP, methodInfo.numNodiSingPP, density, cell2mat(gK'), xVal, tVal);
campoVett = ebem_cells(u, size(xVal, 1), length(tVal));
filePath = strcat("./outputData/", pbParam.domainType, num2str(pbParam.lev), "_NEW_campoVett");
save(filePath, 'campoVett');
end
