function campoVett = BEMenerg_postProcA_setup(pbParam, domainMesh, density, numPoints, xVal, tVal)
% Replacement body (reference: .../BEMenerg_postProcA/BEMenerg_postProcA_setup.m):
% the closed-form post-processing at every (point, time) (ebem_pp_sa).
u = ebem_mex('pp_sa', domainMesh.coordinates, domainMesh.triangles(:, 1:3), ebem_problem(pbParam), ...
             density, xVal, tVal);
campoVett = ebem_cells(u, size(xVal, 1), length(tVal));
filePath = strcat("./outputData/", pbParam.domainType, num2str(pbParam.lev), "_A_campoVett");
save(filePath, 'campoVett');
end
