function q = ebem_problem(pbParam)
% The problem vector of every ebem_mex command: [rho mu lambda Tfin nT]
% (pbParam of readInputFile.m).
q = [pbParam.rho, pbParam.mu, pbParam.lambda, pbParam.Tfin, pbParam.nT];
end
