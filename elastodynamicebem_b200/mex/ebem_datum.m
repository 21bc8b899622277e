function datum = ebem_datum(pbParam)
% Boundary datum id of ebem_mex('rhs' / 'timemarch_*') for the cases of
% BEMenerg_core_calcNucleoTn.m: 'TEST' (the manufactured case, solution
% phi = (1,1,1)) is 8; the 'DIR' cases follow pbParam.domainType.
if pbParam.BOU == "TEST"
    datum = 8;
    return
end
switch pbParam.domainType
    case "sphereUniform",       datum = 2;
    case "screenUniform",       datum = 3;
    case "barH1",               datum = 4;
    case "barH3",               datum = 5;
    case "sphereWave",          datum = 6;
    case "elementoIndustriale", datum = 7;
    otherwise
        error("Problema non codificato")
end
end
