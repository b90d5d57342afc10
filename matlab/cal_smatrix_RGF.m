function [smatrix, channels] = cal_smatrix_RGF(syst, out, in)
%CAL_SMATRIX_RGF  Scattering matrix of a 2D structure by the recursive
%Green's function method, computed on the GPU by librgf (via rgf_mex).
%
%   [smatrix, channels] = cal_smatrix_RGF(syst, out, in)
%
%   Same inputs, outputs and conventions as the reference function of the
%   same name: syst.epsilon ([ny, nx]), syst.epsilon_L, syst.epsilon_R,
%   syst.k0dx (may be complex), syst.yBC ('periodic', 'Dirichlet'/'PEC',
%   'Neumann'/'PMC', 'DirichletNeumann'/'PECPMC', 'NeumannDirichlet'/'PMCPEC'
%   or a real number k*a for Bloch periodic); out / in a cell array of
%   'left' / 'right' or a structure with fields ind_out_L, ind_out_R /
%   ind_in_L, ind_in_R (1-based channel indices).
if nargin < 3
    error('Not enough input arguments.');
end
rgf_check_syst(syst, out, in, 2);
[smatrix, channels] = rgf_mex('smatrix2d', syst, out, in);
channels.fun_phi = rgf_fun_phi(syst.yBC, size(syst.epsilon, 1));
end
