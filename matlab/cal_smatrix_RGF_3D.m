function [smatrix, channels] = cal_smatrix_RGF_3D(syst, out, in)
%CAL_SMATRIX_RGF_3D  Scattering matrix of a 3D structure by the recursive
%Green's function method, computed on the GPU by librgf (via rgf_mex).
%
%   [smatrix, channels] = cal_smatrix_RGF_3D(syst, out, in)
%
%   syst.epsilon is [nx, ny, nz]; syst.xyBC is 'periodic', 'Dirichlet'/'PEC'
%   or [kxa, kya] (Bloch); otherwise as cal_smatrix_RGF.
if nargin < 3
    error('Not enough input arguments.');
end
rgf_check_syst(syst, out, in, 3);
[smatrix, ch] = rgf_mex('smatrix3d', syst, out, in);
[nx, ny, ~] = size(syst.epsilon);
channels = rgf_channels_3d(ch, syst.xyBC, nx, ny);
end
