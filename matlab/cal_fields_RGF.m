function [smatrix, psi] = cal_fields_RGF(syst, out, in)
%CAL_FIELDS_RGF  Scattering matrix of a 2D structure and the fields inside
%it (librgf, via rgf_mex; the reference computes S only).
%
%   [smatrix, psi] = cal_fields_RGF(syst, out, in)
%
%   Inputs as cal_smatrix_RGF.  psi is [ny, nx, n_in]: psi(:, n, b) is the
%   response at slice n to input channel b (the columns of smatrix), i.e.
%   G(n, s) * B(:, b) with G the Green's function of the whole structure and
%   B the channel's source profile on its lead's surface.
if nargin < 3
    error('Not enough input arguments.');
end
rgf_check_syst(syst, out, in, 2);
[smatrix, psi] = rgf_mex('fields2d', syst, out, in);
end
