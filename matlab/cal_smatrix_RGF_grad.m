function [smatrix, dF_deps] = cal_smatrix_RGF_grad(syst, out, in, D)
%CAL_SMATRIX_RGF_GRAD  S-matrix of a 2D structure and the derivative of a
%real objective with respect to every permittivity pixel (librgf's adjoint
%sweep; the reference has no gradient).
%
%   [smatrix, dF_deps] = cal_smatrix_RGF_grad(syst, out, in, D)
%
%   D is the matrix of weights dF/dS (the size of smatrix), such that
%   dF = 2*real(sum(D(:) .* dS(:))); for F = sum(abs(S(:)).^2) use
%   D = conj(S) (e.g. from a first call of cal_smatrix_RGF).  dF_deps has the
%   size of syst.epsilon and is the derivative with respect to the real part
%   of epsilon.
if nargin < 4
    error('Not enough input arguments.');
end
rgf_check_syst(syst, out, in, 2);
[smatrix, g] = rgf_mex('grad2d', syst, out, in, D);
dF_deps = 2 * real(g);
end
