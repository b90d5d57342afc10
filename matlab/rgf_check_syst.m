function rgf_check_syst(syst, out, in, dim)
%RGF_CHECK_SYST  Argument checks of cal_smatrix_RGF / cal_smatrix_RGF_3D,
%with the reference's error texts (cal_smatrix_RGF.m:78-91,
%cal_smatrix_RGF_3D.m:77-90), run before the MEX gateway is called.  The
%channel-index bounds (which need N_prop) and the warnings for ignored cell
%elements are raised by the gateway and the library with the same texts.
%
%   dim = 2 (syst.yBC, epsilon [ny, nx]) or 3 (syst.xyBC, epsilon [nx, ny, nz]).
if dim == 2
    bc = 'yBC';
else
    bc = 'xyBC';
end
if ~(isstruct(syst) && numel(syst) == 1); error('syst must be a structure'); end
names = {'epsilon', 'epsilon_L', 'epsilon_R', 'k0dx', bc};
for k = 1:numel(names)
    if ~isfield(syst, names{k}); error('syst.%s must be provided', names{k}); end
end
if dim == 2
    if ~(ismatrix(syst.epsilon) && isnumeric(syst.epsilon)); error('syst.epsilon must be a numeric matrix'); end
else
    if ~((ndims(syst.epsilon) == 3 || ndims(syst.epsilon) == 2) && isnumeric(syst.epsilon))
        error('syst.epsilon must be a 3D array');
    end
end
scalars = {'epsilon_L', 'epsilon_R', 'k0dx'};
for k = 1:numel(scalars)
    v = syst.(scalars{k});
    if ~(isscalar(v) && isnumeric(v)); error('syst.%s must be a numeric scalar', scalars{k}); end
end
if dim == 2
    % the reference accepts a character row here (cal_smatrix_RGF.m:89); a
    % real scalar k*a (Bloch periodic, as its help text and setup_channels.m
    % allow) is accepted as well
    yBC = syst.yBC;
    if ~(((ischar(yBC) || isstring(yBC)) && isrow(yBC)) || (isnumeric(yBC) && isscalar(yBC)))
        error('syst.yBC must be ''periodic'' or ''Dirichlet''');
    end
    if size(syst.epsilon, 1) == 0; error('need at least one site along the transverse (y) direction'); end
else
    if size(syst.epsilon, 1) * size(syst.epsilon, 2) == 0
        error('need at least one site along the transverse directions (x,y)');
    end
end
if ~(isstruct(in) || iscell(in)); error('input argument ''in'' must be a structure or a cell array'); end
if ~(isstruct(out) || iscell(out)); error('input argument ''out'' must be a structure or a cell array'); end
end
