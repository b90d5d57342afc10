function channels = setup_channels_3D(nx, ny, BC, k0dx, epsilon_L, epsilon_R)
%SETUP_CHANNELS_3D  Transverse modes and longitudinal wave numbers of the
%two leads of a 3D structure, computed on the GPU by librgf.
if nargin < 5
    error('Not enough input arguments.');
end
if nargin < 6 || isempty(epsilon_R)
    ch = rgf_mex('channels3d', nx, ny, BC, k0dx, epsilon_L);
else
    ch = rgf_mex('channels3d', nx, ny, BC, k0dx, epsilon_L, epsilon_R);
end
channels = rgf_channels_3d(ch, BC, nx, ny);
if nargin < 6 || isempty(epsilon_R)
    channels.R = struct('N_prop', NaN);
end
end
