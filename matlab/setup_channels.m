function channels = setup_channels(ny, BC, k0dx, epsilon_L, epsilon_R)
%SETUP_CHANNELS  Transverse modes and longitudinal wave numbers of the two
%leads of a 2D structure, computed on the GPU by librgf.  Same signature and
%output as the reference function; with epsilon_R omitted only the left
%side is set up (channels.R.N_prop = NaN).
if nargin < 4
    error('Not enough input arguments.');
end
if nargin < 5 || isempty(epsilon_R)
    channels = rgf_mex('channels2d', ny, BC, k0dx, epsilon_L);
    channels.R = struct('N_prop', NaN);
else
    channels = rgf_mex('channels2d', ny, BC, k0dx, epsilon_L, epsilon_R);
end
channels.fun_phi = rgf_fun_phi(BC, ny);
end
