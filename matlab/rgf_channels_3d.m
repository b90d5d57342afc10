function channels = rgf_channels_3d(ch, BC, nx, ny)
%RGF_CHANNELS_3D  Arranges the channel data returned by rgf_mex for a 3D
%lead as the reference's setup_channels_3D does: nx-by-ny kxdx / kydx /
%kzdx, and the separable profile handle fun_phi(kx, ky).
channels.kxdx = reshape(ch.kxdx, nx, ny);
channels.kydx = reshape(ch.kydx, nx, ny);
mx = (1:nx).';
my = (1:ny);
if isnumeric(BC) || strcmpi(BC, 'periodic')
    channels.fun_phi = @(kx, ky) exp(1i * mx * kx) * exp(1i * my * ky) / sqrt(nx * ny);
else
    channels.fun_phi = @(kx, ky) sin(mx * kx) * sin(my * ky) * sqrt(4 / ((nx + 1) * (ny + 1)));
end
for side = {'L', 'R'}
    s = ch.(side{1});
    t.N_prop = s.N_prop;
    t.kzdx = reshape(s.kxdx, nx, ny);
    t.ind_prop = s.ind_prop;
    t.sqrt_mu = s.sqrt_mu;
    channels.(side{1}) = t;
end
end
