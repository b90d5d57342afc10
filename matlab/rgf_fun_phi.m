function f = rgf_fun_phi(BC, ny)
%RGF_FUN_PHI  Transverse mode profiles phi(y; ky) of a 2D lead as a function
%handle of a row of ky*dx values (ny rows, one column per ky), for the
%boundary condition BC.
m = (1:ny).';
if isnumeric(BC)
    f = @(k) exp(1i * m * k(:).') / sqrt(ny);
    return
end
switch lower(BC)
    case 'periodic'
        f = @(k) exp(1i * m * k(:).') / sqrt(ny);
    case {'dirichlet', 'pec'}
        f = @(k) sin(m * k(:).') * sqrt(2 / (ny + 1));
    case {'neumann', 'pmc'}
        f = @(k) (cos((m - 0.5) * k(:).') - (k(:).' == 0) * (1 - sqrt(1 / 2))) * sqrt(2 / ny);
    case {'dirichletneumann', 'pecpmc'}
        f = @(k) sin(m * k(:).') * sqrt(2 / (ny + 0.5));
    case {'neumanndirichlet', 'pmcpec'}
        f = @(k) cos((m - 0.5) * k(:).') * sqrt(2 / (ny + 0.5));
    otherwise
        error('BC = %s is not an eligible option', BC);
end
end
