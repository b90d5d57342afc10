function A = build_laplacian_1d(n, BC)
%BUILD_LAPLACIAN_1D  1D finite-difference Laplacian with boundary condition
%BC, built on the GPU by librgf and returned as a sparse matrix (real
%unless a Bloch phase makes it complex).
A = sparse(rgf_mex('laplacian', n, BC));
if all(imag(nonzeros(A)) == 0)
    A = real(A);
end
end
