"""CPU oracle for the RGF slice recursion -- TEST INFRASTRUCTURE ONLY.

This package is a plain numpy/scipy (complex128) restatement of the MATLAB
reference chiaweihsu/RGF:

    src/build_laplacian_1d.m   -> oracle.rgf_ref.build_laplacian_1d
    src/setup_channels.m       -> oracle.rgf_ref.setup_channels
    src/setup_channels_3D.m    -> oracle.rgf_ref.setup_channels_3D
    src/cal_smatrix_RGF.m      -> oracle.rgf_ref.cal_smatrix_RGF
    src/cal_smatrix_RGF_3D.m   -> oracle.rgf_ref.cal_smatrix_RGF_3D

Only the test-suite, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import it, and only as the checker or as the timed CPU
baseline.  The product (``rgf_b200``) never imports, links or calls anything
in here.

Parity status: MATLAB/Octave is not available on any machine this code runs
on, so parity against MATLAB's own double-precision output is *unpinned*.
The oracle is pinned instead by (1) analytic known answers (homogeneous slab:
r = 0, t = diag(exp(i kx (nx+1)))), (2) an independent dense block-tridiagonal
solve of the same discretised problem (``oracle.dense_fdfd``), and (3) the
reference's own invariants (unitarity, reciprocity under ind_prop_conj,
cross-branch consistency), see ``tests/test_oracle.py``.
"""
