"""numpy/scipy FP64 restatement of chiaweihsu/RGF (the oracle).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()``
and the CPU-baseline leg of ``bench.py``; never by the product.

Every function follows the MATLAB source line by line; the docstrings cite the
file:line ranges (paths are relative to the reference project root).  MATLAB
conventions that matter for the numbers are reproduced explicitly:

* channel indices in ``in``/``out`` and in ``channels[...]['ind_prop']`` are
  1-based, as in MATLAB;
* MATLAB's ``asin`` returns ``pi/2 - 1i*acosh(x)`` for a real argument
  ``x > 1`` (C99/numpy return ``+1i*acosh(x)``); :func:`_asin_sqrt_matlab`
  restates MATLAB's value because the branch flip of
  ``setup_channels.m:211-215`` is written against it;
* ``inv`` is LAPACK getrf+getri (``scipy.linalg.inv``) and ``\\`` is
  getrf+getrs (``numpy.linalg.solve``).

Deliberate divergences from the MATLAB text (documented quirks):

* Q1: ``cal_smatrix_RGF.m:89`` rejects a numeric (Bloch) ``yBC`` although the
  help text (``:32-34``) and ``setup_channels.m:105-111`` support it; the
  oracle accepts it.
* Q9: for a periodic/Bloch Laplacian with ``n == 1`` MATLAB's ``spdiags``
  receives coincident diagonals (``build_laplacian_1d.m:51``).  The oracle
  builds the physical hopping sum instead (``Lap = 2cos(ka) - 2``).
"""
from __future__ import annotations

import warnings
from typing import Any, Callable, Dict

import numpy as np
import scipy.linalg as sla

__all__ = [
    "build_laplacian_1d",
    "setup_channels",
    "setup_channels_3D",
    "cal_smatrix_RGF",
    "cal_smatrix_RGF_3D",
    "parse_channel_request",
]


# --------------------------------------------------------------------------
# helpers
# --------------------------------------------------------------------------
def _field(s: Any, name: str):
    if isinstance(s, dict):
        return s[name]
    return getattr(s, name)


def _has(s: Any, name: str) -> bool:
    if isinstance(s, dict):
        return name in s
    return hasattr(s, name)


def _is_numeric_scalar(x) -> bool:
    return np.isscalar(x) and isinstance(x, (int, float, complex, np.number)) and not isinstance(x, bool)


def _bc_to_kind(BC, allow_vector: bool = False):
    """Normalise a BC argument: returns (kind, ka).

    kind is one of 'Bloch', 'Dirichlet', 'Neumann', 'DirichletNeumann',
    'NeumannDirichlet'; ka is the Bloch phase (0 for 'periodic') or None.
    Follows setup_channels.m:98-115 and build_laplacian_1d.m:42-53.
    """
    if isinstance(BC, str):
        b = BC.lower()
        if b == "bloch":
            raise ValueError(
                "To use Bloch periodic boundary condition, set BC to k*a where k is "
                "the Bloch wave number and a is the periodicity")
        if b == "periodic":
            return "Bloch", 0.0
        if b in ("dirichlet", "pec"):
            return "Dirichlet", None
        if b in ("neumann", "pmc"):
            return "Neumann", None
        if b in ("dirichletneumann", "pecpmc"):
            return "DirichletNeumann", None
        if b in ("neumanndirichlet", "pmcpec"):
            return "NeumannDirichlet", None
        raise ValueError(f"Boundary condition BC = {BC} is not an eligible option")
    if _is_numeric_scalar(BC):
        return "Bloch", BC
    raise ValueError("Boundary condition BC has to be a character vector or string, "
                     "or numeric scalar (for Bloch periodic BC)")


# --------------------------------------------------------------------------
# build_laplacian_1d.m
# --------------------------------------------------------------------------
def build_laplacian_1d(n: int, BC) -> np.ndarray:
    """Dense restatement of build_laplacian_1d.m:1-75.

    Returns the n-by-n matrix ``-grad_1^H grad_1`` (``:71-75``) where grad_1
    is the forward difference with the boundary rule of ``:48-69``:

    * Bloch (``:51``): rows [f(1)-e^{-ika}f(n), f(2)-f(1), ..., f(n)-f(n-1)]
    * Dirichlet (``:55``): (n+1)-by-n, f(0)=f(n+1)=0
    * Neumann (``:59``): (n-1)-by-n, df(1/2)=df(n+1/2)=0
    * DirichletNeumann (``:63``), NeumannDirichlet (``:67``): n-by-n.

    Entries are accumulated, so n == 1 Bloch gives the physical
    ``2*cos(ka) - 2`` (quirk Q9; MATLAB's spdiags sees coincident diagonals).
    """
    if not (isinstance(n, (int, np.integer)) and n >= 0):
        raise ValueError("The number of sites n must be a non-negative integer scalar")
    kind, ka = _bc_to_kind(BC)
    if kind == "Bloch" and np.iscomplexobj(ka) and np.imag(ka) != 0:
        warnings.warn(f"k*a = {np.real(ka):g} + 1i*{np.imag(ka):g} is a complex number.")
    if kind == "Bloch":
        g = np.zeros((n, n), dtype=complex)
        for j in range(n):
            g[j, j] += 1.0
            if j >= 1:
                g[j, j - 1] += -1.0
        if n >= 1:
            g[0, n - 1] += -np.exp(-1j * ka)
    elif kind == "Dirichlet":
        g = np.zeros((n + 1, n))
        for j in range(n):
            g[j, j] += 1.0
            g[j + 1, j] += -1.0
    elif kind == "Neumann":
        g = np.zeros((max(n - 1, 0), n))
        for i in range(n - 1):
            g[i, i + 1] += 1.0
            g[i, i] += -1.0
    elif kind == "DirichletNeumann":
        g = np.zeros((n, n))
        for j in range(n):
            g[j, j] += 1.0
            if j + 1 < n:
                g[j + 1, j] += -1.0
    else:  # NeumannDirichlet
        g = np.zeros((n, n))
        for j in range(n):
            g[j, j] += -1.0
            if j >= 1:
                g[j - 1, j] += 1.0
    return -(g.conj().T @ g)


# --------------------------------------------------------------------------
# setup_channels.m
# --------------------------------------------------------------------------
def _asin_sqrt_matlab(z: np.ndarray, z_is_real: bool) -> np.ndarray:
    """MATLAB's ``asin(sqrt(z))`` (setup_channels.m:190).

    For a real-typed z MATLAB's sqrt gives sqrt(z) for z >= 0 and
    1i*sqrt(-z) for z < 0; MATLAB's asin gives pi/2 - 1i*acosh(w) for a real
    w > 1 and 1i*asinh(y) for w = 1i*y.  For a complex-typed z (nonzero
    imaginary part everywhere, since Im z = Im(k0dx^2 eps)/4) both functions
    are the principal branches, which numpy implements.
    """
    if not z_is_real:
        return np.arcsin(np.sqrt(z.astype(complex)))
    zr = np.real(z)
    out = np.empty(zr.shape, dtype=complex)
    neg = zr < 0
    w = np.sqrt(np.where(neg, 0.0, zr))
    big = (~neg) & (w > 1)
    small = (~neg) & (w <= 1)
    out[small] = np.arcsin(w[small])
    out[big] = np.pi / 2 - 1j * np.arccosh(w[big])
    out[neg] = 1j * np.arcsinh(np.sqrt(-zr[neg]))
    return out


def _setup_longitudinal(k0dx2_epsilon, kt_sq_terms, ka, ind_zero_ky,
                        want_conj: bool) -> Dict[str, Any]:
    """setup_channels.m:179-238 (2D) / setup_channels_3D.m:146-188 (3D).

    ``kt_sq_terms`` is the tuple of transverse terms subtracted in MATLAB's
    order: (sin(kydx/2).^2,) in 2D, (sin(kxdx/2).^2, sin(kydx/2).^2) in 3D,
    each flattened in column-major order.
    """
    k2e = complex(k0dx2_epsilon)
    is_real = (k2e.imag == 0)
    z = (0.25 * k2e.real) if is_real else (0.25 * k2e)   # :185 / 3D :152
    for term in kt_sq_terms:
        z = z - term
    kxdx = 2 * _asin_sqrt_matlab(np.asarray(z), is_real)  # :190
    zr = np.real(z)
    zi = np.imag(z) if not is_real else np.zeros_like(zr)
    ind_prop = np.nonzero((zr > 0) & (zr < 1))[0] + 1     # :195 (1-based)
    side: Dict[str, Any] = {}
    side["N_prop"] = int(ind_prop.size)                  # :198
    # :211-215 branch flip
    if (not is_real) or (is_real and k2e.real > 4):
        ind_flip = ((zr < 0) & (zi < 0)) | ((zr > 1) & (zi <= 0))
        kxdx = np.where(ind_flip, -kxdx, kxdx)
    side["kxdx"] = kxdx
    side["ind_prop"] = ind_prop
    side["sqrt_mu"] = np.sqrt(np.sin(kxdx[ind_prop - 1]).astype(complex))  # :219
    if is_real and np.all(np.imag(side["sqrt_mu"]) == 0):
        side["sqrt_mu"] = np.real(side["sqrt_mu"]).astype(complex)
    # :222-236
    if want_conj:
        Np = side["N_prop"]
        if ka is None:
            side["ind_prop_conj"] = np.arange(1, Np + 1)
        elif ka == 0:
            if (ind_zero_ky in set(ind_prop.tolist())) or (Np % 2 == 0):
                side["ind_prop_conj"] = np.arange(Np, 0, -1)
            else:
                side["ind_prop_conj"] = np.concatenate([np.arange(Np - 1, 0, -1), [Np]])
    return side


def setup_channels(ny: int, BC, k0dx, epsilon_L, epsilon_R=None) -> Dict[str, Any]:
    """setup_channels.m:1-176.

    Returns a dict with keys 'kydx' (ny,), 'fun_phi' (callable kydx -> ny x
    len(kydx) matrix), 'L' and 'R' (dicts with 'N_prop', 'kxdx', 'ind_prop'
    (1-based), 'sqrt_mu', and 'ind_prop_conj' where it exists).
    When epsilon_R is None or NaN only the left side is set up and
    ``channels['R'] = {'N_prop': nan}`` (``:171-174``).
    """
    if not (isinstance(ny, (int, np.integer)) and ny > 0):
        raise ValueError("ny must be a positive integer scalar")
    if not _is_numeric_scalar(k0dx):
        raise ValueError("k0dx must be a numeric scalar")
    if not _is_numeric_scalar(epsilon_L):
        raise ValueError("epsilon_L must be a numeric scalar")
    two_sided = not (epsilon_R is None or (np.isscalar(epsilon_R) and np.isnan(epsilon_R)))
    if two_sided and not _is_numeric_scalar(epsilon_R):
        raise ValueError("epsilon_R must be a numeric scalar")
    kind, ka = _bc_to_kind(BC)
    if kind == "Bloch" and np.imag(ka) != 0:
        raise ValueError(f"k*a = {np.real(ka):g} + 1i*{np.imag(ka):g} is a complex number; "
                         "has to be real for a complete orthonormal transverse basis.")
    if ka is not None:
        ka = float(np.real(ka))
    ind_zero_ky = None
    ch: Dict[str, Any] = {}
    m = np.arange(1, ny + 1, dtype=float)
    mh = np.arange(0.5, ny, 1.0)  # 0.5:ny
    if kind == "Bloch":  # :122-133
        ind_zero_ky = (ny + 1) // 2 if ny % 2 == 1 else ny // 2
        kydx = (ka / ny) + (m - ind_zero_ky) * (2 * np.pi / ny)
        s = np.sqrt(ny)

        def fun_phi(k, m=m, s=s):
            k = np.atleast_1d(np.asarray(k, dtype=float))
            return np.exp(1j * np.outer(m, k)) / s
    elif kind == "Dirichlet":  # :134-138
        kydx = m * (np.pi / (ny + 1))
        s = np.sqrt(2 / (ny + 1))

        def fun_phi(k, m=m, s=s):
            k = np.atleast_1d(np.asarray(k, dtype=float))
            return np.sin(np.outer(m, k)) * s
    elif kind == "Neumann":  # :139-146
        kydx = (m - 1) * (np.pi / ny)
        s = np.sqrt(2 / ny)

        def fun_phi(k, mh=mh, s=s):
            k = np.atleast_1d(np.asarray(k, dtype=float))
            return (np.cos(np.outer(mh, k)) - ((k == 0) * (1 - np.sqrt(1 / 2)))[None, :]) * s
    elif kind == "DirichletNeumann":  # :147-151
        kydx = mh * (np.pi / (ny + 0.5))
        s = np.sqrt(2 / (ny + 0.5))

        def fun_phi(k, m=m, s=s):
            k = np.atleast_1d(np.asarray(k, dtype=float))
            return np.sin(np.outer(m, k)) * s
    else:  # NeumannDirichlet :152-156
        kydx = mh * (np.pi / (ny + 0.5))
        s = np.sqrt(2 / (ny + 0.5))

        def fun_phi(k, mh=mh, s=s):
            k = np.atleast_1d(np.asarray(k, dtype=float))
            return np.cos(np.outer(mh, k)) * s
    ch["kydx"] = kydx
    ch["fun_phi"] = fun_phi
    ch["bc_kind"] = kind
    ch["ka"] = ka
    kt = (np.sin(kydx / 2) ** 2,)
    ch["L"] = _setup_longitudinal((k0dx ** 2) * epsilon_L, kt, ka, ind_zero_ky, True)  # :162
    if two_sided:
        if epsilon_R == epsilon_L:
            ch["R"] = ch["L"]  # :166-167
        else:
            ch["R"] = _setup_longitudinal((k0dx ** 2) * epsilon_R, kt, ka, ind_zero_ky, True)
    else:
        ch["R"] = {"N_prop": np.nan}
    return ch


# --------------------------------------------------------------------------
# setup_channels_3D.m
# --------------------------------------------------------------------------
def _bc3d(BC):
    """Normalise the 3D xyBC (setup_channels_3D.m:66-99): returns (kind, kxa, kya)."""
    if isinstance(BC, str):
        b = BC.lower()
        if b == "bloch":
            raise ValueError("To use Bloch periodic boundary condition, set BC to [kx*ax, ky*ay]")
        if b == "periodic":
            return "Bloch", 0.0, 0.0
        if b in ("dirichlet", "pec"):
            return "Dirichlet", None, None
        raise ValueError(f"Boundary condition BC = {BC} is not an eligible option")
    arr = np.asarray(BC)
    if arr.size == 2 and np.issubdtype(arr.dtype, np.number):
        kxa, kya = arr.ravel()[0], arr.ravel()[1]
        if np.imag(kxa) != 0:
            raise ValueError("kx*a is a complex number; has to be real for a complete orthonormal transverse basis.")
        if np.imag(kya) != 0:
            raise ValueError("ky*a is a complex number; has to be real for a complete orthonormal transverse basis.")
        return "Bloch", float(np.real(kxa)), float(np.real(kya))
    raise ValueError("Boundary condition BC has to be a character vector or string, or numeric "
                     "vector with 2 elements (for Bloch periodic BC)")


def setup_channels_3D(nx: int, ny: int, BC, k0dx, epsilon_L, epsilon_R=None) -> Dict[str, Any]:
    """setup_channels_3D.m:1-143.

    'kxdx'/'kydx' are nx-by-ny arrays (x fastest, MATLAB layout); 'L'/'R'
    hold 'kzdx' (nx-by-ny), 'ind_prop' (1-based column-major linear
    indices), 'N_prop' and 'sqrt_mu'.  There is no ind_prop_conj in 3D.
    """
    if not (isinstance(nx, (int, np.integer)) and nx > 0):
        raise ValueError("nx must be a positive integer scalar")
    if not (isinstance(ny, (int, np.integer)) and ny > 0):
        raise ValueError("ny must be a positive integer scalar")
    two_sided = not (epsilon_R is None or (np.isscalar(epsilon_R) and np.isnan(epsilon_R)))
    kind, kxa, kya = _bc3d(BC)
    ch: Dict[str, Any] = {}
    mx = np.arange(1, nx + 1, dtype=float)
    my = np.arange(1, ny + 1, dtype=float)
    if kind == "Bloch":  # :102-118
        ind0x = (nx + 1) // 2 if nx % 2 == 1 else nx // 2
        ind0y = (ny + 1) // 2 if ny % 2 == 1 else ny // 2
        kx1 = (kxa / nx) + (mx - ind0x) * (2 * np.pi / nx)
        ky1 = (kya / ny) + (my - ind0y) * (2 * np.pi / ny)
        s = np.sqrt(nx * ny)

        def fun_phi(kx, ky, mx=mx, my=my, s=s):
            return np.outer(np.exp(1j * mx * kx), np.exp(1j * my * ky) / s)
    else:  # Dirichlet :119-123
        kx1 = mx * (np.pi / (nx + 1))
        ky1 = my * (np.pi / (ny + 1))
        s = np.sqrt(4 / ((nx + 1) * (ny + 1)))

        def fun_phi(kx, ky, mx=mx, my=my, s=s):
            return np.outer(np.sin(mx * kx), np.sin(my * ky) * s)
    ch["kxdx"] = np.repeat(kx1[:, None], ny, axis=1)
    ch["kydx"] = np.repeat(ky1[None, :], nx, axis=0)
    ch["fun_phi"] = fun_phi
    ch["bc_kind"] = kind
    ch["ka"] = (kxa, kya)
    kt = ((np.sin(ch["kxdx"] / 2) ** 2).ravel(order="F"), (np.sin(ch["kydx"] / 2) ** 2).ravel(order="F"))

    def longi(k2e):
        side = _setup_longitudinal(k2e, kt, None, None, False)
        side["kzdx"] = side.pop("kxdx").reshape((nx, ny), order="F")
        return side

    ch["L"] = longi((k0dx ** 2) * epsilon_L)
    if two_sided:
        ch["R"] = ch["L"] if epsilon_R == epsilon_L else longi((k0dx ** 2) * epsilon_R)
    else:
        ch["R"] = {"N_prop": np.nan}
    return ch


# --------------------------------------------------------------------------
# in/out parsing: cal_smatrix_RGF.m:103-178 (identical in the 3D file :101-176)
# --------------------------------------------------------------------------
def parse_channel_request(req, kind: str, N_prop_L: int, N_prop_R: int):
    """Return (ind_L, ind_R) as 1-based int arrays.

    ``req`` is a dict (MATLAB struct with fields ind_{kind}_L/R) or a list
    (MATLAB cell of 'left'/'L'/'right'/'R'); anything else raises.
    """
    ind_L = np.zeros(0, dtype=np.int64)
    ind_R = np.zeros(0, dtype=np.int64)
    if isinstance(req, dict):
        for side, Np in (("L", N_prop_L), ("R", N_prop_R)):
            key = f"ind_{kind}_{side}"
            if key in req:
                v = np.asarray(req[key]).reshape(-1)
                if v.size:
                    ok = np.issubdtype(v.dtype, np.number) and not np.iscomplexobj(v)
                    ok = ok and np.all(np.round(v) == v) and v.min() > 0 and v.max() <= Np
                    if not ok:
                        raise ValueError(f"{kind}.{key}, when specified, must be an array of positive "
                                         f"integers not exceeding N_prop_{side}={Np}")
                v = v.astype(np.int64)
                if side == "L":
                    ind_L = v
                else:
                    ind_R = v
    elif isinstance(req, (list, tuple)):
        for k, el in enumerate(req, start=1):
            if not isinstance(el, str):
                warnings.warn(f"element {kind}{{{k}}} has wrong format and is ignored; should be one "
                              "of {'left', 'right', 'L', 'R'}")
                continue
            if el in ("left", "L"):
                ind_L = np.arange(1, N_prop_L + 1, dtype=np.int64)
            elif el in ("right", "R"):
                ind_R = np.arange(1, N_prop_R + 1, dtype=np.int64)
            else:
                warnings.warn(f"element {kind}{{{k}}} = {el} ignored; should be one of "
                              "{'left', 'right', 'L', 'R'}")
    else:
        raise ValueError(f"input argument '{kind}' must be a structure or a cell array")
    return ind_L, ind_R


def _delta_matrix(ind_out_L, ind_out_R, ind_in_L, ind_in_R) -> np.ndarray:
    """cal_smatrix_RGF.m:286-288: D has a 1 wherever an output index equals
    an input index on the same side (MATLAB ``intersect``, first occurrence)."""
    NoL, NoR, NiL, NiR = len(ind_out_L), len(ind_out_R), len(ind_in_L), len(ind_in_R)
    D = np.zeros((NoL + NoR, NiL + NiR))
    _, io, ii = np.intersect1d(ind_out_L, ind_in_L, return_indices=True)
    D[io, ii] = 1
    _, io, ii = np.intersect1d(ind_out_R, ind_in_R, return_indices=True)
    D[NoL + io, NiL + ii] = 1
    return D


# --------------------------------------------------------------------------
# the slice recursion: cal_smatrix_RGF.m:186-289 / cal_smatrix_RGF_3D.m:184-304
# --------------------------------------------------------------------------
def _recursion(phi, chL, chR, eps_R_eq_L, A0, k0dx2, eps_slices, ind_in_L, ind_in_R,
               ind_out_L, ind_out_R, slice_hook: Callable | None = None):
    """Shared body of both drivers (the 2D and 3D files are identical here).

    ``eps_slices`` is an (N, L) array whose column n is the slice
    permittivity in the driver's ordering.  ``slice_hook(n)`` is called after
    each slice (used by the CPU-baseline timer to stop early).
    """
    N = phi.shape[0]
    NiL, NiR, NoL, NoR = len(ind_in_L), len(ind_in_R), len(ind_out_L), len(ind_out_R)
    kxL = chL["kxdx"].ravel(order="F")
    kxR = chR["kxdx"].ravel(order="F")
    # :191-195
    B_L = phi[:, chL["ind_prop"][ind_in_L - 1] - 1] * chL["sqrt_mu"][ind_in_L - 1][None, :]
    B_R = phi[:, chR["ind_prop"][ind_in_R - 1] - 1] * chR["sqrt_mu"][ind_in_R - 1][None, :]
    C_L = chL["sqrt_mu"][ind_out_L - 1][:, None] * phi[:, chL["ind_prop"][ind_out_L - 1] - 1].conj().T
    C_R = chR["sqrt_mu"][ind_out_R - 1][:, None] * phi[:, chR["ind_prop"][ind_out_R - 1] - 1].conj().T
    # :198-203
    G0_L = (phi * np.exp(1j * kxL)[None, :]) @ phi.conj().T
    G0_R = G0_L if eps_R_eq_L else (phi * np.exp(1j * kxR)[None, :]) @ phi.conj().T
    I = np.eye(N)
    L = eps_slices.shape[1]

    def A_nn(n):  # :221 etc.; spdiags of the slice permittivity
        return A0 - np.diag(k0dx2 * eps_slices[:, n])

    inv = sla.inv
    solve = np.linalg.solve
    if NiR == 0 and NoR == 0:  # :217-225
        G_LL = G0_R
        for n in range(L - 1, -1, -1):
            G_LL = inv(A_nn(n) - G_LL)
            if slice_hook:
                slice_hook(n)
        G_LL = solve(I - G0_L @ G_LL, G0_L)
        S = (-2j) * (C_L @ (G_LL @ B_L))
    elif NiR == 0:  # :226-236
        G_LL = G0_R
        G_RL = G0_R
        for n in range(L - 1, -1, -1):
            G_LL = inv(A_nn(n) - G_LL)
            G_RL = G_RL @ G_LL
            if slice_hook:
                slice_hook(n)
        G_LL = solve(I - G0_L @ G_LL, G0_L)
        G_RL = G_RL @ G_LL
        S = (-2j) * np.vstack([(C_L @ G_LL) @ B_L, C_R @ (G_RL @ B_L)])
    elif NiL == 0 and NoL == 0:  # :237-245
        G_RR = G0_L
        for n in range(L):
            G_RR = inv(A_nn(n) - G_RR)
            if slice_hook:
                slice_hook(n)
        G_RR = solve(I - G0_R @ G_RR, G0_R)
        S = (-2j) * (C_R @ (G_RR @ B_R))
    elif NiL == 0:  # :246-256
        G_RR = G0_L
        G_LR = G0_L
        for n in range(L):
            G_RR = inv(A_nn(n) - G_RR)
            G_LR = G_LR @ G_RR
            if slice_hook:
                slice_hook(n)
        G_RR = solve(I - G0_R @ G_RR, G0_R)
        G_LR = G_LR @ G_RR
        S = (-2j) * np.vstack([C_L @ (G_LR @ B_R), (C_R @ G_RR) @ B_R])
    else:  # :257-280
        G_RR = G0_L
        G_RL = G0_L
        G_LL = G0_L
        G_LR = G0_L
        for n in range(L):
            G_RR = inv(A_nn(n) - G_RR)
            G_RL = G_RR @ G_RL
            G_LL = G_LL + G_LR @ G_RL
            G_LR = G_LR @ G_RR
            if slice_hook:
                slice_hook(n)
        G_RR = solve(I - G0_R @ G_RR, G0_R)
        G_RL = G_RR @ G_RL
        G_LL = G_LL + G_LR @ G_RL
        G_LR = G_LR @ G_RR
        S = (-2j) * np.block([[C_L @ (G_LL @ B_L), C_L @ (G_LR @ B_R)],
                              [C_R @ (G_RL @ B_L), C_R @ (G_RR @ B_R)]])
    return S - _delta_matrix(ind_out_L, ind_out_R, ind_in_L, ind_in_R)


def _check_syst(syst, bc_key: str):
    """cal_smatrix_RGF.m:79-88 (and _3D.m:77-86)."""
    if not (isinstance(syst, dict) or hasattr(syst, "__dict__")):
        raise ValueError("syst must be a structure")
    for key in ("epsilon", "epsilon_L", "epsilon_R", "k0dx", bc_key):
        if not _has(syst, key):
            raise ValueError(f"syst.{key} must be provided")
    for key in ("epsilon_L", "epsilon_R", "k0dx"):
        if not _is_numeric_scalar(_field(syst, key)):
            raise ValueError(f"syst.{key} must be a numeric scalar")


def cal_smatrix_RGF(syst, out, in_, slice_hook=None):
    """cal_smatrix_RGF.m:1-291.  Returns (smatrix, channels).

    ``syst`` has fields epsilon ([ny, nx] array), epsilon_L, epsilon_R,
    k0dx and yBC (string or, deviating from ``:89`` per quirk Q1, a numeric
    Bloch phase ka).  ``out``/``in_`` are a dict (MATLAB struct) or a list
    (MATLAB cell).
    """
    _check_syst(syst, "yBC")
    eps = np.asarray(_field(syst, "epsilon"))
    if eps.ndim != 2 or not np.issubdtype(eps.dtype, np.number):
        raise ValueError("syst.epsilon must be a numeric matrix")
    ny, nx = eps.shape  # :92
    if ny == 0:
        raise ValueError("need at least one site along the transverse (y) direction")
    yBC = _field(syst, "yBC")
    eL, eR, k0dx = _field(syst, "epsilon_L"), _field(syst, "epsilon_R"), _field(syst, "k0dx")
    channels = setup_channels(int(ny), yBC, k0dx, eL, eR)  # :98
    NpL, NpR = channels["L"]["N_prop"], channels["R"]["N_prop"]
    ind_in_L, ind_in_R = parse_channel_request(in_, "in", NpL, NpR)
    ind_out_L, ind_out_R = parse_channel_request(out, "out", NpL, NpR)
    Ni = len(ind_in_L) + len(ind_in_R)
    No = len(ind_out_L) + len(ind_out_R)
    if Ni == 0 or No == 0:  # :181-184
        return np.zeros((No, Ni)), channels
    phi = channels["fun_phi"](channels["kydx"])  # :187
    A0 = -build_laplacian_1d(int(ny), yBC) + 2 * np.eye(ny)  # :209
    S = _recursion(phi, channels["L"], channels["R"], eR == eL, A0, k0dx ** 2,
                   eps.astype(complex), ind_in_L, ind_in_R, ind_out_L, ind_out_R, slice_hook)
    return S, channels


def cal_smatrix_RGF_3D(syst, out, in_, slice_hook=None):
    """cal_smatrix_RGF_3D.m:1-306.  Returns (smatrix, channels).

    ``syst.epsilon`` is an [nx, ny, nz] array (a 2D [nx, ny] array means
    nz = 1); ``syst.xyBC`` is 'periodic', 'Dirichlet'/'PEC' or [kxa, kya].
    """
    _check_syst(syst, "xyBC")
    eps = np.asarray(_field(syst, "epsilon"))
    if eps.ndim not in (2, 3) or not np.issubdtype(eps.dtype, np.number):
        raise ValueError("syst.epsilon must be a 3D array")
    if eps.ndim == 2:
        eps = eps[:, :, None]
    nx, ny, nz = eps.shape  # :89
    nxy = nx * ny
    if nxy == 0:
        raise ValueError("need at least one site along the transverse directions (x,y)")
    xyBC = _field(syst, "xyBC")
    eL, eR, k0dx = _field(syst, "epsilon_L"), _field(syst, "epsilon_R"), _field(syst, "k0dx")
    channels = setup_channels_3D(int(nx), int(ny), xyBC, k0dx, eL, eR)  # :96
    NpL, NpR = channels["L"]["N_prop"], channels["R"]["N_prop"]
    ind_in_L, ind_in_R = parse_channel_request(in_, "in", NpL, NpR)
    ind_out_L, ind_out_R = parse_channel_request(out, "out", NpL, NpR)
    Ni = len(ind_in_L) + len(ind_in_R)
    No = len(ind_out_L) + len(ind_out_R)
    if Ni == 0 or No == 0:
        return np.zeros((No, Ni)), channels
    # :185-188: column a of phi is fun_phi(kxdx(a), kydx(a)) reshaped, x fastest
    kxf = channels["kxdx"].ravel(order="F")
    kyf = channels["kydx"].ravel(order="F")
    phi = np.empty((nxy, nxy), dtype=complex)
    for a in range(nxy):
        phi[:, a] = channels["fun_phi"](kxf[a], kyf[a]).ravel(order="F")
    # :209-224
    if isinstance(xyBC, str):
        xBC = yBC = xyBC
    else:
        xBC, yBC = np.asarray(xyBC).ravel()[0], np.asarray(xyBC).ravel()[1]
        xBC, yBC = float(np.real(xBC)), float(np.real(yBC))
    Lx = build_laplacian_1d(int(nx), xBC)
    Ly = build_laplacian_1d(int(ny), yBC)
    A0 = -np.kron(np.eye(ny), Lx) - np.kron(Ly, np.eye(nx)) + 2 * np.eye(nxy)
    chL = dict(channels["L"])
    chR = dict(channels["R"])
    chL["kxdx"] = chL["kzdx"]
    chR["kxdx"] = chR["kzdx"]
    eps_slices = eps.reshape((nxy, nz), order="F").astype(complex)  # :279
    S = _recursion(phi, chL, chR, eR == eL, A0, k0dx ** 2, eps_slices,
                   ind_in_L, ind_in_R, ind_out_L, ind_out_R, slice_hook)
    return S, channels
