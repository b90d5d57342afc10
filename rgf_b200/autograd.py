"""torch.autograd harness over the C ABI gradient entry (rgf_smatrix_grad_2d).

``SMatrix.apply(eps, syst, out, in_)`` returns S (complex128, host tensor)
for a real permittivity tensor ``eps`` of shape [ny, nx]; its backward calls
the library's adjoint sweep.  The library does all GPU work; torch only
carries the gradient bookkeeping.

With torch's convention for complex outputs, the incoming gradient is
grad_S = dL/dRe(S) + i dL/dIm(S), so dL/d eps = Re sum conj(grad_S) dS/d eps,
i.e. D = conj(grad_S) / 2 and dL/d eps = 2 Re g.
"""
from __future__ import annotations

import numpy as np
import torch

from .api import smatrix_grad_RGF


class SMatrix(torch.autograd.Function):
    @staticmethod
    def forward(ctx, eps, syst, out, in_):
        s = dict(syst, epsilon=eps.detach().cpu().numpy().astype(float))
        from .api import cal_smatrix_RGF
        S, _ = cal_smatrix_RGF(s, out, in_)
        ctx.save_for_backward(eps)
        ctx.args = (syst, out, in_)
        return torch.from_numpy(np.ascontiguousarray(S))

    @staticmethod
    def backward(ctx, grad_S):
        (eps,) = ctx.saved_tensors
        syst, out, in_ = ctx.args
        s = dict(syst, epsilon=eps.detach().cpu().numpy().astype(float))
        D = np.conj(grad_S.detach().cpu().numpy()) / 2.0
        _, g = smatrix_grad_RGF(s, out, in_, D)
        return torch.from_numpy(2.0 * np.real(g)).to(eps.dtype), None, None, None
