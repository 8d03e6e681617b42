"""GPU-resident system operator and differentiable projector.

``SPECTOperator(plan, index)`` is the device counterpart of the LinearMapAA
closures the reference builds in ``Ablock`` (src/ml-os-em.jl:70-84,
``forw!``/``back!`` calling ``project!``/``backproject!``): ``A @ x`` projects,
``A.T @ y`` back-projects, both on torch CUDA tensors that never leave the GPU.

``project_ad`` / ``backproject_ad`` are the custom-Jacobian wrappers of the
deep-learning example (docs/lit/examples/6-dl.jl:152-156,
``@adjoint projectb(x) = A*x, dy -> (A'*dy,)``): the backward pass of a
projection is a back-projection and vice versa, so autograd never traces
through the system matrix.

Tensors use the Julia shapes and column-major layout of the C ABI:
image ``(nx, ny, nz)`` and views ``(nx, nz, nindex)`` with x fastest in
memory.  ``julia_empty``/``to_julia_layout`` make such tensors from torch's
row-major ones (a permuted view of a contiguous ``(nz, ny, nx)`` tensor).
All calls run on torch's current CUDA stream.
"""
import numpy as np

from . import SPECTplan, project_, backproject_


def _torch():
    import torch

    return torch


def julia_empty(shape, device="cuda", zero=False):
    """float32 tensor of Julia ``shape`` laid out column-major on ``device``."""
    torch = _torch()
    rev = tuple(reversed(shape))
    t = (torch.zeros if zero else torch.empty)(rev, dtype=torch.float32, device=device)
    return t.permute(*reversed(range(len(shape))))


def to_julia_layout(t):
    """``t`` (Julia shape) as float32, column-major, on its device (copies
    only when its layout differs)."""
    torch = _torch()
    t = t.detach().to(torch.float32)
    nd = t.dim()
    perm = tuple(reversed(range(nd)))
    return t.permute(*perm).contiguous().permute(*perm)


class SPECTOperator:
    """``A = SPECTOperator(plan, index=None)``: the (nindex·nx·nz) × (nx·ny·nz)
    system matrix of the views ``index`` (all views when None)."""

    def __init__(self, plan: SPECTplan, index=None, adjoint=False):
        self.plan = plan
        self.index = None if index is None else np.ascontiguousarray(np.asarray(index, np.int32).ravel())
        self.nindex = plan.nview if self.index is None else int(self.index.size)
        self.adjoint = adjoint
        nx, ny, nz = plan.imgsize
        self.imgsize = (nx, ny, nz)
        self.viewsize = (nx, nz, self.nindex)

    @property
    def shape(self):
        m, n = int(np.prod(self.viewsize)), int(np.prod(self.imgsize))
        return (n, m) if self.adjoint else (m, n)

    @property
    def T(self):
        return SPECTOperator(self.plan, self.index, adjoint=not self.adjoint)

    H = T

    def _stream(self):
        return _torch().cuda.current_stream()

    def forward(self, x):
        """views = P x (project!); ``x`` is a CUDA tensor of the image shape."""
        x = to_julia_layout(x)
        y = julia_empty(self.viewsize, device=x.device)
        project_(y, x, self.plan, index=self.index, stream=self._stream())
        return y

    def backward(self, y):
        """image = Pᵀ y (backproject!); ``y`` is a CUDA tensor of the views shape."""
        y = to_julia_layout(y)
        x = julia_empty(self.imgsize, device=y.device)
        backproject_(x, y, self.plan, index=self.index, stream=self._stream())
        return x

    def __matmul__(self, v):
        return self.backward(v) if self.adjoint else self.forward(v)

    __call__ = __matmul__


def _autograd_fns():
    torch = _torch()

    class _Project(torch.autograd.Function):
        @staticmethod
        def forward(ctx, x, op):
            ctx.op = op
            return op.forward(x)

        @staticmethod
        def backward(ctx, dy):
            return ctx.op.backward(dy), None

    class _Backproject(torch.autograd.Function):
        @staticmethod
        def forward(ctx, y, op):
            ctx.op = op
            return op.backward(y)

        @staticmethod
        def backward(ctx, dx):
            return ctx.op.forward(dx), None

    return _Project, _Backproject


_FNS = None


def _fns():
    global _FNS
    if _FNS is None:
        _FNS = _autograd_fns()
    return _FNS


def project_ad(x, A: SPECTOperator):
    """Differentiable ``A @ x``; its vector-Jacobian product is ``A.T @ dy``."""
    return _fns()[0].apply(x, A)


def backproject_ad(y, A: SPECTOperator):
    """Differentiable ``A.T @ y``; its vector-Jacobian product is ``A @ dx``."""
    return _fns()[1].apply(y, A)
