"""torch.autograd interface to the Laplace particle FMM.

    phi_i = sum_j G(x_i - y_j) q_j,     G(r) = 1 / (4 pi |r|),  r == 0 excluded

with targets x (n_trg, 3), sources y (n_src, 3) and densities q (n_src,).
There is no counterpart in the reference; the forward pass is the reference's
particle FMM (PVFMMEval, src/pvfmm-wrapper.cpp:543-811) run with the
LaplacePotGrad kernel, which returns phi and E = -grad phi at the targets in
one pass (the gradient's sign convention is that of the reference's
laplace_grad kernel, include/kernel.txx:1300-1344).

Backward, with g = dL/dphi:

    dL/dq_j = sum_i G(y_j - x_i) g_i                      (potential part of A)
    dL/dy_j = q_j sum_i g_i (x_i - y_j) / (4 pi |x_i - y_j|^3) = -q_j A_E,j
    dL/dx_i = g_i grad phi(x_i) = -g_i E_i

where A = (A_phi, A_E) is one more LaplacePotGrad FMM with densities g at the
targets evaluated at the sources (PVFMMEvalAdjointDevice*).  When the sources
and targets are the same tensor that evaluation reuses the forward pass's
octree; otherwise a companion context builds the exchanged tree.  Gradients
with respect to the same tensor passed as sources and targets add up.

All tensors live on one CUDA device.  Coordinates always enter the library
as FP64 (a float32 tensor is widened on the device), so the bounding-box map
adds no FP32 rounding to the point positions: with FP32 coordinates mapped in
FP32, as the reference's float interface does, close pairs lose ~1e-4 of the
gradient's accuracy.  The arithmetic form is `precision`: "mixed" (FP32 near
field and V-list, FP64 check->equivalent chain) or "plain" (FP64 throughout);
outputs and gradients come back in the inputs' dtypes.  Double backward is not
supported.
"""
from typing import Optional

import numpy as np
import torch

from . import PRECISION_MIXED, PRECISION_PLAIN, FMMKernel, FMMParticleContext


class LaplaceFMM:
    """Differentiable Laplace single-layer potential through the particle FMM.

    ``fmm(src, den)`` evaluates at the sources themselves (one octree for
    both roles); ``fmm(src, den, trg)`` at separate targets.
    """

    def __init__(self, max_points: int = 256, multipole_order: int = 8, precision: str = "mixed",
                 unit_box: bool = False):
        if precision not in ("mixed", "plain"):
            raise ValueError('precision must be "mixed" or "plain"')
        self.precision = precision
        self.ctx = FMMParticleContext(-1.0, max_points, multipole_order, FMMKernel.LaplacePotGrad, dtype=np.float64,
                                      precision=PRECISION_MIXED if precision == "mixed" else PRECISION_PLAIN)
        if unit_box:
            self.ctx.set_unit_box(True)
        self.generation = 0   # trees built so far; backward reuses the tree only if unchanged

    def __call__(self, src: torch.Tensor, den: torch.Tensor, trg: Optional[torch.Tensor] = None) -> torch.Tensor:
        if trg is None:
            trg = src
        return _LaplaceFMMFunction.apply(self, src, den, trg)

    def close(self):
        self.ctx.close()


def _check(name, t, cols):
    if not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor")
    if cols and (t.dim() != 2 or t.shape[1] != cols):
        raise ValueError(f"{name} must have shape (n, {cols})")
    if not cols and t.dim() != 1:
        raise ValueError(f"{name} must have shape (n,)")


class _LaplaceFMMFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, fmm: LaplaceFMM, src, den, trg):
        _check("src", src, 3)
        _check("den", den, 0)
        _check("trg", trg, 3)
        if den.shape[0] != src.shape[0]:
            raise ValueError("den must have one value per source")
        alias = trg is src or (trg.data_ptr() == src.data_ptr() and trg.shape == src.shape
                               and trg.stride() == src.stride() and trg.dtype == src.dtype)
        dt = torch.float64
        s = src.detach().to(dt).contiguous()
        q = den.detach().to(dt).contiguous()
        t = s if alias else trg.detach().to(dt).contiguous()
        out = torch.empty(t.shape[0], 4, dtype=dt, device=s.device)
        stream = torch.cuda.current_stream(s.device).cuda_stream
        with torch.cuda.device(s.device):
            fmm.ctx.evaluate_device(s.data_ptr(), q.data_ptr(), s.shape[0], t.data_ptr(), out.data_ptr(), t.shape[0],
                                    True, stream)
        fmm.generation += 1
        ctx.fmm = fmm
        ctx.gen = fmm.generation
        ctx.alias = alias
        ctx.out_dtypes = (src.dtype, den.dtype, trg.dtype)
        ctx.save_for_backward(s, q, t, out)
        return out[:, 0].to(den.dtype)

    @staticmethod
    @torch.autograd.function.once_differentiable
    def backward(ctx, grad_phi):
        s, q, t, out = ctx.saved_tensors
        fmm = ctx.fmm
        need_src, need_den, need_trg = ctx.needs_input_grad[1], ctx.needs_input_grad[2], ctx.needs_input_grad[3]
        g = grad_phi.detach().to(torch.float64).contiguous()
        g_src = g_den = g_trg = None
        if need_src or need_den:
            adj = torch.empty(s.shape[0], 4, dtype=torch.float64, device=s.device)
            reuse = ctx.alias and fmm.generation == ctx.gen
            stream = torch.cuda.current_stream(s.device).cuda_stream
            with torch.cuda.device(s.device):
                fmm.ctx.evaluate_adjoint_device(s.data_ptr(), s.shape[0], t.data_ptr(), g.data_ptr(), t.shape[0],
                                                adj.data_ptr(), not reuse, stream)
            if ctx.alias and not reuse:
                fmm.generation += 1   # the context's tree now belongs to this pass's points
            if need_den:
                g_den = adj[:, 0].to(ctx.out_dtypes[1])
            if need_src:
                g_src = (-q[:, None] * adj[:, 1:]).to(ctx.out_dtypes[0])
        if need_trg:
            g_trg = (-g[:, None] * out[:, 1:]).to(ctx.out_dtypes[2])
        return None, g_src, g_den, g_trg
