"""torch.autograd bridge for the adjoint (no counterpart in the reference crate).

``implicit_function(positions, normals, queries, params)`` returns chi at the (K, 3) model-space
``queries``: the implicit function of the screened Poisson solve of the oriented points
(src/fem_tree.rs:130-299 and the evaluation of :490-513).  Its backward runs the library's
adjoint (``pr_ctx_loss_backward``): one more solve with the same operator, then per-point
gathers, and returns dL/dpositions and dL/dnormals.  The unit-cube transform, which follows
the bounding box of the positions, is held fixed (not differentiated).  Tensors may live on
any device; the solve runs on the context's GPU and the results come back in the inputs'
dtype and device.
"""
import torch

from . import Context, PR_SOLVE_CONVERGED, ReconstructParams


class _ImplicitFunction(torch.autograd.Function):
    @staticmethod
    def forward(fctx, positions, normals, queries, params, context):
        pts = torch.cat([positions.detach(), normals.detach()], dim=1).to("cpu", torch.float64).numpy()
        q = queries.detach().to("cpu", torch.float64).numpy()
        context.solve(pts, params)
        _, _, m = context.info()
        m = m.reshape(4, 4).T  # column-major -> row-major
        qu = q @ m[:3, :3].T + m[:3, 3]
        chi = context.evaluate(qu)
        fctx.context = context
        fctx.queries = q
        fctx.n = pts.shape[0]
        fctx.meta = (positions.dtype, positions.device, normals.dtype, normals.device)
        return torch.from_numpy(chi).to(queries.device, queries.dtype)

    @staticmethod
    def backward(fctx, grad_chi):
        g = grad_chi.detach().to("cpu", torch.float64).numpy()
        _, dp, dn, _ = fctx.context.loss_backward(fctx.queries, dl_dchi=g, n_points=fctx.n)
        pdt, pdev, ndt, ndev = fctx.meta
        return (torch.from_numpy(dp).to(pdev, pdt), torch.from_numpy(dn).to(ndev, ndt), None, None, None)


def implicit_function(positions, normals, queries, params=None, context=None):
    """chi at `queries`, differentiable w.r.t. `positions` and `normals` ((N, 3) each).

    The backward must run before `context` solves again (it reads the context's state)."""
    params = params or ReconstructParams(point_weight=4.0)
    if params.solve_mode != PR_SOLVE_CONVERGED:
        raise ValueError("the adjoint needs solve_mode PR_SOLVE_CONVERGED")
    context = context or _default_context()
    return _ImplicitFunction.apply(positions, normals, queries, params, context)


_CTX = None


def _default_context():
    global _CTX
    if _CTX is None:
        _CTX = Context(0)
    return _CTX


__all__ = ["implicit_function"]
