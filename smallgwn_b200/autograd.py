"""torch.autograd binding of the Taylor winding number's forward / backward C ABI pair.

    field = WindingField(vertices, faces, order=1, accuracy_scale=2.0)
    w = winding_number(vertices, queries, field)      # vertices (V, 3), queries (Q, 3): CUDA float32
    (g * w).sum().backward()                         # vertices.grad, queries.grad

The forward refits the BVH and its moments to the current vertex positions (topology fixed) and
runs gwnb_winding_taylor_forward_f32; the backward runs gwnb_winding_taylor_backward_f32, which
recomputes the traversal from the saved query buffers instead of storing it. Acceptance decisions
of the Taylor traversal are piecewise constant and carry no derivative.
"""
from __future__ import annotations

import numpy as np
import torch

from . import api


def _check(status: api.gwn_status, what: str) -> None:
    if not status.is_ok():
        raise RuntimeError(f"{what}: {status.message}")


class WindingField:
    """A triangle mesh with moving vertices: geometry, BVH4 and Taylor moments resident on the GPU."""

    def __init__(self, vertices: torch.Tensor, faces, order: int = 1, accuracy_scale: float = 2.0,
                 method: api.gwn_bvh_build_method = api.gwn_bvh_build_method.k_hploc) -> None:
        if order not in (0, 1):
            raise ValueError("the Taylor adjoint supports orders 0 and 1")
        v = vertices.detach().to("cpu", torch.float32).numpy()
        f = np.asarray(faces.cpu() if isinstance(faces, torch.Tensor) else faces, dtype=np.uint32)
        self.order = order
        self.accuracy_scale = float(accuracy_scale)
        self.geometry = api.gwn_geometry_object()
        _check(api.gwn_upload_geometry(self.geometry, v[:, 0], v[:, 1], v[:, 2], f[:, 0], f[:, 1], f[:, 2]),
               "upload")
        self.bvh = api.gwn_bvh4_object()
        _check(api.gwn_build_bvh(self.geometry, self.bvh, api.gwn_bvh_build_options(method=method)), "build")
        self.moment = api.gwn_bvh4_moment_object(order)
        _check(api.gwn_refit_bvh_moment(order, self.bvh, self.moment), "moments")

    def refit(self, vertices: torch.Tensor, stream: int) -> None:
        xyz = [vertices[:, k].detach().contiguous() for k in range(3)]
        _check(api.gwn_update_geometry(self.geometry, *xyz, stream), "update")
        _check(api.gwn_refit_bvh(self.geometry, self.bvh, stream), "refit")
        _check(api.gwn_refit_bvh_moment(self.order, self.bvh, self.moment, stream), "moments")


class _TaylorWinding(torch.autograd.Function):
    @staticmethod
    def forward(ctx, vertices: torch.Tensor, queries: torch.Tensor, field: WindingField) -> torch.Tensor:
        stream = torch.cuda.current_stream().cuda_stream
        field.refit(vertices, stream)
        q = [queries[:, k].detach().contiguous() for k in range(3)]
        out = torch.empty(queries.shape[0], dtype=torch.float32, device=queries.device)
        st, saved = api.gwn_winding_taylor_forward(field.order, field.bvh, field.moment, *q, out,
                                                   accuracy_scale=field.accuracy_scale, stream=stream)
        _check(st, "Taylor forward")
        ctx.field, ctx.saved, ctx.vertex_count = field, saved, vertices.shape[0]
        return out

    @staticmethod
    def backward(ctx, grad_out: torch.Tensor):
        field, saved = ctx.field, ctx.saved
        stream = torch.cuda.current_stream().cuda_stream
        g = grad_out.detach().contiguous().float()
        dv = dq = None
        if ctx.needs_input_grad[0]:
            dv = torch.empty(3, ctx.vertex_count, dtype=torch.float32, device=g.device)
        if ctx.needs_input_grad[1]:
            dq = torch.empty(3, g.numel(), dtype=torch.float32, device=g.device)
        vs = list(dv) if dv is not None else [None] * 3
        qs = list(dq) if dq is not None else [None] * 3
        _check(api.gwn_winding_taylor_backward(saved, field.geometry, field.bvh, field.moment, g, *vs, *qs,
                                               stream=stream), "Taylor backward")
        return (dv.t() if dv is not None else None), (dq.t() if dq is not None else None), None


def winding_number(vertices: torch.Tensor, queries: torch.Tensor, field: WindingField) -> torch.Tensor:
    """Taylor winding numbers of `queries` against the mesh at `vertices`, differentiable in both."""
    return _TaylorWinding.apply(vertices, queries, field)
