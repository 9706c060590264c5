"""torch.autograd.Function wrappers of the library's adjoint entry points (test harness): the
forward pass calls the propagation / closest-approach entry point, the backward pass the adjoint
(gpop_propagate_vjp, gpop_miss_gradient). CPU float64 tensors in, CPU tensors out."""
import numpy as np
import torch


def _np(t):
    return t.detach().cpu().numpy().astype(np.float64)


class Propagate(torch.autograd.Function):
    """(r0, v0) [n, 3] -> (r_N, v_N) after `steps` GJ8 steps (FP64 context)."""

    @staticmethod
    def forward(fctx, r0, v0, gctx, start, h, steps):
        rN, vN = gctx.propagate(start, h, steps, _np(r0), _np(v0))
        fctx.save_for_backward(r0, v0)
        fctx.args = (gctx, start, h, steps)
        return torch.from_numpy(rN), torch.from_numpy(vN)

    @staticmethod
    def backward(fctx, g_r, g_v):
        r0, v0 = fctx.saved_tensors
        gctx, start, h, steps = fctx.args
        gr, gv = gctx.propagate_vjp(start, h, steps, _np(r0), _np(v0),
                                    None if g_r is None else _np(g_r),
                                    None if g_v is None else _np(g_v))
        return torch.from_numpy(gr), torch.from_numpy(gv), None, None, None, None


class MissDistance(torch.autograd.Function):
    """(r0, v0) [n, 3] and pairs [p, 2] -> miss distance of each pair at its TCA."""

    @staticmethod
    def forward(fctx, r0, v0, gctx, start, h, steps, pairs):
        pr = np.asarray(pairs, dtype=np.int32).reshape(-1, 2)
        _, miss, grad = gctx.miss_gradient(start, h, steps, _np(r0), _np(v0), pr)
        fctx.grad = grad
        fctx.pairs = pr
        fctx.n = r0.shape[0]
        return torch.from_numpy(miss)

    @staticmethod
    def backward(fctx, g_miss):
        w = _np(g_miss)
        gr = np.zeros((fctx.n, 3))
        gv = np.zeros((fctx.n, 3))
        for side in range(2):
            idx = fctx.pairs[:, side]
            np.add.at(gr, idx, w[:, None] * fctx.grad[:, 6 * side:6 * side + 3])
            np.add.at(gv, idx, w[:, None] * fctx.grad[:, 6 * side + 3:6 * side + 6])
        return torch.from_numpy(gr), torch.from_numpy(gv), None, None, None, None, None
