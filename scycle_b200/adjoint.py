"""Python view of the discrete adjoint (scy_adj_*) and its torch binding.

``Adjoint(qd)`` takes a begun RK32 linear-elastic driver (its state is the
initial state of every forward run), the accepted step sizes of a run, and
targets for the surface displacement and slip velocity of every accepted
state; ``gradient()`` returns the misfit and its gradient with respect to the
fault's a, b and Dc at every fault node.  ``knot_matrix`` builds the
piecewise-linear depth interpolation of the reference's ``*Vals / *Depths``
profiles (setVec, source/genFuncs.cpp:574-617) so that gradients can be taken
with respect to knot values; ``MisfitFunction`` is a ``torch.autograd.Function``
over (a, b, Dc).
"""
import ctypes as C

import numpy as np

from . import _lib as S


def _declare(L):
    if getattr(L, "_adj_declared", False):
        return
    vp, dp = C.c_void_p, C.POINTER(C.c_double)
    L.scy_adj_create.argtypes = [vp, C.c_int, C.POINTER(vp)]
    L.scy_adj_destroy.argtypes = [vp]
    L.scy_adj_set_steps.argtypes = [vp, dp, C.c_long]
    L.scy_adj_set_targets.argtypes = [vp, dp, dp, C.c_double, C.c_double]
    L.scy_adj_set_fault_params.argtypes = [vp, dp, dp, dp]
    L.scy_adj_forward.argtypes = [vp, dp]
    L.scy_adj_observations.argtypes = [vp, dp, dp]
    L.scy_adj_gradient.argtypes = [vp, dp, dp, dp, dp]
    L._adj_declared = True


def _arr(x):
    return None if x is None else np.ascontiguousarray(x, dtype=np.float64)


class Adjoint:
    def __init__(self, qd, checkpoint_every=50):
        L = S.lib()
        _declare(L)
        self.qd = qd  # keeps the driver alive
        self.Ny, self.Nz = qd.Ny, qd.Nz
        h = C.c_void_p()
        S.check(L.scy_adj_create(qd.h, int(checkpoint_every), C.byref(h)))
        self.h = h
        self.n = 0

    def set_steps(self, dts):
        d = _arr(dts)
        S.check(S.lib().scy_adj_set_steps(self.h, S.as_dptr(d), d.size))
        self.n = d.size

    def set_targets(self, surf, vel, w_surf=1.0, w_vel=1.0):
        s, v = _arr(surf), _arr(vel)
        assert s.size == self.n * self.Ny and v.size == self.n * self.Nz
        S.check(S.lib().scy_adj_set_targets(self.h, S.as_dptr(s), S.as_dptr(v), float(w_surf), float(w_vel)))

    def set_params(self, a=None, b=None, Dc=None):
        a, b, Dc = _arr(a), _arr(b), _arr(Dc)
        S.check(S.lib().scy_adj_set_fault_params(self.h, S.as_dptr(a), S.as_dptr(b), S.as_dptr(Dc)))

    def forward(self):
        J = C.c_double()
        S.check(S.lib().scy_adj_forward(self.h, C.byref(J)))
        return J.value

    def observations(self):
        s = np.empty((self.n, self.Ny))
        v = np.empty((self.n, self.Nz))
        S.check(S.lib().scy_adj_observations(self.h, S.as_dptr(s), S.as_dptr(v)))
        return s, v

    def gradient(self):
        J = C.c_double()
        ga, gb, gd = np.empty(self.Nz), np.empty(self.Nz), np.empty(self.Nz)
        S.check(S.lib().scy_adj_gradient(self.h, C.byref(J), S.as_dptr(ga), S.as_dptr(gb), S.as_dptr(gd)))
        return J.value, ga, gb, gd

    def close(self):
        h = getattr(self, "h", None)
        if h:
            self.h = None
            try:
                S.lib().scy_adj_destroy(h)
            except Exception:
                pass

    __del__ = close


def knot_matrix(z, depths):
    """P (len(z) x len(depths)): values at z = P @ values at the knots,
    linear between knots and constant beyond the ends."""
    z, d = np.asarray(z, dtype=np.float64), np.asarray(depths, dtype=np.float64)
    P = np.zeros((z.size, d.size))
    for k in range(d.size):
        e = np.zeros(d.size)
        e[k] = 1.0
        P[:, k] = np.interp(z, d, e)
    return P


def misfit_function():
    """A torch.autograd.Function: J = MisfitFunction.apply(a, b, Dc, adjoint)
    with a, b, Dc torch tensors of length Nz (float64, any device)."""
    import torch

    class MisfitFunction(torch.autograd.Function):
        @staticmethod
        def forward(ctx, a, b, Dc, adj):
            adj.set_params(a.detach().cpu().numpy(), b.detach().cpu().numpy(), Dc.detach().cpu().numpy())
            J, ga, gb, gd = adj.gradient()
            ctx.save_for_backward(*[torch.as_tensor(g, dtype=a.dtype, device=a.device) for g in (ga, gb, gd)])
            return torch.as_tensor(J, dtype=a.dtype, device=a.device)

        @staticmethod
        def backward(ctx, gJ):
            ga, gb, gd = ctx.saved_tensors
            return gJ * ga, gJ * gb, gJ * gd, None

    return MisfitFunction
