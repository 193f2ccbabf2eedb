"""Python view of the SbpOps / elliptic-solver C ABI.

Mirrors the reference SbpOps interface (source/sbpOps.hpp:42-104) for tests
and drivers: device memory comes from torch CUDA tensors; every call goes
through libscycle_b200.so.  There is no CPU fallback: without the library or
a GPU the calls raise.
"""
import ctypes as C

import numpy as np

from . import _lib as S


def _require_torch_cuda():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("scycle_b200 needs a CUDA device")
    return torch


class SbpOps:
    def __init__(self, order, Ny, Nz, Ly, Lz, mu, grid="constantGridSpacing", y=None, z=None,
                 compat="fullyCompatible", bcs=("Dirichlet", "Neumann", "Dirichlet", "Neumann")):
        self.torch = _require_torch_cuda()
        self.Ny, self.Nz, self.N = Ny, Nz, Ny * Nz
        desc, self._keep = S.grid_desc(order, Ny, Nz, Ly, Lz, mu, grid, y, z, compat, bcs)
        h = C.c_void_p()
        S.check(S.lib().scy_sbp_create(C.byref(desc), C.byref(h)))
        self.h = h
        self.bcs = bcs

    def close(self):
        h = getattr(self, "h", None)
        if h:
            self.h = None
            try:
                S.lib().scy_sbp_destroy(h)
            except Exception:
                pass

    __del__ = close

    def _dev(self, a, n=None):
        t = self.torch
        if isinstance(a, np.ndarray):
            return t.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()
        assert a.dtype == t.float64 and a.is_cuda and a.is_contiguous()
        return a

    def sync(self):
        S.check(S.lib().scy_sbp_synchronize(self.h))

    def apply(self, op, x):
        t = self.torch
        xd = self._dev(x)
        out = t.empty_like(xd)
        t.cuda.synchronize()
        S.check(S.lib().scy_sbp_apply(self.h, S.OPS[op], C.c_void_p(xd.data_ptr()), C.c_void_p(out.data_ptr())))
        self.sync()
        return out

    def set_rhs(self, bcL, bcR, bcT, bcB):
        t = self.torch
        args = [self._dev(v) for v in (bcL, bcR, bcT, bcB)]
        out = t.empty(self.N, dtype=t.float64, device="cuda")
        t.cuda.synchronize()
        S.check(S.lib().scy_sbp_set_rhs(self.h, *[C.c_void_p(a.data_ptr()) for a in args], C.c_void_p(out.data_ptr())))
        self.sync()
        return out

    def solve(self, rhs, u0=None, rtol=1e-12, atol=0.0, max_its=200, precision="fp64", check_every=1,
              precond="auto"):
        t = self.torch
        b = self._dev(rhs)
        u = t.zeros(self.N, dtype=t.float64, device="cuda") if u0 is None else self._dev(u0).clone()
        o = S.SolveOpts(rtol, atol, max_its, S.PREC[precision], 0 if u0 is None else 1, check_every,
                        S.PRECOND[precond], 1)
        st = S.SolveStats()
        t.cuda.synchronize()
        S.check(S.lib().scy_sbp_solve(self.h, C.c_void_p(b.data_ptr()), C.c_void_p(u.data_ptr()), C.byref(o),
                                      C.byref(st)))
        self.sync()
        return u, st

    def change_bc_types(self, R, T, L, B):
        S.check(S.lib().scy_sbp_change_bc_types(self.h, S.BC[R], S.BC[T], S.BC[L], S.BC[B]))

    def n_levels(self):
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        S.check(S.lib().scy_sbp_info(self.h, C.byref(a), C.byref(b), C.byref(c)))
        return c.value
