"""Python view of the batched ensemble C ABI (scy_batch_*).

``Batch(paths)`` creates one quasi-dynamic driver per input file (the
reference's .in format) and runs them together: every RK attempt of every
instance is one round of shared launches (one CUDA graph launch per round),
while each instance keeps its own step control.  ``instance(i)`` is a
``QD`` view of instance i (fields, attempt logs, counters).
"""
import ctypes as C

from . import _lib as S
from . import _lib_ext as X
from .qd import QD


class _InstanceView(QD):
    """A QD over a handle that the batch owns (never destroyed here)."""

    def close(self):
        self.h = None

    __del__ = close


class Batch:
    def __init__(self, paths, solve_rtol=1e-12, solve_atol=0.0, precision="fp64", cg_its=0, graphs=True,
                 concurrent=True, solve_max_its=300, exact_jacobian=True, fd_dense=False, transform_planes=0):
        self.paths = [str(p) for p in paths]
        arr = (C.c_char_p * len(self.paths))(*[p.encode() for p in self.paths])
        o = S.SolveOpts(solve_rtol, solve_atol, solve_max_its, 0, 1, 1, S.PRECOND["auto"])
        bo = X.BatchOpts(S.PREC[precision], int(cg_its), 1 if graphs else 0, 1 if concurrent else 0,
                         1 if exact_jacobian else 0, 1 if fd_dense else 0, int(transform_planes))
        h = C.c_void_p()
        S.check(S.lib().scy_batch_create_from_in(len(self.paths), arr, C.byref(o), C.byref(bo), C.byref(h)))
        self.h = h
        n, g = C.c_int(), C.c_int()
        gof = (C.c_int * len(self.paths))()
        S.check(S.lib().scy_batch_info(h, C.byref(n), C.byref(g), gof))
        self.n, self.n_groups, self.group_of = n.value, g.value, list(gof)
        self._views = []
        for i in range(self.n):
            qh = C.c_void_p()
            S.check(S.lib().scy_batch_instance(h, i, C.byref(qh)))
            v = _InstanceView.__new__(_InstanceView)
            v._keep, v.h, v.P = [], qh, None
            ny, nz = C.c_int(), C.c_int()
            v.ode = X.OdeOpts()
            S.check(S.lib().scy_qd_get_problem(qh, C.byref(ny), C.byref(nz), C.byref(v.ode)))
            v.Ny, v.Nz, v.N = ny.value, nz.value, ny.value * nz.value
            self._views.append(v)

    def instance(self, i):
        return self._views[i]

    def run(self, nsteps):
        st = X.BatchStats()
        S.check(S.lib().scy_batch_run(self.h, int(nsteps), C.byref(st)))
        return st

    def state_size(self):
        n = C.c_long()
        S.check(S.lib().scy_batch_state_size(self.h, C.byref(n)))
        return n.value

    def set_states(self, host):
        """Every instance's integrated state from one float64 array (pinned
        or pageable), concatenated in instance order."""
        S.check(S.lib().scy_batch_set_states(self.h, S.as_dptr(host)))

    def fault_field(self, name, out=None):
        """A fault field of every instance, concatenated (Nz each)."""
        if out is None:
            import numpy as np
            out = np.empty(sum(v.Nz for v in self._views))
        S.check(S.lib().scy_batch_get_fault_field(self.h, X.FIELDS[name], S.as_dptr(out)))
        return out

    def set_graphs(self, on):
        S.check(S.lib().scy_batch_set_graphs(self.h, 1 if on else 0))

    def profile(self, on):
        S.check(S.lib().scy_batch_profile(self.h, 1 if on else 0))

    def profile_collect(self, kernel):
        """(milliseconds, launches, algorithmic bytes) of the timed launches of
        "ysolve", "residual", "matvec", "ztransform" or "zsplit"."""
        ms, nl, by = C.c_double(), C.c_longlong(), C.c_double()
        k = {"ysolve": 0, "residual": 1, "matvec": 2, "ztransform": 3, "zsplit": 4}[kernel]
        S.check(S.lib().scy_batch_profile_collect(self.h, k, C.byref(ms), C.byref(nl), C.byref(by)))
        return ms.value, nl.value, by.value

    def tuning(self, group=0):
        """The autotuner's choices for a group: the operator kernels' form
        (cross form with instances per block, or separable form with rows
        per thread), the sweep launch shape, the z-transform product's shape
        and digits, and the timings (us)."""
        kpb, var, zt, rpt, minb = C.c_int(), C.c_int(), C.c_int(), C.c_int(), C.c_int()
        us = (C.c_double * 22)()
        S.check(S.lib().scy_batch_tuning(self.h, int(group), C.byref(kpb), C.byref(var), C.byref(zt), us))
        S.check(S.lib().scy_batch_operator_form(self.h, int(group), C.byref(rpt), C.byref(minb)))
        shapes = ["2 chains x 2 warps (8 instances)", "1 chain x 4 warps (8)", "4 chains x 1 warp (8)",
                  "1 chain x 2 warps (4)", "2 chains x 1 warp (4)", "1 chain x 1 warp (2)"]
        form = "cross"
        if rpt.value:
            form = "separable, %d rows per thread, %s" % (
                rpt.value, "registers fitted to %d blocks per SM" % minb.value if minb.value > 1
                else "compiler's register count")
        return {"operator_form": form,
                "instances_per_block": kpb.value, "sweep_variant": shapes[var.value],
                "ztransform_shape": "persistent (one CTA per SM, two accumulator sets)" if zt.value & 4 else
                                    "two CTAs per SM" if zt.value & 1 else "one CTA per tile",
                "ztransform_digits": "bf16 (kind::f16)" if zt.value & 2 else "int8 (kind::i8)",
                "operator_us_by_kpb": {k: us[i] for i, k in enumerate((1, 2, 4, 8)) if us[i] > 0},
                "sweep_us_by_variant": {shapes[v]: us[4 + v] for v in range(6) if us[4 + v] > 0},
                "ztransform_us_int8_by_ctas_per_sm": {1: us[10], 2: us[11]},
                "ztransform_us_bf16_by_ctas_per_sm": {1: us[12], 2: us[13]},
                "ztransform_us_persistent": {"int8": us[20], "bf16": us[21]},
                "operator_us_separable_by_rows_per_thread": {r: us[14 + i] for i, r in enumerate((1, 2, 4))
                                                             if us[14 + i] > 0},
                "operator_us_separable_4_blocks_per_sm_by_rows_per_thread": {
                    r: us[17 + i] for i, r in enumerate((1, 2, 4)) if us[17 + i] > 0}}

    def profile_clear(self):
        S.check(S.lib().scy_batch_profile_clear(self.h))

    def close(self):
        h = getattr(self, "h", None)
        if h:
            self.h = None
            for v in getattr(self, "_views", []):
                v.h = None
            try:
                S.lib().scy_batch_destroy(h)
            except Exception:
                pass

    __del__ = close
