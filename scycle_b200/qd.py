"""Python view of the quasi-dynamic driver C ABI (StrikeSlip_LinearElastic_qd).

``QD.from_problem(P)`` takes the host arrays of a problem (grid, material,
fault fields, boundary settings) and creates the device driver; ``d_dt``,
``integrate`` and ``field`` go through libscycle_b200.so.
"""
import ctypes as C

import numpy as np

from . import _lib as S
from . import _lib_ext as X


class QD:
    @classmethod
    def from_in(cls, path, solve_rtol=1e-12, precision="fp64", solve_max_its=300, check_every=1, precond="auto",
                exact_jacobian=True):
        """Driver created by the C++ reader of the reference's .in format."""
        self = cls.__new__(cls)
        self._keep = []
        o = S.SolveOpts(solve_rtol, 0.0, solve_max_its, S.PREC[precision], 1, check_every, S.PRECOND[precond])
        h = C.c_void_p()
        S.check(S.lib().scy_qd_create_from_in(path.encode(), C.byref(o), C.byref(h)))
        self.h = h
        ny, nz = C.c_int(), C.c_int()
        self.ode = X.OdeOpts()
        S.check(S.lib().scy_qd_get_problem(h, C.byref(ny), C.byref(nz), C.byref(self.ode)))
        S.check(S.lib().scy_qd_set_jacobian(h, 1 if exact_jacobian else 0))
        self.Ny, self.Nz, self.N = ny.value, nz.value, ny.value * nz.value
        self.P = None
        return self

    def set_mode(self, mode):
        """"solve" (every d_dt solves the momentum balance) or "response"
        (fault stress from the precomputed discrete fault response)."""
        S.check(S.lib().scy_qd_set_mode(self.h, {"solve": 0, "response": 1}[mode]))

    def integrate_begin_from_in(self):
        S.check(S.lib().scy_qd_integrate_begin_from_in(self.h))

    def steady_state_info(self):
        """(effective-viscosity iterations, last relative change, CG
        iterations) of the power-law steady-state guess."""
        its, err, cg = C.c_int(), C.c_double(), C.c_long()
        S.check(S.lib().scy_qd_steady_state_info(self.h, C.byref(its), C.byref(err), C.byref(cg)))
        return its.value, err.value, cg.value

    def steady_state_trace(self):
        """Rows (correction steps, relative residual before, after, CG
        iterations, viscosity change) per viscosity iteration of the
        power-law steady-state guess."""
        n = C.c_long()
        S.check(S.lib().scy_qd_steady_state_trace(self.h, None, 0, C.byref(n)))
        out = np.zeros(max(1, n.value) * 5)
        S.check(S.lib().scy_qd_steady_state_trace(self.h, S.as_dptr(out), n.value, C.byref(n)))
        return out[: n.value * 5].reshape(n.value, 5)

    def state_size(self):
        n = C.c_long()
        S.check(S.lib().scy_qd_state_size(self.h, C.byref(n)))
        return n.value

    def set_state_vector(self, var, recompute=True):
        """The whole integrated state ([gVxy | gVxz |] psi | slip)."""
        var = np.ascontiguousarray(var, dtype=np.float64)
        assert var.size == self.state_size()
        S.check(S.lib().scy_qd_set_state(self.h, S.as_dptr(var), 1 if recompute else 0))

    def set_state(self, psi, slip, recompute=True):
        var = np.ascontiguousarray(np.concatenate([psi, slip]), dtype=np.float64)
        S.check(S.lib().scy_qd_set_state(self.h, S.as_dptr(var), 1 if recompute else 0))

    def __init__(self, P, solve_rtol=1e-12, precision="fp64", solve_max_its=300, check_every=1, precond="auto",
                 exact_jacobian=True):
        self.P = P
        d = P["domain"]
        Ny, Nz = P["Ny"], P["Nz"]
        self.Ny, self.Nz, self.N = Ny, Nz, Ny * Nz
        grid = d["gridSpacingType"]
        var = grid == "variableGridSpacing"
        bc = P["bc"]
        gdesc, keep = S.grid_desc(d["order"], Ny, Nz, d["Ly"], d["Lz"], P["mu"], grid,
                                  P["y"] if var else None, P["z"] if var else None, d["sbpCompatibilityType"],
                                  (bc["R"], bc["T"], bc["L"], bc["B"]))
        self._keep = keep
        arr = lambda v: self._hold(np.ascontiguousarray(v, dtype=np.float64))
        eta = np.sqrt(np.abs(np.asarray(P["mu_f"]) * np.asarray(P["rho_f"]))) / P["faultTypeScale"]
        f = X.FaultDesc()
        f.Nz = Nz
        f.a, f.b, f.sN, f.Dc = arr(P["a"]), arr(P["b"]), arr(P["sN"]), arr(P["Dc"])
        f.eta = arr(eta)
        f.locked = arr(P["locked"])
        f.prestress = arr(P["prestress"])
        f.f0, f.v0, f.vL = P["fault"]["f0"], P["fault"]["v0"], d["vL"]
        f.root_tol, f.max_its = P["fault"]["rootTol"], int(P["fault"]["maxNumIts"])
        f.state_law = X.LAWS[P["driver"]["stateLaw"]]
        f.exact_jacobian = 1 if exact_jacobian else 0
        q = X.QDDesc()
        q.grid = gdesc
        q.fault = f
        q.fault_type_scale = P["faultTypeScale"]
        s = P["driver"]
        q.bcL_from_slip = 1 if s["bcLType"] in ("symmFault", "rigidFault") else 0
        q.bcR_remote = 1 if s["bcRType"] == "remoteLoading" else 0
        q.vL = s["vL"]
        q.bcL0 = arr(P["bcL0"])
        q.bcRShift = arr(P["bcRShift"])
        q.solve = S.SolveOpts(solve_rtol, 0.0, solve_max_its, S.PREC[precision], 1, check_every, S.PRECOND[precond])
        h = C.c_void_p()
        S.check(S.lib().scy_qd_create(C.byref(q), C.byref(h)))
        self.h = h

    def _hold(self, a):
        self._keep.append(a)
        return S.as_dptr(a)

    def close(self):
        h = getattr(self, "h", None)
        if h:
            self.h = None
            try:
                S.lib().scy_qd_destroy(h)
            except Exception:
                pass

    __del__ = close

    def d_dt(self, t, psi, slip):
        import torch
        var = torch.from_numpy(np.concatenate([psi, slip]).astype(np.float64)).cuda()
        out = torch.empty_like(var)
        torch.cuda.synchronize()
        S.check(S.lib().scy_qd_d_dt(self.h, float(t), C.c_void_p(var.data_ptr()), C.c_void_p(out.data_ptr())))
        o = out.cpu().numpy()
        return {"psi": o[:self.Nz], "slip": o[self.Nz:]}

    def fault_d_dt(self, psi, slip, tau_body):
        """Fault_qd::d_dt alone, the body's shear stress on the fault given
        (scy_qd_fault_d_dt); linear-elastic state layout [psi | slip]."""
        import torch
        var = torch.from_numpy(np.concatenate([psi, slip]).astype(np.float64)).cuda()
        tau = torch.from_numpy(np.ascontiguousarray(tau_body, dtype=np.float64)).cuda()
        out = torch.zeros_like(var)
        torch.cuda.synchronize()
        S.check(S.lib().scy_qd_fault_d_dt(self.h, C.c_void_p(var.data_ptr()), C.c_void_p(tau.data_ptr()),
                                          C.c_void_p(out.data_ptr())))
        o = out.cpu().numpy()
        return {"psi": o[:self.Nz], "slip": o[self.Nz:]}

    def field(self, name):
        n = self.N if name in X.BODY_FIELDS else (self.Ny if name == "surfDisp" else self.Nz)
        out = np.empty(n)
        S.check(S.lib().scy_qd_get_field(self.h, X.FIELDS[name], S.as_dptr(out)))
        return out

    def ode_opts(self, min_dt, max_steps=None):
        s = self.P["driver"]
        o = X.OdeOpts()
        o.method = {"RK32": 0, "RK43": 1}[s["timeIntegrator"]]
        o.control = {"P": 0, "PID": 1}[s["timeControlType"]]
        o.norm = {"L2_absolute": 0, "L2_relative": 1}[s["normType"]]
        o.tol, o.min_dt, o.max_dt, o.init_dt = s["timeStepTol"], min_dt, s["maxDeltaT"], s["initDeltaT"]
        o.t0, o.t1 = s["initTime"], s["maxTime"]
        o.max_steps = s["maxStepCount"] if max_steps is None else max_steps
        keys = s["timeIntInds"] or []
        o.n_err = len(keys)
        for i, k in enumerate(keys):
            o.err_keys[i] = {"psi": 0, "slip": 1}[k]
            o.err_scale[i] = s["scale"][i] if s["scale"] else 1.0
        return o

    def integrate_begin(self, min_dt, max_steps=None):
        P = self.P
        var0 = np.ascontiguousarray(np.concatenate([P["psi"], P["bcL0"] * P["faultTypeScale"]]), dtype=np.float64)
        S.check(S.lib().scy_qd_integrate_begin(self.h, C.byref(self.ode_opts(min_dt, max_steps)), S.as_dptr(var0)))

    def integrate_steps(self, n):
        st = X.OdeStats()
        S.check(S.lib().scy_qd_integrate_steps(self.h, int(n), C.byref(st)))
        return st

    def force_attempts(self, attempts):
        dts = np.ascontiguousarray([a[0] for a in attempts], dtype=np.float64)
        acc = (C.c_int * len(attempts))(*[int(a[1]) for a in attempts])
        S.check(S.lib().scy_qd_force_attempts(self.h, S.as_dptr(dts), acc, len(attempts)))

    def record_attempts(self, on=True):
        S.check(S.lib().scy_qd_record_attempts(self.h, 1 if on else 0))

    def set_output(self, output_dir, stride1D=1, stride2D=0, append=False):
        """PETSc-binary output at the reference's strides (None: off)."""
        d = None if output_dir is None else str(output_dir).encode()
        S.check(S.lib().scy_qd_set_output(self.h, d, int(stride1D), int(stride2D), 1 if append else 0))

    def flush_output(self):
        S.check(S.lib().scy_qd_flush_output(self.h))

    def step_sizes(self):
        """Per step taken while recording, the size of the attempt whose
        solution was kept."""
        n = C.c_long()
        S.check(S.lib().scy_qd_get_step_sizes(self.h, None, 0, C.byref(n)))
        d = np.empty(n.value)
        S.check(S.lib().scy_qd_get_step_sizes(self.h, S.as_dptr(d), n.value, C.byref(n)))
        return d

    def attempts(self):
        n = C.c_long()
        S.check(S.lib().scy_qd_get_attempts(self.h, None, None, 0, C.byref(n)))
        dts = np.empty(n.value)
        acc = (C.c_int * max(n.value, 1))()
        S.check(S.lib().scy_qd_get_attempts(self.h, S.as_dptr(dts), acc, n.value, C.byref(n)))
        return [(float(dts[i]), bool(acc[i])) for i in range(n.value)]


def inspect_in(path, fields=("y", "z", "mu", "rho", "cs", "a", "b", "sN", "Dc", "psi", "locked", "prestress",
                             "eta", "bcL", "bcRShift")):
    """Host-only view of what the C++ loader derives from an input file."""
    L = S.lib()
    out = {}
    for nm in fields:
        n = C.c_long()
        S.check(L.scy_in_problem_field(path.encode(), nm.encode(), None, 0, C.byref(n)))
        a = np.empty(n.value)
        S.check(L.scy_in_problem_field(path.encode(), nm.encode(), S.as_dptr(a), n.value, C.byref(n)))
        out[nm] = a
    g = S.GridDesc()
    o = X.OdeOpts()
    law, guess, fts = C.c_int(), C.c_int(), C.c_double()
    S.check(L.scy_in_problem_info(path.encode(), C.byref(g), C.byref(o), C.byref(law), C.byref(guess), C.byref(fts)))
    out["grid"] = {k: getattr(g, k) for k in ("order", "Ny", "Nz", "Ly", "Lz", "grid_type", "compat", "bcR", "bcT",
                                               "bcL", "bcB")}
    out["ode"] = {k: getattr(o, k) for k in ("method", "control", "norm", "tol", "min_dt", "max_dt", "init_dt", "t0",
                                             "t1", "max_steps", "n_err")}
    out["ode"]["err_keys"] = list(o.err_keys)[:o.n_err]
    out["state_law"], out["guess_ss"], out["fault_type_scale"] = law.value, guess.value, fts.value
    return out
