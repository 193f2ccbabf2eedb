"""Python view of the quasi-dynamic / fully dynamic cycle driver C ABI
(strikeSlip_linearElastic_qd_fd).

``Cycle.from_in(path)`` reads the reference's input format through the C++
loader; ``Cycle(P)`` takes the host arrays of a problem built by the oracle's
problem reader (tests) and creates the same driver.  ``run(n)`` advances the
global step count by at most n steps; ``field``, ``switches`` and the attempt
replay hooks mirror the quasi-dynamic driver's.
"""
import ctypes as C

import numpy as np

from . import _lib as S
from . import _lib_ext as X
from .qd import QD

FD_SIDE = {"freeSurface": 0, "outGoingCharacteristics": 1}


class Cycle:
    @classmethod
    def from_in(cls, path, solve_rtol=1e-12, precision="fp64", solve_max_its=300, check_every=1, precond="auto",
                exact_jacobian=True):
        self = cls.__new__(cls)
        self._keep = []
        o = S.SolveOpts(solve_rtol, 0.0, solve_max_its, S.PREC[precision], 1, check_every, S.PRECOND[precond])
        h = C.c_void_p()
        S.check(S.lib().scy_cycle_create_from_in(path.encode(), C.byref(o), C.byref(h)))
        self.h = h
        ny, nz, dt = C.c_int(), C.c_int(), C.c_double()
        self.ode = X.OdeOpts()
        S.check(S.lib().scy_cycle_get_problem(h, C.byref(ny), C.byref(nz), C.byref(dt), C.byref(self.ode)))
        S.check(S.lib().scy_cycle_set_jacobian(h, 1 if exact_jacobian else 0))
        self.Ny, self.Nz, self.N, self.dt_fd = ny.value, nz.value, ny.value * nz.value, dt.value
        self.P = None
        return self

    def __init__(self, P, solve_rtol=1e-12, precision="fp64", solve_max_its=300, check_every=1, precond="auto",
                 exact_jacobian=True, ay_index_quirk=True):
        # the quasi-dynamic descriptor is built exactly as for the QD driver
        qd = QD.__new__(QD)
        qd._keep = []
        self._keep = qd._keep
        self.P = P
        desc = _qd_desc(qd, P, solve_rtol, precision, solve_max_its, check_every, precond, exact_jacobian)
        fs = P["fd"]
        arr = lambda v: qd._hold(np.ascontiguousarray(v, dtype=np.float64))
        cd = X.CycleDesc()
        cd.rho, cd.cs, cd.rho_fault = arr(P["rho"]), arr(P["cs"]), arr(P["rho_f"])
        cd.fd_bcR, cd.fd_bcT, cd.fd_bcB = FD_SIDE[fs["bcR_fd"]], FD_SIDE[fs["bcT_fd"]], FD_SIDE[fs["bcB_fd"]]
        cd.deltaT_fd, cd.CFL = fs["deltaT_fd"], fs["CFL"]
        cd.trigger_qd2fd, cd.trigger_fd2qd = fs["trigger_qd2fd"], fs["trigger_fd2qd"]
        cd.limit_qd, cd.limit_fd = fs["limit_qd"], fs["limit_fd"]
        cd.max_num_cycles = int(fs["maxNumCycles"])
        cd.ay_index_quirk = 1 if ay_index_quirk else 0
        h = C.c_void_p()
        S.check(S.lib().scy_cycle_create(C.byref(desc), C.byref(cd), C.byref(h)))
        self.h = h
        self.Ny, self.Nz, self.N = P["Ny"], P["Nz"], P["Ny"] * P["Nz"]
        dt = C.c_double()
        S.check(S.lib().scy_cycle_get_problem(h, None, None, C.byref(dt), None))
        self.dt_fd = dt.value
        self.ode = qd_ode_opts(P)

    def close(self):
        h = getattr(self, "h", None)
        if h:
            self.h = None
            try:
                S.lib().scy_cycle_destroy(h)
            except Exception:
                pass

    __del__ = close

    def begin(self, psi, slip):
        var0 = np.ascontiguousarray(np.concatenate([psi, slip]), dtype=np.float64)
        S.check(S.lib().scy_cycle_begin(self.h, C.byref(self.ode), S.as_dptr(var0)))

    def begin_from_in(self):
        S.check(S.lib().scy_cycle_begin_from_in(self.h))

    def run(self, n):
        st = X.CycleStats()
        S.check(S.lib().scy_cycle_run(self.h, int(n), C.byref(st)))
        return st

    def field(self, name):
        n = {"u": self.N, "sxy": self.N, "surfDisp": self.Ny}.get(name, self.Nz)
        out = np.empty(n)
        S.check(S.lib().scy_cycle_get_field(self.h, X.FIELDS[name], S.as_dptr(out)))
        return out

    def switches(self):
        n = C.c_long()
        S.check(S.lib().scy_cycle_get_switches(self.h, None, None, None, 0, C.byref(n)))
        m = n.value
        steps = (C.c_long * max(m, 1))()
        times = np.empty(max(m, 1))
        to_fd = (C.c_int * max(m, 1))()
        S.check(S.lib().scy_cycle_get_switches(self.h, steps, S.as_dptr(times), to_fd, m, C.byref(n)))
        return [dict(step=int(steps[i]), t=float(times[i]), to="fd" if to_fd[i] else "qd") for i in range(m)]

    def set_fd_state(self, t, step, allowed, var, var_prev, u0, slip0, tau0, slipVel):
        """Restart at the start of a fully dynamic step; var / var_prev are
        dicts with psi, slip (Nz) and u (Ny*Nz)."""
        a = lambda v: np.ascontiguousarray(v, dtype=np.float64)
        arrs = [a(var["psi"]), a(var["slip"]), a(var["u"]), a(var_prev["psi"]), a(var_prev["slip"]),
                a(var_prev["u"]), a(u0), a(slip0), a(tau0), a(slipVel)]
        S.check(S.lib().scy_cycle_set_fd_state(self.h, float(t), int(step), 1 if allowed else 0,
                                               *[S.as_dptr(x) for x in arrs]))

    def time_kernels(self, reps=50):
        """(wave launch us, fault launch us, fused step us) on the current wave state."""
        w, f, t = C.c_double(), C.c_double(), C.c_double()
        S.check(S.lib().scy_cycle_time_kernels(self.h, int(reps), C.byref(w), C.byref(f), C.byref(t)))
        return w.value, f.value, t.value

    def set_fd_fused(self, fused=True):
        S.check(S.lib().scy_cycle_set_fd_fused(self.h, 1 if fused else 0))

    def set_mode(self, mode):
        S.check(S.lib().scy_cycle_set_mode(self.h, {"solve": 0, "response": 1}[mode]))

    def set_fd_batch(self, k):
        S.check(S.lib().scy_cycle_set_fd_batch(self.h, int(k)))

    def force_attempts(self, attempts):
        dts = np.ascontiguousarray([a[0] for a in attempts], dtype=np.float64)
        acc = (C.c_int * max(len(attempts), 1))(*[int(a[1]) for a in attempts])
        S.check(S.lib().scy_cycle_force_attempts(self.h, S.as_dptr(dts), acc, len(attempts)))

    def record_attempts(self, on=True):
        S.check(S.lib().scy_cycle_record_attempts(self.h, 1 if on else 0))

    def attempts(self):
        n = C.c_long()
        S.check(S.lib().scy_cycle_get_attempts(self.h, None, None, 0, C.byref(n)))
        dts = np.empty(max(n.value, 1))
        acc = (C.c_int * max(n.value, 1))()
        S.check(S.lib().scy_cycle_get_attempts(self.h, S.as_dptr(dts), acc, n.value, C.byref(n)))
        return [(float(dts[i]), bool(acc[i])) for i in range(n.value)]


def _qd_desc(qd, P, solve_rtol, precision, solve_max_its, check_every, precond, exact_jacobian):
    """The scy_qd_desc QD.__init__ builds, without creating a driver."""
    d = P["domain"]
    Ny, Nz = P["Ny"], P["Nz"]
    grid = d["gridSpacingType"]
    var = grid == "variableGridSpacing"
    bc = P["bc"]
    gdesc, keep = S.grid_desc(d["order"], Ny, Nz, d["Ly"], d["Lz"], P["mu"], grid,
                              P["y"] if var else None, P["z"] if var else None, d["sbpCompatibilityType"],
                              (bc["R"], bc["T"], bc["L"], bc["B"]))
    qd._keep.extend(keep)
    arr = lambda v: qd._hold(np.ascontiguousarray(v, dtype=np.float64))
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
    return q


def qd_ode_opts(P, max_steps=None):
    s = P["driver"]
    o = X.OdeOpts()
    o.method = {"RK32": 0, "RK43": 1}[s["timeIntegrator"]]
    o.control = {"P": 0, "PID": 1}[s["timeControlType"]]
    o.norm = {"L2_absolute": 0, "L2_relative": 1}[s["normType"]]
    o.tol, o.min_dt, o.max_dt, o.init_dt = s["timeStepTol"], s["minDeltaT"], s["maxDeltaT"], s["initDeltaT"]
    o.t0, o.t1 = s["initTime"], s["maxTime"]
    o.max_steps = s["maxStepCount"] if max_steps is None else max_steps
    keys = s["timeIntInds"] or []
    o.n_err = len(keys)
    for i, k in enumerate(keys):
        o.err_keys[i] = {"psi": 0, "slip": 1}[k]
        o.err_scale[i] = s["scale"][i] if s["scale"] else 1.0
    return o


def inspect_cycle_in(path):
    """Host-only: the cycle settings, wave-equation step and penalty vector the
    C++ loader derives from an input file."""
    L = S.lib()
    cd = X.CycleDesc()
    dt = C.c_double()
    n = C.c_long()
    S.check(L.scy_in_cycle_info(path.encode(), C.byref(cd), C.byref(dt), None, 0, C.byref(n)))
    ay = np.empty(n.value)
    S.check(L.scy_in_cycle_info(path.encode(), None, None, S.as_dptr(ay), n.value, C.byref(n)))
    out = {k: getattr(cd, k) for k in ("fd_bcR", "fd_bcT", "fd_bcB", "deltaT_fd", "CFL", "trigger_qd2fd",
                                        "trigger_fd2qd", "limit_qd", "limit_fd", "max_num_cycles", "ay_index_quirk")}
    out["dt_fd"] = dt.value
    out["ay"] = ay
    return out
