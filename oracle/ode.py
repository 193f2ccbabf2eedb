"""Adaptive explicit Runge-Kutta integrators (oracle; test infrastructure only).

Restates RK32 and RK43 of source/odeSolver.cpp: constructors (:225-240,
:633-645), computeStepSize (:395-445, :846-898), computeError (:449-501,
:902-969), integrate (:505-627, :973-1175).  Variables are dicts keyed by
name; the reference iterates a ``std::map`` so keys are visited in sorted
order (e.g. "psi" before "slip").

An optional *replay* list forces the sequence of attempt step sizes and
accept decisions (used to compare two implementations over many steps
without the step-size controller amplifying round-off differences).
"""
import math

import numpy as np

RK43_TABLEAU = dict(
    c2=1. / 2., c3=83. / 250., c4=31. / 50., c5=17. / 20., c6=1.,
    b1=82889. / 524892., b3=15625. / 83664., b4=69875. / 102672., b5=-2260. / 8211., b6=1. / 4.,
    hb1=4586570599. / 29645900160., hb3=178811875. / 945068544., hb4=814220225. / 1159782912.,
    hb5=-3700637. / 11593932., hb6=61727. / 225920.,
    a21=1. / 2., a31=13861. / 62500., a32=6889. / 62500.,
    a41=-116923316275. / 2393684061468., a42=-2731218467317. / 15368042101831., a43=9408046702089. / 11113171139209.,
    a51=-451086348788. / 2902428689909., a52=-2682348792572. / 7519795681897.,
    a53=12662868775082. / 11960479115383., a54=3355817975965. / 11060851509271.,
    a61=647845179188. / 3216320057751., a62=73281519250. / 8382639484533., a63=552539513391. / 3454668386233.,
    a64=3354512671639. / 8306763924573., a65=4040. / 17871.,
)


def _ieee_div(a, b):
    if b == 0.0:
        return math.copysign(math.inf, a) if a != 0.0 else math.nan
    return a / b


class AdaptiveRK:
    """RK32 (method="RK32") or RK43 (method="RK43") with P / PID control."""

    def __init__(self, method, max_num_steps, final_t, delta_t, control_type="PID"):
        assert method in ("RK32", "RK43", "RK32_WBE", "RK43_WBE")
        # RK32_WBE / RK43_WBE (odeSolverImex.cpp:352-470, :837-): the RK32 /
        # RK43 stages and step size with a strict acceptance test, the plain
        # L2 ratio for L2_relative errors, and after each accepted step the
        # implicit (backward-Euler) update through the driver
        self.imex = method.endswith("_WBE")
        self.method = method[:4]
        self.ord = 3.0 if self.method == "RK32" else 4.0
        self.maxNumSteps = max_num_steps
        self.initT = 0.0; self.currT = 0.0; self.finalT = final_t
        self.deltaT = delta_t; self.newDeltaT = delta_t
        self.minDeltaT = 0.0; self.maxDeltaT = final_t
        self.totTol = 1e-9; self.kappa = 0.9
        self.controlType = control_type
        self.normType = "L2_absolute"
        self.stepCount = 0
        self.errA = [0.0, 0.0]  # errA[0] is the newest (boost circular_buffer push_front)
        self.numRejectedSteps = 0; self.numMinSteps = 0; self.numMaxSteps = 0
        self.errInds = []; self.scale = []
        self.var = None
        self.stage_evals = 0

    def set_tolerance(self, tol):
        self.totTol = tol

    def set_time_step_bounds(self, mn, mx):
        self.minDeltaT, self.maxDeltaT = mn, mx

    def set_time_range(self, t0, t1):
        self.initT = t0; self.currT = t0; self.finalT = t1

    def set_initial_step_count(self, step_count):
        """OdeSolver::setInitialStepCount (odeSolver.cpp:25-29): the step
        budget is counted on from the given step."""
        self.stepCount = step_count
        self.maxNumSteps = step_count + self.maxNumSteps

    def set_tolerance_type(self, t):
        assert t in ("L2_relative", "L2_absolute")
        self.normType = t

    def set_initial_conds(self, var):
        self.var = {k: np.array(v, dtype=np.float64, copy=True) for k, v in var.items()}

    def set_err_inds(self, inds, scale=None):
        self.errInds = list(inds); self.scale = list(scale or [])

    # ------------------------------------------------------------------
    def compute_step_size(self, totErr):
        if self.controlType == "P":
            ratio = self.kappa * math.pow(self.totTol / totErr, 1. / (1. + self.ord))
        elif self.controlType == "PID":
            alpha = 0.49 / self.ord; beta = 0.34 / self.ord; gamma = 0.1 / self.ord
            if self.stepCount < 4:
                ratio = self.kappa * math.pow(self.totTol / totErr, 1. / (1. + self.ord))
            else:
                # IEEE semantics as in C++: a fresh solver's errA = [0, 0]
                # gives 0 * inf = NaN, and the growth cap below then wins
                ratio = (self.kappa * math.pow(self.totTol / totErr, alpha)
                         * math.pow(self.errA[0] / self.totTol, beta)
                         * math.pow(_ieee_div(self.totTol, self.errA[1]), gamma))
        else:
            raise ValueError(self.controlType)
        dt = ratio * self.deltaT
        dt = min(self.deltaT * 5.0, dt)
        dt = min(self.maxDeltaT, dt)
        dt = max(self.minDeltaT, dt)
        if self.minDeltaT == dt:
            self.numMinSteps += 1
        elif self.maxDeltaT == dt:
            self.numMaxSteps += 1
        return dt

    def compute_error(self, lo, hi):
        """lo/hi are the embedded pair (y2/y3 for RK32, y3/y4 for RK43)."""
        tot = 0.0
        for i, key in enumerate(self.errInds):
            d = lo[key] - hi[key]
            if self.normType == "L2_absolute":
                err = math.sqrt(float(np.dot(d, d)))
                tot += err / (math.sqrt(d.size) * self.scale[i])
            else:
                if self.method == "RK32" or self.imex:
                    s = math.sqrt(float(np.dot(hi[key], hi[key])))
                    err = math.sqrt(float(np.dot(d, d)))
                    tot += err / (s * self.scale[i])
                else:
                    err = float(np.max(np.abs(d) / hi[key]))
                    tot += err / self.scale[i]
        return tot

    # ------------------------------------------------------------------
    def integrate(self, obj, replay=None, record=None):
        """Run to finalT / maxNumSteps.  ``obj`` provides d_dt(t, var) -> dvar
        and time_monitor(t, dt, stepCount) -> stop flag.

        ``replay``: optional iterator of (dt, accept) per attempt.  ``record``:
        optional list that receives (dt, accept) per attempt.
        """
        if not self.errInds:
            self.errInds = sorted(self.var.keys())
        if not self.scale:
            self.scale = [1.0] * len(self.errInds)
        if self.finalT == self.initT:
            return
        if self.deltaT == 0:
            self.deltaT = (self.finalT - self.initT) / self.maxNumSteps
        if self.maxNumSteps == 0:
            return
        keys = sorted(self.var.keys())
        ev = self._eval(obj)
        dvar = ev(self.currT, self.var)
        rp = iter(replay) if replay is not None else None
        totErr = 0.0
        while self.stepCount < self.maxNumSteps and self.currT < self.finalT:
            self.stepCount += 1
            attempt = 0
            while attempt < 100:
                attempt += 1
                if self.currT + self.deltaT > self.finalT:
                    self.deltaT = self.finalT - self.currT
                forced = next(rp, None) if rp is not None else None
                if forced is not None:
                    self.deltaT = forced[0]
                lo, hi = self._attempt(ev, keys, dvar)
                totErr = self.compute_error(lo, hi)
                if self.method == "RK32" and not self.imex:
                    acc = totErr <= self.totTol
                else:
                    acc = totErr < self.totTol
                if forced is not None:
                    acc = forced[1]
                if record is not None:
                    record.append((self.deltaT, bool(acc)))
                if acc:
                    break
                newdt = self.compute_step_size(totErr)
                if forced is None:
                    self.deltaT = newdt
                if self.minDeltaT == self.deltaT:
                    break
                self.numRejectedSteps += 1
            # accept the higher-order solution (odeSolver.cpp:599-603 / :1148-1152)
            self.currT = self.currT + self.deltaT
            self.var = {k: hi[k].copy() for k in keys}
            if self.imex:
                obj.imex_before(self.currT, self.deltaT)
            dvar = ev(self.currT, self.var)
            if self.imex:
                obj.imex_after(self.currT, self.deltaT, dvar)
            if totErr != 0.0:
                self.newDeltaT = self.compute_step_size(totErr)
            self.errA = [totErr, self.errA[0]]
            stop = obj.time_monitor(self.currT, self.deltaT, self.stepCount)
            self.deltaT = self.newDeltaT
            if stop:
                break

    def _eval(self, obj):
        def ev(t, var):
            self.stage_evals += 1
            return obj.d_dt(t, var)
        return ev

    def _attempt(self, ev, keys, f1):
        dt = self.deltaT
        var = self.var
        if self.method == "RK32":
            # odeSolver.cpp:567-592
            k1 = {k: var[k] + 0.5 * dt * f1[k] for k in keys}
            fa = ev(self.currT + 0.5 * dt, k1)
            k2 = {k: (var[k] + (-dt) * f1[k]) + 2 * dt * fa[k] for k in keys}
            fb = ev(self.currT + dt, k2)
            y2 = {k: (var[k] + 0.5 * dt * f1[k]) + 0.5 * dt * fb[k] for k in keys}
            y3 = {k: ((var[k] + dt / 6.0 * f1[k]) + 2 * dt / 3.0 * fa[k]) + dt / 6.0 * fb[k] for k in keys}
            return y2, y3
        T = RK43_TABLEAU
        t = self.currT
        k2 = {k: var[k] + T["a21"] * dt * f1[k] for k in keys}
        f2 = ev(t + T["c2"] * dt, k2)
        k3 = {k: (var[k] + T["a31"] * dt * f1[k]) + T["a32"] * dt * f2[k] for k in keys}
        f3 = ev(t + T["c3"] * dt, k3)
        k4 = {k: ((var[k] + T["a41"] * dt * f1[k]) + T["a42"] * dt * f2[k]) + T["a43"] * dt * f3[k] for k in keys}
        f4 = ev(t + T["c4"] * dt, k4)
        k5 = {k: (((var[k] + T["a51"] * dt * f1[k]) + T["a52"] * dt * f2[k]) + T["a53"] * dt * f3[k])
              + T["a54"] * dt * f4[k] for k in keys}
        f5 = ev(t + T["c5"] * dt, k5)
        k6 = {k: ((((var[k] + T["a61"] * dt * f1[k]) + T["a62"] * dt * f2[k]) + T["a63"] * dt * f3[k])
                  + T["a64"] * dt * f4[k]) + T["a65"] * dt * f5[k] for k in keys}
        f6 = ev(t + T["c6"] * dt, k6)
        y3 = {k: ((((var[k] + T["hb1"] * dt * f1[k]) + T["hb3"] * dt * f3[k]) + T["hb4"] * dt * f4[k])
                  + T["hb5"] * dt * f5[k]) + T["hb6"] * dt * f6[k] for k in keys}
        y4 = {k: ((((var[k] + T["b1"] * dt * f1[k]) + T["b3"] * dt * f3[k]) + T["b4"] * dt * f4[k])
                  + T["b5"] * dt * f5[k]) + T["b6"] * dt * f6[k] for k in keys}
        return y3, y4
