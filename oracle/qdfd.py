"""Quasi-dynamic / fully dynamic earthquake-cycle driver (oracle; test infrastructure only).

Restates strikeSlip_linearElastic_qd_fd (source/strikeSlip_linearElastic_qd_fd.cpp):
constructor defaults :8-33, loadSettings :135-230, checkInput :232-305,
parseBCs :308-352, computeTimeStep :356-442, computePenaltyVectors :446-505,
integrate :511-581, checkSwitchRegime :586-662, initiateIntegrands :668-744,
prepare_fd2qd :747-804, prepare_qd2fd :807-888, integrate_singleQDTimeStep
:891-956, propagateWaves :1170-1239, integrate_qd :1436-1508, integrate_fd
:1511-1545, d_dt (quasi-dynamic) :1548-1597, d_dt (fully dynamic)
:1676-1757, timeMonitor :1814-1859; and OdeSolver_WaveEq::integrate
(source/odeSolver_WaveEq.cpp:147-186) with its single-argument
setInitialConds (:91-115), which starts every fully dynamic phase with
varPrev equal to var.

Quirks kept for parity:
* the switch criterion is R = max(eta_rad V / tauQS), not max V (:597-604);
* computePenaltyVectors advances its output index only inside the last
  ``if`` (:493-495), so the outgoing-characteristics damping ay lands on
  entries 0..Nz of the body vector (see ``penalty_ay``);
* checkInput compares limit_qd with trigger_fd2qd but resets it from
  trigger_qd2fd (:296-298); limit_qd is 10 vL with the constructor's vL;
* the first step-size update of each phase's fresh RK object has no error
  history (errA = [0, 0]); with PID control past step 4 the ratio is NaN and
  the 5x growth cap decides (odeSolver.cpp:846-898).
"""
import math

import numpy as np
import scipy.sparse.linalg as spla

from .fault import FaultFD
from .infile import atof, atoi, parse_lines
from .ode import AdaptiveRK
from .problem import _load_vec_file, build_qd_problem, parse_bc
from .qd import QDLinearElastic
from .sbp2d import SbpOps


def qdfd_settings(text):
    """loadSettings + constructor defaults + checkInput adjustments of
    strikeSlip_linearElastic_qd_fd (:8-33, :135-230, :232-305)."""
    s = dict(vL=1e-9, trigger_qd2fd=1e-3, trigger_fd2qd=1e-3, limit_qd=10 * 1e-9, limit_fd=1e-1,
             limit_stride_fd=-1.0, deltaT_fd=-1.0, CFL=-1.0, maxNumCycles=1000,
             minDeltaT=1e-3, maxDeltaT=1e10, initDeltaT=1e-3,
             bcR_fd="outGoingCharacteristics", bcT_fd="freeSurface", bcL_fd="symmFault",
             bcB_fd="outGoingCharacteristics")
    for var, rhs, _ in parse_lines(text):
        if var == "trigger_qd2fd": s["trigger_qd2fd"] = atof(rhs)
        elif var == "trigger_fd2qd": s["trigger_fd2qd"] = atof(rhs)
        elif var == "limit_qd": s["limit_qd"] = atof(rhs)
        elif var == "limit_fd": s["limit_fd"] = atof(rhs)
        elif var == "limit_stride_fd": s["limit_stride_fd"] = atof(rhs)
        elif var == "deltaT_fd": s["deltaT_fd"] = atof(rhs)
        elif var == "CFL": s["CFL"] = atof(rhs)
        elif var == "maxNumCycles": s["maxNumCycles"] = atoi(rhs)
        elif var == "minDeltaT": s["minDeltaT"] = atof(rhs)
        elif var == "maxDeltaT": s["maxDeltaT"] = atof(rhs)
        elif var == "initDeltaT": s["initDeltaT"] = atof(rhs)
        elif var == "momBal_bcR_fd": s["bcR_fd"] = rhs
        elif var == "momBal_bcT_fd": s["bcT_fd"] = rhs
        elif var == "momBal_bcL_fd": s["bcL_fd"] = rhs
        elif var == "momBal_bcB_fd": s["bcB_fd"] = rhs
    if s["initDeltaT"] < s["minDeltaT"] or s["initDeltaT"] < 1e-14:
        s["initDeltaT"] = s["minDeltaT"]
    if s["limit_fd"] < s["trigger_qd2fd"]:
        s["limit_fd"] = 10 * s["trigger_qd2fd"]
    if s["limit_qd"] > s["trigger_fd2qd"]:
        s["limit_qd"] = s["trigger_qd2fd"] / 10.0
    if s["limit_stride_fd"] == -1:
        s["limit_stride_fd"] = s["limit_fd"] / 10.0
    return s


def build_qdfd_problem(text, input_dir=None):
    """build_qd_problem plus the cycle settings; the quasi-dynamic phase's
    minDeltaT defaults to 1e-3 here rather than to the CFL-based minimum."""
    P = build_qd_problem(text, input_dir)
    fd = qdfd_settings(text)
    P["fd"] = fd
    P["driver"]["minDeltaT"] = fd["minDeltaT"]
    P["driver"]["maxDeltaT"] = fd["maxDeltaT"]
    P["driver"]["initDeltaT"] = fd["initDeltaT"]
    P["slip_file"] = _load_vec_file(P["domain"]["inputDir"], "slip", P["Nz"])
    return P


def penalty_ay(Ny, Nz, h11y, h11z, bcR, bcT, bcL, bcB, cs):
    """computePenaltyVectors' ay (:475-503), index quirk included: the output
    index Jj only advances while the last condition holds (iy = 0 with a
    fault-type left boundary), so rows iy >= 1 all write entry Nz."""
    N = Ny * Nz
    ay = np.zeros(N)
    Jj = 0
    for Ii in range(N):
        ay[Jj] = 0
        if Ii // Nz == Ny - 1 and bcR == "outGoingCharacteristics": ay[Jj] += 0.5 / h11y
        if Ii % Nz == 0 and bcT == "outGoingCharacteristics": ay[Jj] += 0.5 / h11z
        if (Ii + 1) % Nz == 0 and bcB == "outGoingCharacteristics": ay[Jj] += 0.5 / h11z
        if Ii // Nz == 0 and bcL in ("outGoingCharacteristics", "symmFault", "rigidFault"):
            Jj += 1
    return ay * cs


class QDFDLinearElastic(QDLinearElastic):
    def __init__(self, P, keep_history=True, refine=0):
        super().__init__(P, keep_history, refine)
        self.N = self.Ny * self.Nz
        self.fdset = P["fd"]
        d = P["domain"]
        self.min_dt = P["driver"]["minDeltaT"]
        self.rho = np.asarray(P["rho"], float)
        self.cs = np.asarray(P["cs"], float)
        grid = d["gridSpacingType"]
        self.var_grid = grid == "variableGridSpacing"
        # the fully dynamic phase's operator: all four material boundaries Neumann
        self.sbp_fd = SbpOps(d["order"], self.Ny, self.Nz, d["Ly"], d["Lz"], P["mu"], grid=grid,
                             y=P["y"] if self.var_grid and self.Ny > 1 else None,
                             z=P["z"] if self.var_grid and self.Nz > 1 else None,
                             compat=d["sbpCompatibilityType"],
                             bcs=("Neumann", "Neumann", "Neumann", "Neumann"))
        h11 = 0.5 if d["order"] == 2 else 17.0 / 48.0
        self.h11y = h11 * self.sbp.dy
        self.h11z = h11 * self.sbp.dz
        alphay = np.full(self.N, self.h11y)
        if self.var_grid:
            alphay = self.sbp.yq.diagonal() * alphay
            self.Jinv = (self.sbp.qy @ self.sbp.rz).diagonal()
        fs = self.fdset
        self.ay = penalty_ay(self.Ny, self.Nz, self.h11y, self.h11z, fs["bcR_fd"], fs["bcT_fd"], fs["bcL_fd"],
                             fs["bcB_fd"], self.cs)
        self.ffd = FaultFD(self.fault, P["rho_f"], alphay[:self.Nz], self.fts)
        self.deltaT_fd = self.compute_time_step()
        self.deltaT = -1.0
        self.currTime = P["driver"]["initTime"]
        self.stepCount = 0
        self.cycleCount = 0
        self.allowed = False
        self.inDynamic = False
        self.u0 = np.zeros(self.N)
        self.switches = []
        self.stop_at_step = None
        self.hard_stop = False
        self.fd_steps = 0
        self.qd_steps = 0
        self.on_fd_start = None  # test hook: called with (self, var, varPrev) as a wave phase starts

    # ------------------------------------------------------------------
    def compute_time_step(self):
        """computeTimeStep (:356-442)."""
        d = self.P["domain"]
        order = d["order"]
        gcfl = 0.7071
        if order == 4:
            gcfl = 0.7071 / math.sqrt(1.4498)
        if order == 6:
            gcfl = 0.7071 / math.sqrt(2.1579)
        if self.var_grid:
            dy = self.sbp.yq.diagonal() * (1.0 / (self.Ny - 1))
            dz = self.sbp.zr.diagonal() * (1.0 / (self.Nz - 1))
        else:
            dy = np.full(self.N, d["Ly"] / (self.Ny - 1.0))
            dz = np.full(self.N, d["Lz"] / (self.Nz - 1.0))
        min_ts_dy = np.min(dy / self.cs)
        min_ts_dz = np.min(dz / self.cs)
        max_deltaT = gcfl * min(abs(min_ts_dy), abs(min_ts_dz))
        cfl_deltaT = self.fdset["CFL"] * gcfl * max_deltaT
        req = self.fdset["deltaT_fd"]
        dt = max_deltaT
        if req <= 0. and cfl_deltaT <= 0.:
            dt = max_deltaT
        elif req > 0. and cfl_deltaT <= 0.:
            dt = req
        elif req <= 0. and cfl_deltaT > 0.:
            dt = cfl_deltaT
        else:
            dt = req
        return dt

    # ------------------------------------------------------------------
    def check_switch_regime(self, fault):
        """checkSwitchRegime (:586-662)."""
        R = self.fault.eta * fault.slipVel / fault.tauQSP
        maxV = float(np.max(R))
        fs = self.fdset
        must = False
        if self.inDynamic and not self.allowed and maxV > fs["limit_fd"]:
            self.allowed = True
        if not self.inDynamic and not self.allowed and maxV < fs["limit_qd"]:
            self.allowed = True
        if self.inDynamic and self.allowed and maxV < fs["trigger_fd2qd"]:
            must = True
        if not self.inDynamic and self.allowed and maxV > fs["trigger_qd2fd"]:
            must = True
        self.last_R = maxV
        return must

    def time_monitor(self, t, dt, step):
        """timeMonitor (:1814-1859) without output."""
        self.currTime = t
        self.deltaT = dt
        if self.stepCount == step and self.stepCount != 0:
            return False
        self.stepCount = step
        f = self.ffd if self.inDynamic else self.fault
        if self.history is not None:
            rk = getattr(self, "rk_current", None)
            self.history.append(dict(t=t, dt=dt, step=step, phase="fd" if self.inDynamic else "qd",
                                     new_dt=None if self.inDynamic or rk is None else rk.newDeltaT,
                                     slip=f.slip.copy(), slipVel=f.slipVel.copy(), psi=f.psi.copy(),
                                     tauP=f.tauP.copy(), tauQSP=f.tauQSP.copy(),
                                     surfDisp=self.u[::self.Nz].copy()))
        if self.inDynamic:
            self.fd_steps += 1
        else:
            self.qd_steps += 1
        stop = self.check_switch_regime(f)
        if stop:
            self.switches.append(dict(step=step, t=t, to="qd" if self.inDynamic else "fd", R=self.last_R))
        if self.stop_at_step is not None and step >= self.stop_at_step:
            self.hard_stop = True
            return True
        return stop

    # ------------------------------------------------------------------
    def initiate_integrands(self):
        """initiateIntegrands (:668-744)."""
        s = self.P["driver"]
        slip = self.bcL.copy()
        if s["bcLType"] == "symmFault":
            slip = slip * 2.0
        if self.P.get("slip_file") is not None:
            slip = self.P["slip_file"].copy()
        if s["guessSteadyStateICs"] == 1:
            slip = self.solve_ss()
        self.fault.slip = slip.copy()
        self.varQSEx = {"slip": slip, "psi": self.fault.psi.copy()}
        fq, ff = self.fault, self.ffd
        ff.psi = fq.psi.copy(); ff.slipVel = fq.slipVel.copy(); ff.slip = fq.slip.copy()
        ff.slip0 = fq.slip.copy(); ff.tauQSP = fq.tauQSP.copy(); ff.tauP = fq.tauP.copy()
        ff.tau0 = fq.strength.copy()
        self.varFD = {"psi": ff.psi.copy(), "slip": ff.slip.copy(), "u": self.u.copy()}
        self.u0 = np.zeros(self.N)

    def prepare_fd2qd(self):
        """prepare_fd2qd (:747-804)."""
        ff, fq = self.ffd, self.fault
        self.varQSEx = {"psi": ff.psi.copy(), "slip": ff.slip.copy()}
        fq.psi = ff.psi.copy(); fq.slipVel = ff.slipVel.copy(); fq.slip = ff.slip.copy()
        fq.tauP = ff.tauP.copy(); fq.tauQSP = ff.tauQSP.copy(); fq.strength = ff.strength.copy()

    def prepare_qd2fd(self, replay, record):
        """prepare_qd2fd (:807-888) including integrate_singleQDTimeStep (:891-956)."""
        uPrev = self.u.copy()
        self.inDynamic = False
        self._run_rk(1, self.deltaT_fd, (self.deltaT_fd, self.deltaT_fd),
                     (self.currTime, self.currTime + self.deltaT_fd), replay, record)
        self.inDynamic = True
        if self.hard_stop:
            return
        fq, ff = self.fault, self.ffd
        self.varFD = {"slip": fq.slip.copy(), "psi": fq.psi.copy(), "u": self.u - uPrev}
        self.u0 = uPrev
        ff.psi = fq.psi.copy(); ff.slipVel = fq.slipVel.copy(); ff.slip = fq.slip.copy()
        ff.slip0 = fq.slip.copy(); ff.strength = fq.strength.copy(); ff.tau0 = fq.strength.copy()
        ff.tauP = fq.tauP.copy(); ff.tauQSP = fq.tauQSP.copy()
        ff.tau0 = ff.tau0 + 1.0 * fq.prestress

    def _run_rk(self, max_steps, dt0, bounds, trange, replay, record):
        s = self.P["driver"]
        rk = AdaptiveRK(s["timeIntegrator"], max_steps, s["maxTime"], dt0, s["timeControlType"])
        rk.set_tolerance(s["timeStepTol"])
        rk.set_time_step_bounds(*bounds)
        rk.set_time_range(*trange)
        rk.set_initial_step_count(self.stepCount)
        rk.set_tolerance_type(s["normType"])
        rk.set_initial_conds(self.varQSEx)
        rk.set_err_inds(s["timeIntInds"], s["scale"])
        self.rk_current = rk
        rk.integrate(self, replay=replay, record=record)
        return rk

    def integrate_qd(self, replay, record):
        """integrate_qd (:1436-1508)."""
        s = self.P["driver"]
        rk = self._run_rk(s["maxStepCount"], self.deltaT_fd, (self.min_dt, s["maxDeltaT"]),
                          (self.currTime, s["maxTime"]), replay, record)
        self.varQSEx = {k: v.copy() for k, v in rk.var.items()}

    # ------------------------------------------------------------------
    def propagate_waves(self, dt, var, varPrev):
        """propagateWaves (:1170-1239)."""
        D2u = self.sbp_fd.Hinv @ (self.sbp_fd.A @ var["u"])
        if self.var_grid:
            D2u = self.Jinv * D2u
        self.ffd.d2u = D2u[:self.Nz].copy()
        c1 = dt * dt / self.rho
        c2 = dt * self.ay - 1.0
        c3 = dt * self.ay + 1.0
        return (c1 * D2u + 2. * var["u"] + c2 * varPrev["u"]) / c3

    def d_dt_fd(self, t, dt, var, varPrev):
        """Fully dynamic d_dt (:1676-1757)."""
        uNext = self.propagate_waves(dt, var, varPrev)
        psiNext, slipNext = self.ffd.d_dt(self.deltaT, var, varPrev)
        uNext[:self.Nz] = self.ffd.u
        self.u = uNext + 1.0 * self.u0
        sxy = self.sbp.muxDy(self.u)
        ff = self.ffd
        ff.tauQSP = sxy[:self.Nz] + 1.0 * self.fault.prestress
        ff.tauP = -1.0 * (self.fault.eta * ff.slipVel) + ff.tauQSP
        s = self.P["driver"]
        if s["bcLType"] in ("symmFault", "rigidFault"):
            self.bcL = ff.slip / self.fts
        if s["bcRType"] == "remoteLoading":
            self.bcR = np.full(self.Nz, self.vL * t / self.fts) + self.bcRShift
        return {"psi": psiNext, "slip": slipNext, "u": uNext}

    def integrate_fd(self):
        """integrate_fd (:1511-1545) with OdeSolver_WaveEq::integrate
        (odeSolver_WaveEq.cpp:147-186)."""
        s = self.P["driver"]
        var = {k: v.copy() for k, v in self.varFD.items()}
        varPrev = {k: v.copy() for k, v in var.items()}
        currT, finalT, dt = self.currTime, s["maxTime"], self.deltaT_fd
        stepCount = self.stepCount
        maxNumSteps = stepCount + s["maxStepCount"]
        if finalT == currT:
            return
        if self.on_fd_start is not None:
            self.on_fd_start(self, var, varPrev)
        self.time_monitor(currT, dt, stepCount)
        while stepCount < maxNumSteps and currT < finalT:
            currT = currT + dt
            if currT > finalT:
                currT = finalT
            stepCount += 1
            varNext = self.d_dt_fd(currT, dt, var, varPrev)
            varPrev, var = var, varNext
            if self.time_monitor(currT, dt, stepCount):
                break
        self.varFD = var

    # ------------------------------------------------------------------
    def integrate_cycles(self, replay=None, record=None, stop_at_step=None):
        """integrate (:511-581).  ``stop_at_step`` ends the whole run after
        that global step (a test hook, not a reference setting)."""
        s = self.P["driver"]
        fs = self.fdset
        self.stop_at_step = stop_at_step
        rp = iter(replay) if replay is not None else None
        self.initiate_integrands()
        self.u_history_start = self.u.copy()

        def phase_pair():
            self.allowed = False
            self.inDynamic = False
            self.prepare_fd2qd()
            self.integrate_qd(rp, record)
            return not self.hard_stop

        if not phase_pair():
            return
        if self.currTime >= s["maxTime"] or self.stepCount >= s["maxStepCount"]:
            return
        self.allowed = False
        self.inDynamic = True
        self.prepare_qd2fd(rp, record)
        if self.hard_stop:
            return
        self.integrate_fd()
        if self.hard_stop:
            return
        if self.currTime >= s["maxTime"] or self.stepCount >= s["maxStepCount"] or fs["maxNumCycles"] <= 1:
            return
        self.cycleCount += 1
        while (self.cycleCount < fs["maxNumCycles"] and self.stepCount <= s["maxStepCount"]
               and self.currTime <= s["maxTime"]):
            if not phase_pair():
                return
            self.allowed = False
            self.inDynamic = True
            self.prepare_qd2fd(rp, record)
            if self.hard_stop:
                return
            self.integrate_fd()
            if self.hard_stop:
                return
            self.cycleCount += 1
