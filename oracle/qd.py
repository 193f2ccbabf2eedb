"""Linear-elastic quasi-dynamic driver (oracle; test infrastructure only).

Restates StrikeSlip_LinearElastic_qd (source/strikeSlip_linearElastic_qd.cpp:
computeMinTimeStep :262-322, initiateIntegrand :377-413, timeMonitor
:417-462, integrate :666-751, d_dt :756-798, solveMomentumBalance :874-891)
on top of the oracle SBP operator, fault and integrator.  The momentum
balance is solved with a SciPy SuperLU factorisation of the assembled
matrix, factorised once per boundary-condition set, standing in for the
reference's MUMPS Cholesky (linearElastic.cpp:251-260, :465-489).
"""
import numpy as np
import scipy.sparse.linalg as spla

from .fault import FaultQD
from .ode import AdaptiveRK
from .sbp2d import SbpOps


class QDLinearElastic:
    def __init__(self, P, keep_history=True, refine=0):
        """``refine``: steps of iterative refinement after each direct solve,
        with the residual formed in extended precision (numpy longdouble):
        the solves then reach the discrete solution to rounding, rather than
        the direct solve's forward error (about eps times the condition
        number, 1e-12 relative in the fault stress at 401 x 401 on the
        stretched grid).  The parity fixtures use it; 0 is the plain direct
        solve the reference makes."""
        self.refine = int(refine)
        self.P = P
        d, s = P["domain"], P["driver"]
        self.Ny, self.Nz = P["Ny"], P["Nz"]
        grid = d["gridSpacingType"]
        bc = P["bc"]
        self.sbp = SbpOps(d["order"], self.Ny, self.Nz, d["Ly"], d["Lz"], P["mu"], grid=grid,
                          y=P["y"] if grid != "constantGridSpacing" and self.Ny > 1 else None,
                          z=P["z"] if grid != "constantGridSpacing" and self.Nz > 1 else None,
                          compat=d["sbpCompatibilityType"],
                          bcs=(bc["R"], bc["T"], bc["L"], bc["B"]))
        self.lu = spla.splu(self.sbp.A.tocsc())
        self.fault = FaultQD(P["z"][:self.Nz], P["a"], P["b"], P["sN"], P["Dc"], P["psi"],
                             P["mu_f"], P["rho_f"], locked=P["locked"], prestress=P["prestress"],
                             f0=P["fault"]["f0"], v0=P["fault"]["v0"], vL=d["vL"],
                             state_law=s["stateLaw"], fault_type_scale=P["faultTypeScale"],
                             root_tol=P["fault"]["rootTol"], max_its=P["fault"]["maxNumIts"])
        self.vL = s["vL"]
        self.fts = P["faultTypeScale"]
        self.bcL = P["bcL0"].copy()
        self.bcRShift = P["bcRShift"].copy()
        self.bcR = np.zeros(self.Nz)
        self.bcT = np.zeros(self.Ny)
        self.bcB = np.zeros(self.Ny)
        self.u = np.zeros(self.Ny * self.Nz)
        self.sxy = np.zeros(self.Ny * self.Nz)
        self.min_dt = self._compute_min_time_step()
        self.history = [] if keep_history else None
        self.solves = 0

    def _compute_min_time_step(self):
        """computeMinTimeStep (strikeSlip_linearElastic_qd.cpp:262-322)."""
        s, d = self.P["driver"], self.P["domain"]
        if d["gridSpacingType"] == "variableGridSpacing":
            dy = self.sbp.yq.diagonal() / (self.Ny - 1)
            dz = self.sbp.zr.diagonal() / (self.Nz - 1)
        else:
            dy = np.full(self.Ny * self.Nz, d["Ly"] / (self.Ny - 1.0))
            dz = np.full(self.Ny * self.Nz, d["Lz"] / (self.Nz - 1.0))
        m = min(np.min(dy / self.P["cs"]), np.min(dz / self.P["cs"]))
        return m if s["minDeltaT"] == -1 else s["minDeltaT"]

    # ------------------------------------------------------------------
    def solve_momentum_balance(self):
        """setRHS, computeU, computeStresses (linearElastic.cpp:465-509, :711-738)."""
        rhs = self.sbp.set_rhs(self.bcL, self.bcR, self.bcT, self.bcB)
        self.u = self._refined(self.sbp.A, self.lu, rhs)
        self.solves += 1
        self.sxy = self.sbp.muxDy(self.u)
        self.rhs = rhs

    def _refined(self, A, lu, b):
        x = lu.solve(b)
        if self.refine <= 0:
            return x
        A = A.tocsr()
        ip, ix = A.indptr, A.indices
        dv = A.data.astype(np.longdouble)
        bl = b.astype(np.longdouble)
        for _ in range(self.refine):
            prod = dv * x.astype(np.longdouble)[ix]
            Ax = np.add.reduceat(prod, ip[:-1])
            Ax[ip[:-1] == ip[1:]] = 0  # empty rows
            x = x + lu.solve(np.asarray(bl - Ax, dtype=np.float64))
        return x

    def d_dt(self, t, var):
        """strikeSlip_linearElastic_qd.cpp:756-798."""
        s = self.P["driver"]
        if s["bcLType"] in ("symmFault", "rigidFault"):
            self.bcL = var["slip"] / self.fts
        if s["bcRType"] == "remoteLoading":
            self.bcR = np.full(self.Nz, self.vL * t / self.fts) + self.bcRShift
        self.fault.update_fields(var)
        self.solve_momentum_balance()
        dslip, dpsi = self.fault.d_dt(self.sxy[:self.Nz].copy())
        return {"slip": dslip, "psi": dpsi}

    def time_monitor(self, t, dt, step):
        if self.history is not None:
            f = self.fault
            self.history.append(dict(t=t, dt=dt, step=step, slip=f.slip.copy(), slipVel=f.slipVel.copy(),
                                     psi=f.psi.copy(), tauP=f.tauP.copy(), tauQSP=f.tauQSP.copy(),
                                     surfDisp=self.u[::self.Nz].copy()))
        return False

    def initiate_integrand(self):
        """initiateIntegrand (strikeSlip_linearElastic_qd.cpp:377-413)."""
        var = {"slip": self.bcL * self.fts, "psi": self.fault.psi.copy()}
        if self.P["driver"]["guessSteadyStateICs"] == 1:
            var["slip"] = self.solve_ss()
            var["psi"] = self.fault.psi.copy()
        return var

    def solve_ss(self):
        """solveSS + solveSSb (strikeSlip_linearElastic_qd.cpp:895-1006) with
        Fault::guessSS / computePsiSS (fault.cpp:619-672).  Returns the slip."""
        f = self.fault
        f.slipVel = np.full(self.Nz, self.vL)
        if not self.P["fault"]["stateVals"]:
            f.psi = f.f0 - f.b * np.log(abs(self.vL) / f.v0)
        tau = f.sN * f.a * np.arcsinh(0.5 * self.vL * np.exp(f.psi / f.a) / f.v0)
        bc = self.P["bc"]
        self.sbp.change_bc_types(bc["R"], bc["T"], "Neumann", bc["B"])
        lu = spla.splu(self.sbp.A.tocsc())
        rhs = self.sbp.set_rhs(tau, np.zeros(self.Nz), self.bcT, self.bcB)
        u = self._refined(self.sbp.A, lu, rhs)
        mn = u.min()
        if mn < 0:
            u = u + abs(mn)
        self.bcRShift = u[-self.Nz:].copy()
        self.bcR = self.bcRShift.copy()
        uL = u[:self.Nz].copy()
        self.bcL = uL.copy()
        self.u = u
        self.sbp.change_bc_types(bc["R"], bc["T"], bc["L"], bc["B"])
        return uL * self.fts

    def integrate(self, max_steps=None, replay=None, record=None, var0=None):
        """integrate (strikeSlip_linearElastic_qd.cpp:666-751).  ``var0``: a
        state from an earlier ``initiate_integrand()`` call (the initial
        guess is then not repeated, so a timing can leave it out)."""
        s = self.P["driver"]
        var = self.initiate_integrand() if var0 is None else {k: v.copy() for k, v in var0.items()}
        rk = AdaptiveRK(s["timeIntegrator"], s["maxStepCount"] if max_steps is None else max_steps,
                        s["maxTime"], s["initDeltaT"], s["timeControlType"])
        rk.set_tolerance(s["timeStepTol"])
        rk.set_time_step_bounds(self.min_dt, s["maxDeltaT"])
        rk.set_time_range(s["initTime"], s["maxTime"])
        rk.set_tolerance_type(s["normType"])
        rk.set_initial_conds(var)
        rk.set_err_inds(s["timeIntInds"], s["scale"])
        self.time_monitor(s["initTime"], s["initDeltaT"], 0)
        rk.integrate(self, replay=replay, record=record)
        self.rk = rk
        return rk
