"""Power-law viscoelastic quasi-dynamic driver (oracle; test infrastructure only).

Restates PowerLaw (source/powerLaw.cpp: constructor :752-796, loadSettings
:851-915, setMaterialParameters :1010-1058, loadFieldsFromFiles :1061-1095,
setUpSBPContext :1098-1125, initializeMomBalMats :1239-1318, initiateIntegrand
:1517-1536, updateFields :1539-1554, computeViscStrainSourceTerms :1651-1671,
computeViscosity :1674-1704, computeViscStrainRates :1707-1743,
computeViscousStrainRateSAT :1746-1799, computeTotalStrains :1802-1821,
computeStresses / computeSDev :1824-1887), DislocationCreep
(:224-474) and the StrikeSlip_PowerLaw_qd driver
(source/strikeSlip_powerLaw_qd.cpp: constructor :8-70, loadSettings :118-198,
checkInput :200-256, initiateIntegrand :305-350, integrate :561-631, d_dt
:633-690, solveMomentumBalance :787-823) on the oracle SBP operator, fault and
integrator.  The integrated variables are, in the std::map's key order,
gVxy, gVxz (viscous strains, Ny*Nz each), psi and slip (Nz each).

The steady-state initial guess of guessSteadyStateICs = 1 (initiateIntegrand
:320-324 -> solveSS :922-955, guessTauSS :888-918, solveSSViscoelasticProblem
:1018-1107, setSSBCs :1295-1342; PowerLaw::guessSteadyStateEffVisc
:1999-2037, initializeSSMatrices / setSSRHS :2040-2096, updateSSa / updateSSb
:2099-2195; DislocationCreep::guessInvEffVisc :399-433) is restated in
PowerLawQD.solve_ss.

Not restated: diffusion creep, pseudoplasticity, linear Maxwell viscosity,
thermal / hydraulic / grain-size coupling, and the repeated steady-state
cycles of integrateSS (:827-885, a separate driver mode).
"""
import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from .infile import atof, atoi, load_vector_double, load_vector_string, parse_lines, set_vec
from .ode import AdaptiveRK
from .problem import _load_vec_file, build_qd_problem, driver_settings
from .fault import compute_vel_qd
from .qd import QDLinearElastic
from .sbp2d import SbpOps


def pl_settings(text):
    """PowerLaw::loadSettings + DislocationCreep::loadSettings with the
    constructor defaults (powerLaw.cpp:752-760, :260-305, :851-915)."""
    m = dict(wDislCreep="yes", wDiffCreep="no", wPlasticity="no", wLinearMaxwell="no", maxEffVisc=1e30,
             muVals=[], muDepths=[], rhoVals=[], rhoDepths=[], TVals=[], TDepths=[],
             disl_AVals=[], disl_ADepths=[], disl_BVals=[], disl_BDepths=[], disl_nVals=[], disl_nDepths=[])
    vec_keys = [k for k in m if isinstance(m[k], list)]
    for var, rhs, full in parse_lines(text):
        if var in vec_keys:
            m[var] = m[var] + load_vector_double(full)
        elif var in ("wDislCreep", "wDiffCreep", "wPlasticity", "wLinearMaxwell"):
            m[var] = rhs
        elif var == "maxEffVisc":
            m["maxEffVisc"] = atof(rhs)
    return m


def build_pl_problem(text, input_dir=None):
    """The quasi-dynamic problem with the power-law material: mu, rho, T and
    the creep parameters interpolated against z (setVec(..., *_z, ...)), and
    the driver's minDeltaT default of 1e-3."""
    P = build_qd_problem(text, input_dir)
    d = P["domain"]
    m = pl_settings(text)
    z = P["z"]
    P["pl"] = m
    P["mu"] = set_vec(z, m["muVals"], m["muDepths"])
    P["rho"] = set_vec(z, m["rhoVals"], m["rhoDepths"])
    N = P["N"]
    for nm, key in (("mu", "mu"), ("rho", "rho")):
        v = _load_vec_file(d["inputDir"], nm, N)
        if v is not None:
            P[key] = v
    P["cs"] = np.sqrt(np.abs(P["mu"] / P["rho"]))
    P["T"] = set_vec(z, m["TVals"], m["TDepths"])
    v = _load_vec_file(d["inputDir"], "T", N)
    if v is not None:
        P["T"] = v
    P["A"] = set_vec(z, m["disl_AVals"], m["disl_ADepths"])
    P["B"] = set_vec(z, m["disl_BVals"], m["disl_BDepths"])
    P["n"] = set_vec(z, m["disl_nVals"], m["disl_nDepths"])
    P["gVxy0"] = _load_vec_file(d["inputDir"], "GVxy", N)
    P["gVxz0"] = _load_vec_file(d["inputDir"], "GVxz", N)
    if P["gVxy0"] is None:
        P["gVxy0"] = np.zeros(N)
    if P["gVxz0"] is None:
        P["gVxz0"] = np.zeros(N)
    # StrikeSlip_PowerLaw_qd's constructor default minDeltaT is 1e-3
    # (strikeSlip_powerLaw_qd.cpp:22); the file may override it
    s = P["driver"]
    if s["minDeltaT"] == -1.0:
        s["minDeltaT"] = 1e-3
    if s["initDeltaT"] < s["minDeltaT"] or s["initDeltaT"] < 1e-14:
        s["initDeltaT"] = s["minDeltaT"]
    P["slip_file"] = _load_vec_file(d["inputDir"], "slip", P["Nz"])
    # steady-state iteration settings (strikeSlip_powerLaw_qd.cpp:27-29,
    # :157-163) and its optional input files
    ss = dict(fss_EffVisc=0.2, gss_t=1e-10, atolSS_effVisc=1e-3, maxSSIts_effVisc=50)
    for var, rhs, full in parse_lines(text):
        if var in ("fss_EffVisc", "gss_t", "atolSS_effVisc"):
            ss[var] = atof(rhs)
        elif var == "maxSSIts_effVisc":
            ss[var] = atoi(rhs)
    ss["effVisc_file"] = _load_vec_file(d["inputDir"], "effVisc", N)
    ss["tauSS_file"] = _load_vec_file(d["inputDir"], "tauSS", P["Nz"])
    P["ss"] = ss
    return P


class PowerLawQD(QDLinearElastic):
    """StrikeSlip_PowerLaw_qd with dislocation creep."""

    def __init__(self, P, keep_history=True, refine=0):
        super().__init__(P, keep_history, refine)
        self.N = self.Ny * self.Nz
        self.min_dt = P["driver"]["minDeltaT"]
        self.mu = np.asarray(P["mu"], float)
        self.A, self.Bq, self.nexp, self.T = P["A"], P["B"], P["n"], P["T"]
        self.cap = P["pl"]["maxEffVisc"]
        self.gVxy = P["gVxy0"].copy()
        self.gVxz = P["gVxz0"].copy()
        self.sdev = np.zeros(self.N)
        self.effVisc = np.zeros(self.N)
        self._momentum_mats()

    def _momentum_mats(self):
        """initializeMomBalMats (powerLaw.cpp:1239-1318): B and C."""
        s = self.sbp
        mu = sp.diags(self.mu)
        if self.sbp.grid == "variableGridSpacing":
            yqxzrxH = (s.yq @ s.zr @ s.H).tocsr()
            yqxHy = (s.yq @ s.Hy_Iz).tocsr()
            zrxHz = (s.zr @ s.Iy_Hz).tocsr()
        else:
            yqxHy = (s.H @ s.Iy_Hzinv).tocsr()
            zrxHz = (s.H @ s.Hyinv_Iz).tocsr()
            yqxzrxH = s.H.copy()
        B = (yqxzrxH @ s.Dy_Iz @ mu).tocsr()
        if s.bcL == "Neumann":
            B = B + zrxHz @ mu @ s.E0y_Iz
        if s.bcR == "Neumann":
            B = B - zrxHz @ mu @ s.ENy_Iz
        C = (yqxzrxH @ s.Iy_Dz @ mu).tocsr()
        if s.bcT == "Neumann":
            C = C + yqxHy @ mu @ s.Iy_E0z
        if s.bcB == "Neumann":
            C = C - yqxHy @ mu @ s.Iy_ENz
        self.Bm, self.Cm = B.tocsr(), C.tocsr()

    def strain_rate_sat(self, u):
        """computeViscousStrainRateSAT (powerLaw.cpp:1746-1799)."""
        s = self.sbp
        out = np.zeros(self.N)
        if s.bcL == "Dirichlet":
            out = out + s.Hyinv_Iz @ (s.E0y_Iz @ u)
            out = out - s.Hyinv_Iz @ (s.e0y_Iz @ self.bcL)
        if s.bcR == "Dirichlet":
            out = out - s.Hyinv_Iz @ (s.ENy_Iz @ u)
            out = out + s.Hyinv_Iz @ (s.eNy_Iz @ self.bcR)
        if s.grid == "variableGridSpacing":
            out = s.qy @ out
        return out

    def d_dt(self, t, var):
        """StrikeSlip_PowerLaw_qd::d_dt + solveMomentumBalance (:633-690, :787-823)."""
        st = self.P["driver"]
        if st["bcLType"] in ("symmFault", "rigidFault"):
            self.bcL = var["slip"] / self.fts
        if st["bcRType"] == "remoteLoading":
            self.bcR = np.full(self.Nz, self.vL * t / self.fts) + self.bcRShift
        self.gVxy = var["gVxy"].copy()
        self.gVxz = var["gVxz"].copy()
        self.fault.update_fields(var)
        source = self.Bm @ self.gVxy + self.Cm @ self.gVxz
        rhs = self.sbp.set_rhs(self.bcL, self.bcR, self.bcT, self.bcB) + 1.0 * source
        self.u = self.lu.solve(rhs)
        self.solves += 1
        gTxy = self.sbp.Dy_Iz @ self.u
        gTxz = self.sbp.Iy_Dz @ self.u
        sxy = (gTxy - self.gVxy) * self.mu
        sxz = (gTxz - self.gVxz) * self.mu
        self.sxy, self.sxz = sxy, sxz
        self.sdev = np.sqrt(np.abs(sxy * sxy + sxz * sxz))
        inv = 1e3 * self.A * np.power(self.sdev, self.nexp - 1.0) * np.exp(-self.Bq / self.T)
        self.effVisc = 1.0 / (np.full(self.N, 1.0 / self.cap) + 1.0 * inv)
        SAT = self.strain_rate_sat(self.u)
        dgxy = (self.mu * SAT + 1.0 * sxy) / self.effVisc
        dgxz = sxz / self.effVisc
        dslip, dpsi = self.fault.d_dt(sxy[:self.Nz].copy())
        return {"gVxy": dgxy, "gVxz": dgxz, "psi": dpsi, "slip": dslip}

    def time_monitor(self, t, dt, step):
        if self.history is not None:
            f = self.fault
            self.history.append(dict(t=t, dt=dt, step=step, slip=f.slip.copy(), slipVel=f.slipVel.copy(),
                                     psi=f.psi.copy(), tauP=f.tauP.copy(), tauQSP=f.tauQSP.copy(),
                                     surfDisp=self.u[::self.Nz].copy(), gVxy=self.gVxy.copy(),
                                     gVxz=self.gVxz.copy(), sdev=self.sdev.copy(),
                                     effVisc=self.effVisc.copy()))
        return False

    def initiate_integrand(self):
        """StrikeSlip_PowerLaw_qd::initiateIntegrand (:305-350): slip = 2 bcL
        (or inputDir/slip), with guessSteadyStateICs = 1 the steady-state
        iteration first, then the viscous strains of the material and psi of
        the fault."""
        slip = self.bcL * 2.0
        if self.P.get("slip_file") is not None:
            slip = self.P["slip_file"].copy()
        if self.P["driver"]["guessSteadyStateICs"] == 1:
            slip = self.solve_ss()
        return {"gVxy": self.gVxy.copy(), "gVxz": self.gVxz.copy(), "psi": self.fault.psi.copy(), "slip": slip}

    def solve_ss(self):
        """solveSS(0) (strikeSlip_powerLaw_qd.cpp:922-955) with
        solveSSViscoelasticProblem (:1018-1107) and setSSBCs (:1295-1342).
        Sets psi, slipVel, tauP of the fault, the material's effVisc, sxy,
        sxz, sdev, viscous strains and u, bcRShift / bcR; returns the slip.
        self.ss_its / self.ss_err keep the iteration count and last change."""
        f, ss = self.fault, self.P["ss"]
        N, Nz = self.N, self.Nz
        # Fault::guessSS (fault.cpp:633-672)
        f.slipVel = np.full(Nz, self.vL)
        if not self.P["fault"]["stateVals"]:
            f.psi = f.f0 - f.b * np.log(abs(self.vL) / f.v0)
        f.tauP = f.sN * f.a * np.arcsinh(0.5 * self.vL * np.exp(f.psi / f.a) / f.v0)
        # PowerLaw::guessSteadyStateEffVisc (powerLaw.cpp:1999-2037) with
        # DislocationCreep::guessInvEffVisc (:399-433)
        dg = ss["gss_t"]
        temp = self.A * np.exp(-self.Bq / self.T)
        inv_disl = dg / np.power(dg / temp, 1.0 / self.nexp)
        eff = 1.0 / (np.full(N, 1.0 / self.cap) + inv_disl)
        if ss["effVisc_file"] is not None:
            eff = ss["effVisc_file"].copy()
        # guessTauSS (:888-918): tauSS = min(tauRS, gss_t * effVisc on the fault)
        if ss["tauSS_file"] is not None:
            f.tauP = ss["tauSS_file"].copy()
        else:
            f.tauP = np.minimum(f.tauP, eff[:Nz] * dg)
        f.tauQSP = f.tauP.copy()
        # Fault_qd::computeVel (fault.cpp:812-858)
        V, its, conv = compute_vel_qd(f.slipVel, f.tauQSP, f.eta, f.sN, f.psi, f.a, f.locked, f.v0, f.vL,
                                      f.root_tol, f.max_its)
        if not conv:
            raise FloatingPointError("rootFinder BracketedNewton did not converge")
        f.slipVel = V
        # solveSSViscoelasticProblem: bcL = tauSS (traction), bcR = vL / 2
        bcL = f.tauP.copy()
        bcR = np.full(Nz, self.vL / 2.0)
        d = self.P["domain"]
        grid = d["gridSpacingType"]
        err, it = 1e10, 0
        trace = []  # the relative change of every iteration
        v = np.zeros(N)
        sxy = np.zeros(N)
        sxz = np.zeros(N)
        while it < ss["maxSSIts_effVisc"] and err >= ss["atolSS_effVisc"]:
            old = eff.copy()
            # initializeSSMatrices / setSSRHS (powerLaw.cpp:2040-2096): the
            # operator with mu = effVisc, R Dirichlet, T / L / B Neumann
            sbp = SbpOps(d["order"], self.Ny, self.Nz, d["Ly"], d["Lz"], eff, grid=grid,
                         y=self.P["y"] if grid != "constantGridSpacing" and self.Ny > 1 else None,
                         z=self.P["z"] if grid != "constantGridSpacing" and self.Nz > 1 else None,
                         compat=d["sbpCompatibilityType"],
                         bcs=("Dirichlet", "Neumann", "Neumann", "Neumann"))
            rhs = sbp.set_rhs(bcL, bcR, self.bcT, self.bcB)
            # updateSSa (:2099-2137)
            v = self._refined(sbp.A, spla.splu(sbp.A.tocsc()), rhs)
            gxy_t = sbp.Dy_Iz @ v
            gxz_t = sbp.Iy_Dz @ v
            sxy = eff * gxy_t
            sxz = eff * gxz_t
            sdev = np.sqrt(np.abs(sxy * sxy + sxz * sxz))
            inv = 1e3 * self.A * np.power(sdev, self.nexp - 1.0) * np.exp(-self.Bq / self.T)
            new = 1.0 / (np.full(N, 1.0 / self.cap) + 1.0 * inv)
            # MyVecLog10AXPBY (genFuncs.cpp:339-365)
            fss = ss["fss_EffVisc"]
            eff = np.power(10.0, (1.0 - fss) * np.log10(old) + fss * np.log10(new))
            # computeNormDiff_L2_scaleL2 (genFuncs.cpp:221-238)
            err = np.linalg.norm(eff - old) / np.linalg.norm(old)
            trace.append(err)
            it += 1
        self.ss_its, self.ss_err, self.ss_trace = it, err, trace
        self.effVisc = eff
        self.sxy, self.sxz = sxy, sxz
        self.sdev = np.sqrt(np.abs(sxy * sxy + sxz * sxz))
        # updateSSb (:2140-2195) at initTime
        t0 = self.P["driver"]["initTime"]
        u = v * t0
        mn = u.min()
        if mn < 0:
            u = u + abs(mn)
        self.gVxy = (sbp.Dy_Iz @ v) * t0 - sxy / self.mu if it else self.gVxy
        self.gVxz = (sbp.Iy_Dz @ v) * t0 - sxz / self.mu if it else self.gVxz
        # setSSBCs: non-negative u, bcRShift = u at y = Ly, slip = u at y = 0
        mn = u.min()
        if mn < 0:
            u = u + abs(mn)
        self.u = u
        self.bcRShift = u[-Nz:].copy()
        self.bcR = self.bcRShift.copy()
        slip = u[:Nz].copy()
        if self.P["driver"]["bcLType"] == "symmFault":
            slip = slip * 2.0
        return slip
