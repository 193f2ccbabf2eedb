"""Heat equation: settings, fields and the initial steady-state geotherm
(oracle; test infrastructure only).

Restates HeatEquation (source/heatEquation.cpp): loadSettings :138-216,
checkInput :369-407, setFields :316-366, loadFieldsFromFiles :217-259 and
computeInitialSteadyStateTemp :525-683, on the oracle SBP operator with the
"z" Laplace type (sbpOps_m_constGrid.cpp:621-690, :886-905).  The initial
temperature solves k T'' = -Qrad column by column in the lithosphere (the
first Nz_lab nodes of every column, down to Lz_lab = TDepths[1]) with
Dirichlet values from the linear extrapolation of TVals[0..1] at z = 0 and
z = Lz_lab, then follows the mantle adiabat of the last two TVals below the
lithosphere when four TVals are given.

Differences from the reference, both where it is undefined: he_Lrad has no
default there (an uninitialised member); here a missing he_Lrad with a
nonzero he_A0Vals is an error and with zero he_A0Vals gives Qrad = 0.

The transient problem (setUpTransientProblem :1627-1711) and its
backward-Euler step (be_transient :1146-1240) are restated with the shear
heating sources (constructMapV :460-523, computeViscousShearHeating
:1509-1540, computeFrictionalShearHeating :1543-1576): a shear zone of zero
width puts the frictional heat tau*V/2 into the fault boundary as a flux,
a finite width spreads it into the body with the Gaussian Gw.  As in the
reference, the body source J*Q enters the step only on the variable grid
(on the constant grid be_transient multiplies H by a fresh, zero vector),
and the boundary data enter the step as + dt (rho c)^-1 setRhs, the sign of
the source term: the steady problem solves A T = setRhs, so a zero-width
shear zone's flux bcL = -tau V / 2 lowers the temperature at the fault in
the step as written.  Both are kept.

QDThermal restates StrikeSlip_LinearElastic_qd with thermalCoupling =
uncoupled or coupled and the RK32_WBE / RK43_WBE integrators (constructor :45-52,
initiateIntegrand :395-404, the IMEX d_dt :800-870): after every accepted
step the heat equation takes one backward-Euler step with the new slip
velocity and shear stress, and in coupled mode the fault's temperature is
the heat equation's of the step before, set at the start of that d_dt;
flash heating (stateLaw = flashHeating, fault.cpp:2162-2243) reads it.

be_steadyState (:1242-1318, setUpSteadyStateProblem :1577-1625) is the
heatEquationType = steadyState step: A dT = setRhs - H J Q on both grids.

PLThermal restates StrikeSlip_PowerLaw_qd with the heat equation
(constructor :43-52, initiateIntegrand :329-333, the IMEX d_dt :692-781):
coupled, the material's temperature (the viscosity's exp(-B/T)) starts at
the heat equation's geotherm and, like the fault's, is the previous step's
at every IMEX d_dt; the heat step adds the viscous shear heating sdev |dgV|.
"""
import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from .infile import atof, atoi, load_vector_double, parse_lines, set_vec
from .powerlaw import PowerLawQD
from .problem import _load_vec_file
from .qd import QDLinearElastic
from .sbp2d import SbpOps


def heat_settings(text, Nz):
    """HeatEquation::loadSettings + the constructor defaults (:7-23) and
    checkInput (:369-407)."""
    h = dict(heatEquationType="transient", withViscShearHeating="yes", withFrictionalHeating="yes",
             withRadioHeatGeneration="yes", linSolver_heateq="CG", kspTol_heateq=1e-11, Nz_lab=Nz,
             rhoVals=[], rhoDepths=[], kVals=[], kDepths=[], cVals=[], cDepths=[], TVals=[], TDepths=[],
             wVals=[], wDepths=[], he_A0Vals=[], he_A0Depths=[], he_Lrad=None)
    lists = ("rhoVals", "rhoDepths", "kVals", "kDepths", "cVals", "cDepths", "TVals", "TDepths",
             "wVals", "wDepths", "he_A0Vals", "he_A0Depths")
    for var, rhs, full in parse_lines(text):
        if var in lists:
            h[var] = h[var] + load_vector_double(full)
        elif var in ("heatEquationType", "withViscShearHeating", "withFrictionalHeating",
                     "withRadioHeatGeneration", "linSolver_heateq"):
            h[var] = rhs
        elif var == "kspTol_heateq":
            h[var] = atof(rhs)
        elif var == "Nz_lab":
            h[var] = atoi(rhs)
        elif var == "he_Lrad":
            h[var] = atof(rhs)
    if h["heatEquationType"] not in ("transient", "steadyState"):
        raise ValueError("heatEquationType must be transient or steadyState")
    for a, b in (("kVals", "kDepths"), ("rhoVals", "rhoDepths"), ("cVals", "cDepths"),
                 ("TVals", "TDepths"), ("wVals", "wDepths")):
        if len(h[a]) != len(h[b]):
            raise ValueError("%s and %s differ in length" % (a, b))
    if not 2 <= len(h["TVals"]) <= 4:
        raise ValueError("TVals needs 2 to 4 entries")
    if h["Nz_lab"] > Nz:
        raise ValueError("Nz_lab must not exceed Nz")
    h["Lz_lab"] = h["TDepths"][1]
    if h["withRadioHeatGeneration"] == "yes":
        if len(h["he_A0Vals"]) != len(h["he_A0Depths"]):
            raise ValueError("he_A0Vals and he_A0Depths differ in length")
        if not h["he_A0Vals"]:
            h["he_A0Vals"], h["he_A0Depths"] = [0.0], [0.0]
    return h


class HeatEquation:
    """The fields of HeatEquation and its initial steady-state temperature."""

    def __init__(self, P, text):
        d = P["domain"]
        self.P = P
        self.Ny, self.Nz = P["Ny"], P["Nz"]
        self.N = self.Ny * self.Nz
        h = heat_settings(text, self.Nz)
        self.h = h
        if h["Lz_lab"] > d["Lz"]:
            raise ValueError("the LAB depth TDepths[1] must not exceed Lz")
        z = P["z"]
        # setFields (:316-366)
        self.k = set_vec(z, h["kVals"], h["kDepths"])
        self.rho = set_vec(z, h["rhoVals"], h["rhoDepths"])
        self.c = set_vec(z, h["cVals"], h["cDepths"])
        self.Tamb = set_vec(z, h["TVals"], h["TDepths"])
        self.T = self.Tamb.copy()
        self.dT = np.zeros(self.N)
        if h["withRadioHeatGeneration"] == "yes":
            A0 = set_vec(z, h["he_A0Vals"], h["he_A0Depths"])
            if h["he_Lrad"] is None:
                if np.any(A0 != 0):
                    raise ValueError("he_Lrad is needed with a nonzero he_A0Vals")
                self.Qrad = np.zeros(self.N)
            else:
                self.Qrad = A0 * np.exp(-z / h["he_Lrad"])
        else:
            self.Qrad = np.zeros(self.N)
        # loadFieldsFromFiles (:217-259)
        inp = d["inputDir"]
        for nm, attr in (("rho", "rho"), ("k", "k"), ("h", "Qrad"), ("c", "c")):
            v = _load_vec_file(inp, nm, self.N)
            if v is not None:
                setattr(self, attr, v)
        Tamb = _load_vec_file(inp, "Tamb", self.N)
        T = _load_vec_file(inp, "T", self.N)
        dT = _load_vec_file(inp, "dT", self.N)
        self.load_ics = Tamb is not None
        if Tamb is not None:
            self.Tamb = Tamb
        if T is not None:
            self.T = T
        elif Tamb is not None:
            self.T = Tamb.copy()
        if dT is not None:
            self.dT = dT
        elif Tamb is not None:
            self.dT = self.T - self.Tamb
        if not self.load_ics:
            self.initial_steady_state_temp()
        # constructMapV (:460-523): shear-zone width w (m -> km) and the
        # Gaussian Gw = exp(-y^2 / (2 w^2)) / sqrt(2 pi) / w
        self.w = np.zeros(self.N)
        self.Gw = np.zeros(self.N)
        if h["wVals"]:
            self.w = set_vec(z, h["wVals"], h["wDepths"]) * 1e-3
            y = P["y"]
            self.Gw = np.exp(-y * y / (2.0 * self.w * self.w)) / np.sqrt(2.0 * np.pi) / self.w
        self.wMax = float(np.max(self.w))
        if h["heatEquationType"] == "transient":
            self.setup_transient()
        else:
            self.setup_steady_state()

    def lith_index(self):
        """bodyFull2bodyLith (constructScatters :409-458): the nodes with
        iz < Nz_lab, column by column."""
        Nzl = self.h["Nz_lab"]
        iy, iz = np.meshgrid(np.arange(self.Ny), np.arange(Nzl), indexing="ij")
        return (iy * self.Nz + iz).ravel()

    def initial_steady_state_temp(self):
        """computeInitialSteadyStateTemp (:525-683)."""
        h, d = self.h, self.P["domain"]
        TV, TD = h["TVals"], h["TDepths"]
        if self.Nz == 1:
            self.Tamb = np.full(self.N, TV[0])
            self.T = self.Tamb.copy()
            self.dT = np.zeros(self.N)
            return
        slope = (TV[1] - TV[0]) / (TD[1] - TD[0])
        bcT = np.full(self.Ny, slope * (0.0 - TD[0]) + TV[0])
        bcB = np.full(self.Ny, slope * (h["Lz_lab"] - TD[0]) + TV[0])
        idx = self.lith_index()
        Nzl = h["Nz_lab"]
        grid = d["gridSpacingType"]
        var = grid == "variableGridSpacing"
        # SbpOps(order, Ny, Nz_lab, Ly, Lz, k) with the full Ly, Lz (the
        # constant grid then spaces Nz_lab points over Lz, as the reference
        # does), Dirichlet on every side, Laplace type "z"
        sbp = SbpOps(d["order"], self.Ny, Nzl, d["Ly"], d["Lz"], self.k[idx], grid=grid,
                     y=self.P["y"][idx] if var and self.Ny > 1 else None,
                     z=self.P["z"][idx] if var and Nzl > 1 else None,
                     compat=d["sbpCompatibilityType"], bcs=("Dirichlet",) * 4, laplace="z")
        rhs = sbp.set_rhs(np.zeros(Nzl), np.zeros(Nzl), bcT, bcB)
        if h["withRadioHeatGeneration"] == "yes":
            Q = self.Qrad[idx]
            if var:
                Q = sbp.yq @ (sbp.zr @ Q)  # J = yq zr
            rhs = rhs - sbp.H @ Q
        Tl = spla.splu(sbp.A.tocsc()).solve(rhs)
        self.Tamb = self.Tamb.copy()
        self.Tamb[idx] = Tl
        # the mantle adiabat below the lithosphere
        if Nzl < self.Nz and h["Lz_lab"] < d["Lz"] and len(TV) > 3:
            a = (TV[-1] - TV[-2]) / (TD[-1] - TD[-2])
            z = self.P["z"]
            below = z >= h["Lz_lab"]
            self.Tamb[below] = a * (z[below] - TD[-2]) + TV[-2]
        self.dT = np.zeros(self.N)
        self.T = self.Tamb.copy()

    def setup_transient(self):
        """setUpTransientProblem (:1627-1711): the operator of k with R, T and
        B Dirichlet and L Neumann (zero data), I = (J) H, rcInv = 1/(rho c)
        and D2ath = rcInv A."""
        d = self.P["domain"]
        grid = d["gridSpacingType"]
        var = grid == "variableGridSpacing"
        self.sbp = SbpOps(d["order"], self.Ny, self.Nz, d["Ly"], d["Lz"], self.k, grid=grid,
                          y=self.P["y"] if var and self.Ny > 1 else None,
                          z=self.P["z"] if var and self.Nz > 1 else None,
                          compat=d["sbpCompatibilityType"],
                          bcs=("Dirichlet", "Dirichlet", "Neumann", "Dirichlet"))
        s = self.sbp
        self.I = ((s.yq @ s.zr) @ s.H).tocsr() if var else s.H.copy()
        self.rcInv = sp.diags(1.0 / (self.rho * self.c))
        self.D2ath = (self.rcInv @ s.A).tocsr()

    def setup_steady_state(self):
        """setUpSteadyStateProblem (:1577-1625): the operator of k with R, T
        and B Dirichlet and L Neumann."""
        d = self.P["domain"]
        grid = d["gridSpacingType"]
        var = grid == "variableGridSpacing"
        self.sbp = SbpOps(d["order"], self.Ny, self.Nz, d["Ly"], d["Lz"], self.k, grid=grid,
                          y=self.P["y"] if var and self.Ny > 1 else None,
                          z=self.P["z"] if var and self.Nz > 1 else None,
                          compat=d["sbpCompatibilityType"],
                          bcs=("Dirichlet", "Dirichlet", "Neumann", "Dirichlet"))
        self.lu_ss = spla.splu(self.sbp.A.tocsc())

    def be_steady_state(self, slipVel, tau, Tn, dt, sdev=None, dgxy=None, dgxz=None):
        """be_steadyState (:1242-1318): A dT = setRhs - H J (Qfric + Qvisc)
        on both grids; returns T and keeps T, dT."""
        h = self.h
        s = self.sbp
        var = self.P["domain"]["gridSpacingType"] == "variableGridSpacing"
        bcL = np.zeros(self.Nz)
        Q = np.zeros(self.N)
        if h["withFrictionalHeating"] == "yes":
            bcL, Qfric = self.frictional_heating(tau, slipVel)
            Q = Q - Qfric
        if h["withViscShearHeating"] == "yes" and sdev is not None and dgxy is not None and dgxz is not None:
            Q = Q - sdev * np.sqrt(np.abs(dgxy * dgxy + dgxz * dgxz))
        rhs = s.set_rhs(bcL, np.zeros(self.Nz), np.zeros(self.Ny), np.zeros(self.Ny))
        rhs = rhs + (s.H @ ((s.yq @ s.zr) @ Q) if var else s.H @ Q)
        self.dT = self.lu_ss.solve(rhs)
        self.T = self.Tamb + self.dT
        return self.T.copy()

    def be(self, slipVel, tau, Tn, dt, sdev=None, dgxy=None, dgxz=None):
        """HeatEquation::be (:1108-1143): the transient or steady step, then
        the heat flux."""
        if self.h["heatEquationType"] == "transient":
            T = self.be_transient(slipVel, tau, Tn, dt, sdev, dgxy, dgxz)
        else:
            T = self.be_steady_state(slipVel, tau, Tn, dt, sdev, dgxy, dgxz)
        self.compute_heat_flux()
        return T

    def compute_heat_flux(self):
        """computeHeatFlux (:1713-1733): kTz = 1e9 k Dz T over the body and
        its values at the surface z = 0 (body2T: node iz = 0 of each column)."""
        self.kTz = self.sbp.muxDz(self.T) * 1e9
        self.kTz_z0 = self.kTz[::self.Nz].copy()
        return self.kTz_z0

    def frictional_heating(self, tau, slipVel):
        """computeFrictionalShearHeating (:1543-1576): returns (bcL, Qfric)."""
        q = tau * slipVel
        if self.wMax == 0:
            return -0.5 * q, np.zeros(self.N)
        Qfric = np.tile(q, self.Ny) * self.Gw  # MapV: node i takes fault value i % Nz
        return np.zeros(self.Nz), Qfric

    def be_transient(self, slipVel, tau, Tn, dt, sdev=None, dgxy=None, dgxz=None):
        """be_transient (:1146-1240): one backward-Euler step from Tn over dt;
        returns T and keeps T, dT."""
        h = self.h
        s = self.sbp
        var = self.P["domain"]["gridSpacingType"] == "variableGridSpacing"
        bcL = np.zeros(self.Nz)
        Q = np.zeros(self.N)
        if h["withFrictionalHeating"] == "yes":
            bcL, Qfric = self.frictional_heating(tau, slipVel)
            Q = Q + Qfric
        if h["withViscShearHeating"] == "yes" and sdev is not None and dgxy is not None and dgxz is not None:
            Q = Q + sdev * np.sqrt(np.abs(dgxy * dgxy + dgxz * dgxz))
        temp = s.set_rhs(bcL, np.zeros(self.Nz), np.zeros(self.Ny), np.zeros(self.Ny))
        if var:
            temp = temp + s.H @ ((s.yq @ s.zr) @ Q)
        rhs = dt * (self.rcInv @ temp)
        dTn = Tn - self.Tamb
        Hd = s.H @ dTn
        if var:
            Hd = (s.yq @ s.zr) @ Hd
        rhs = rhs + Hd
        B = (self.I - dt * self.D2ath).tocsc()
        self.dT = spla.spsolve(B, rhs)
        self.T = self.Tamb + self.dT
        return self.T.copy()


class QDThermal(QDLinearElastic):
    """StrikeSlip_LinearElastic_qd with the heat equation (thermalCoupling
    uncoupled / coupled) integrated by RK32_WBE or RK43_WBE."""

    def __init__(self, P, text, keep_history=True):
        super().__init__(P, keep_history)
        s = P["driver"]
        if s["thermalCoupling"] not in ("uncoupled", "coupled"):
            raise ValueError("thermalCoupling must be uncoupled or coupled")
        if s["timeIntegrator"] not in ("RK32_WBE", "RK43_WBE"):
            raise ValueError("the thermal driver integrates with RK32_WBE or RK43_WBE")
        self.he = HeatEquation(P, text)
        self.coupled = s["thermalCoupling"] == "coupled"
        self.flash = s["stateLaw"] == "flashHeating"
        Nz = self.Nz
        if self.flash:
            fs = P["fault"]
            zf = P["z"][:Nz]
            # setThermalFields (fault.cpp:316-345): T = Tamb, k and c on the
            # fault, Vw = Vw_const until the first d_dt
            self.fault.flash = dict(T=self.he.Tamb[:Nz].copy(), rho=np.asarray(P["rho_f"], float),
                                    c=self.he.c[:Nz].copy(), k=self.he.k[:Nz].copy(),
                                    Tw=set_vec(zf, fs["TwVals"], fs["TwDepths"]), D=fs["D"],
                                    tau_c=fs["tau_c"], fw=fs["fw"])
            self.fault.Vw = np.full(Nz, fs["Vw"])

    def initiate_integrand(self):
        var = super().initiate_integrand()
        if self.flash:  # _fault->updateTemperature(_he->_T)
            self.fault.flash["T"] = self.he.T[:self.Nz].copy()
        return var

    def imex_before(self, t, dt):
        """updateTemperature(varImo) at the start of the IMEX d_dt (coupled)."""
        if self.coupled and self.flash:
            self.fault.flash["T"] = self.he.T[:self.Nz].copy()

    def imex_after(self, t, dt, dvar):
        """HeatEquation::be with the new slip velocity and tauP."""
        self.he.be(dvar["slip"], self.fault.tauP.copy(), self.he.T.copy(), dt)


class PLThermal(PowerLawQD):
    """StrikeSlip_PowerLaw_qd with the heat equation (thermalCoupling
    uncoupled / coupled) integrated by RK32_WBE or RK43_WBE."""

    def __init__(self, P, text, keep_history=True):
        super().__init__(P, keep_history)
        s = P["driver"]
        if s["thermalCoupling"] not in ("uncoupled", "coupled"):
            raise ValueError("thermalCoupling must be uncoupled or coupled")
        if s["timeIntegrator"] not in ("RK32_WBE", "RK43_WBE"):
            raise ValueError("the thermal driver integrates with RK32_WBE or RK43_WBE")
        self.he = HeatEquation(P, text)
        self.coupled = s["thermalCoupling"] == "coupled"
        if self.coupled:  # VecCopy(_he->_T, _material->_T)
            self.T = self.he.T.copy()
        self.flash = s["stateLaw"] == "flashHeating"
        Nz = self.Nz
        if self.flash:
            fs = P["fault"]
            zf = P["z"][:Nz]
            self.fault.flash = dict(T=self.he.T[:Nz].copy(), rho=np.asarray(P["rho_f"], float),
                                    c=self.he.c[:Nz].copy(), k=self.he.k[:Nz].copy(),
                                    Tw=set_vec(zf, fs["TwVals"], fs["TwDepths"]), D=fs["D"],
                                    tau_c=fs["tau_c"], fw=fs["fw"])
            self.fault.Vw = np.full(Nz, fs["Vw"])

    def initiate_integrand(self):
        var = super().initiate_integrand()
        if self.flash:
            self.fault.flash["T"] = self.he.T[:self.Nz].copy()
        return var

    def imex_before(self, t, dt):
        if self.coupled:
            if self.flash:
                self.fault.flash["T"] = self.he.T[:self.Nz].copy()
            self.T = self.he.T.copy()

    def imex_after(self, t, dt, dvar):
        self.he.be(dvar["slip"], self.fault.tauP.copy(), self.he.T.copy(), dt, sdev=self.sdev.copy(),
                   dgxy=dvar["gVxy"], dgxz=dvar["gVxz"])
