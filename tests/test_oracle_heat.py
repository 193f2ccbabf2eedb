"""The heat-equation oracle's initial steady-state geotherm (CPU).

HeatEquation::computeInitialSteadyStateTemp solves k T'' = -Qrad in the
lithosphere with Dirichlet temperatures at z = 0 and at the LAB; the SBP-SAT
operator with the "z" Laplace type reproduces linear profiles exactly and
quadratic ones (constant heat production) to the boundary closure's order,
and below the LAB the temperature follows the mantle adiabat of the last
two TVals.
"""
import numpy as np
import pytest

from oracle.heat import HeatEquation, heat_settings
from oracle.problem import build_qd_problem
from scycle_b200.configs import make_qd_problem


def _problem(tmp_path, n=25, grid="constantGridSpacing", extra=None, name="he"):
    kw = dict(Ny=n, Nz=n, grid=grid, name=name, extra=extra or {})
    if grid == "variableGridSpacing":
        kw["stretch_beta"] = 1.5
    path = make_qd_problem(str(tmp_path), **kw)
    text = open(path).read()
    return build_qd_problem(text), text


LINEAR = {"kVals": "[2 2]", "kDepths": "[0 30]", "TVals": "[283 733]", "TDepths": "[0 30]",
          "withRadioHeatGeneration": "no", "rhoVals": "[3 3]", "rhoDepths": "[0 30]",
          "cVals": "[900 900]", "cDepths": "[0 30]"}


def test_linear_geotherm_is_exact(tmp_path):
    P, text = _problem(tmp_path, extra=LINEAR)
    he = HeatEquation(P, text)
    exact = 283.0 + 450.0 * P["z"] / 30.0
    assert np.max(np.abs(he.T - exact)) <= 1e-9 * 733.0
    assert np.array_equal(he.T, he.Tamb) and not np.any(he.dT)


def test_linear_geotherm_stretched_grid_converges(tmp_path):
    """On a stretched grid the SBP remainder term acts on a profile that is
    linear in z but not in the logical coordinate: the error falls at least
    like h^2."""
    errs = []
    for n in (21, 41, 81):
        P, text = _problem(tmp_path / str(n), n=n, grid="variableGridSpacing", extra=LINEAR)
        he = HeatEquation(P, text)
        errs.append(np.max(np.abs(he.T - (283.0 + 450.0 * P["z"] / 30.0))))
    assert errs[0] / errs[1] >= 3.5 and errs[1] / errs[2] >= 3.5
    assert errs[-1] <= 1e-3 * 733.0


def test_heat_production_converges(tmp_path):
    """k T'' = -A0 with T(0) = T0, T(L) = TL: T = T0 + (TL - T0) z / L +
    A0 z (L - z) / (2 k); the error falls at least like h^2."""
    errs = []
    for n in (21, 41, 81):
        extra = {"kVals": "[2 2]", "kDepths": "[0 30]", "TVals": "[283 733]", "TDepths": "[0 30]",
                 "withRadioHeatGeneration": "yes", "he_A0Vals": "[0.5 0.5]", "he_A0Depths": "[0 30]",
                 "he_Lrad": "1e30", "rhoVals": "[3 3]", "rhoDepths": "[0 30]", "cVals": "[900 900]",
                 "cDepths": "[0 30]"}
        P, text = _problem(tmp_path / str(n), n=n, extra=extra)
        he = HeatEquation(P, text)
        z = P["z"]
        exact = 283.0 + 450.0 * z / 30.0 + 0.5 * z * (30.0 - z) / (2.0 * 2.0)
        errs.append(np.max(np.abs(he.T - exact)))
    assert errs[-1] <= 1e-6 * 733.0
    assert errs[0] / errs[1] >= 3.5 or errs[1] <= 1e-10 * 733.0
    assert errs[1] / errs[2] >= 3.5 or errs[2] <= 1e-10 * 733.0


def test_mantle_adiabat_below_the_lab(tmp_path):
    """Four TVals: linear conduction down to the LAB (TDepths[1] = 20 km,
    the first 21 of 31 nodes of every column), the adiabat of TVals[2..3]
    below it."""
    n, nz_lab, lab = 31, 21, 20.0
    extra = {"kVals": "[2 2]", "kDepths": "[0 30]", "rhoVals": "[3 3]", "rhoDepths": "[0 30]",
             "cVals": "[900 900]", "cDepths": "[0 30]", "withRadioHeatGeneration": "no",
             "Nz_lab": str(nz_lab), "TVals": "[283 1200 1200.5 1250]",
             "TDepths": "[0 %r %r 30]" % (lab, lab + 1e-3)}
    P, text = _problem(tmp_path / "lab", n=n, extra=extra)
    he = HeatEquation(P, text)
    z = P["z"]
    above = (np.arange(P["N"]) % n < nz_lab) & (z < lab)  # the LAB node itself takes the adiabat (z >= Lz_lab)
    lin = 283.0 + (1200.0 - 283.0) * z / lab
    assert np.max(np.abs(he.T[above] - lin[above])) <= 1e-9 * 1250.0
    below = z >= lab
    adiabat = (1250.0 - 1200.5) / (30.0 - lab - 1e-3) * (z - lab - 1e-3) + 1200.5
    assert np.allclose(he.T[below], adiabat[below], rtol=0, atol=1e-9 * 1250.0)


def test_heat_settings_checks():
    text = "TVals = [283]\nTDepths = [0]\n"
    with pytest.raises(ValueError):
        heat_settings(text, 10)
    h = heat_settings("TVals = [1 2]\nTDepths = [0 5]\nNz_lab = 7\n", 10)
    assert h["Lz_lab"] == 5 and h["Nz_lab"] == 7 and h["he_A0Vals"] == [0.0]


def _transient_problem(tmp_path, n, grid="constantGridSpacing", extra=None):
    e = dict(LINEAR)
    e.update({"withFrictionalHeating": "no", "withViscShearHeating": "no"})
    e.update(extra or {})
    return _problem(tmp_path, n=n, grid=grid, extra=e)


@pytest.mark.parametrize("grid", ["constantGridSpacing", "variableGridSpacing"])
def test_backward_euler_decays_an_eigenmode(tmp_path, grid):
    """dT = sin(pi z / Lz) cos(pi y / (2 Ly)) meets the transient problem's
    boundary types (Neumann at the fault, Dirichlet elsewhere); one
    backward-Euler step divides it by 1 + dt kappa lambda."""
    n = 41
    P, text = _transient_problem(tmp_path, n, grid)
    he = HeatEquation(P, text)
    y, z = P["y"], P["z"]
    mode = np.sin(np.pi * z / 30.0) * np.cos(np.pi * y / 60.0)
    kappa = 2.0 / (3.0 * 900.0)
    lam = np.pi ** 2 * (1.0 / 900.0 + 1.0 / 3600.0)
    dt = 1.0 / (kappa * lam)
    T = he.be_transient(np.zeros(P["Nz"]), np.zeros(P["Nz"]), he.Tamb + mode, dt)
    dT = T - he.Tamb
    assert np.max(np.abs(dT - mode / 2.0)) <= 2e-3


def test_zero_width_shear_zone_flux_sign(tmp_path):
    """A shear zone of zero width: bcL = -tau V / 2 as the fault boundary's
    Neumann data.  be_transient adds setRhs with the sign of the source
    term, the opposite of the steady problem's A T = setRhs, so the step
    changes the temperature next to the fault by -tau V in sign (a cooling
    the restatement keeps); the change is linear in tau V and largest at
    the fault."""
    P, text = _transient_problem(tmp_path, 31, extra={"withFrictionalHeating": "yes"})
    he = HeatEquation(P, text)
    Nz = P["Nz"]
    he.be_transient(np.full(Nz, 1e-9), np.full(Nz, 30.0), he.Tamb.copy(), 1e9)
    d1 = he.dT.reshape(P["Ny"], Nz).copy()
    he.be_transient(np.full(Nz, 2e-9), np.full(Nz, 30.0), he.Tamb.copy(), 1e9)
    d2 = he.dT.reshape(P["Ny"], Nz).copy()
    assert np.all(d1[0, 1:-1] < 0) and np.all(np.abs(d1[0, 1:-1]) > np.abs(d1[5, 1:-1]))
    assert np.allclose(d2, 2.0 * d1, rtol=1e-10, atol=0)


def test_finite_shear_zone_source_only_on_the_variable_grid(tmp_path):
    """With wVals the frictional heat is a body source tau V Gw; the
    reference's be_transient adds it through J (variable grid) and adds
    nothing on the constant grid."""
    e = {"withFrictionalHeating": "yes", "wVals": "[2000 2000]", "wDepths": "[0 30]"}
    for grid, warms in (("constantGridSpacing", False), ("variableGridSpacing", True)):
        P, text = _transient_problem(tmp_path / grid, 31, grid, extra=e)
        he = HeatEquation(P, text)
        Nz = P["Nz"]
        T = he.be_transient(np.full(Nz, 1e-9), np.full(Nz, 30.0), he.Tamb.copy(), 1e9)
        if warms:
            assert np.max(T - he.Tamb) > 0
        else:
            assert np.max(np.abs(T - he.Tamb)) == 0


def test_flash_heating_law():
    """flashHeating_psi: below Vw the steady state is the regularised
    velocity-weakening friction fLV, above it fw + (fLV - fw) Vw / |V|."""
    from oracle.fault import flash_heating_psi, flash_heating_vw
    a, b, f0, v0, Dc, fw = 0.01, 0.015, 0.6, 1e-6, 0.01, 0.2
    psi = np.array([0.6, 0.7])
    V = np.array([1e-3, 1.0])
    Vw = np.array([0.1, 0.1])
    d = flash_heating_psi(psi, V, Vw, fw, Dc, a, b, f0, v0)
    fLV = (a - b) * np.arcsinh(V / v0 / 2.0 * np.exp(f0 / (a - b)))
    f = a * np.arcsinh(V / 2.0 / v0 * np.exp(psi / a))
    fss = np.array([fLV[0], fw + (fLV[1] - fw) * 0.1 / 1.0])
    assert np.allclose(d, -V / Dc * (f - fss), rtol=1e-14, atol=0)
    vw = flash_heating_vw(300.0, 3.0, 900.0, 2.0, 5.0, 900.0, 3.0)
    assert vw == pytest.approx(np.pi * (2.0 / 2700.0) / 5.0 * (2700.0 * 600.0 / 3.0) ** 2, rel=1e-14)


THERMAL = dict(LINEAR, thermalCoupling="uncoupled", timeIntegrator="RK32_WBE", heatEquationType="transient",
               withFrictionalHeating="no", withViscShearHeating="no")


def test_uncoupled_thermal_run_keeps_the_mechanical_path(tmp_path):
    """Uncoupled and without heat sources, RK32_WBE takes the RK32 path of
    the purely mechanical driver (the strict acceptance test aside) and the
    temperature stays at the geotherm."""
    from oracle.heat import QDThermal
    from oracle.qd import QDLinearElastic
    P, text = _problem(tmp_path / "th", n=21, extra=dict(THERMAL, maxDeltaT="1e7"))
    th = QDThermal(P, text)
    th.integrate(max_steps=25)
    Pm, _ = _problem(tmp_path / "me", n=21, extra=dict(THERMAL, maxDeltaT="1e7", timeIntegrator="RK32"))
    me = QDLinearElastic(Pm)
    me.integrate(max_steps=25)
    assert len(th.history) == len(me.history)
    for a, b in zip(th.history, me.history):
        assert a["t"] == b["t"]
        assert np.array_equal(a["slip"], b["slip"]) and np.array_equal(a["psi"], b["psi"])
    assert np.array_equal(th.he.T, th.he.Tamb) and not np.any(th.he.dT)


def test_coupled_flash_heating_run(tmp_path):
    """Coupled, frictional heating through the fault boundary and the flash
    heating state law: the run advances, the temperature changes, and the
    fault reads the heat equation's temperature of the step before."""
    from oracle.heat import QDThermal
    extra = dict(THERMAL, thermalCoupling="coupled", withFrictionalHeating="yes", stateLaw="flashHeating",
                 TwVals="[1000 1000]", TwDepths="[0 30]", maxDeltaT="1e7")
    P, text = _problem(tmp_path, n=21, extra=extra)
    th = QDThermal(P, text)
    seen = []
    orig = th.imex_after

    def after(t, dt, dvar):
        seen.append(th.he.T[:P["Nz"]].copy())
        orig(t, dt, dvar)
    th.imex_after = after
    th.integrate(max_steps=15)
    assert len(th.history) == 16
    assert np.max(np.abs(th.he.dT)) > 0
    assert np.array_equal(th.fault.flash["T"], seen[-1])
    assert np.all(np.isfinite(th.fault.Vw)) and np.all(th.fault.Vw > 0)


def test_uncoupled_rk43_wbe_matches_rk43_decisions(tmp_path):
    """RK43_WBE without heat sources follows RK43 (L2_absolute errors, the
    same strict acceptance) step for step."""
    from oracle.heat import QDThermal
    from oracle.qd import QDLinearElastic
    P, text = _problem(tmp_path / "th", n=21, extra=dict(THERMAL, maxDeltaT="1e7", timeIntegrator="RK43_WBE"))
    th = QDThermal(P, text)
    th.integrate(max_steps=20)
    Pm, _ = _problem(tmp_path / "me", n=21, extra=dict(THERMAL, maxDeltaT="1e7", timeIntegrator="RK43"))
    me = QDLinearElastic(Pm)
    me.integrate(max_steps=20)
    assert [h["t"] for h in th.history] == [h["t"] for h in me.history]
    assert np.array_equal(th.history[-1]["slip"], me.history[-1]["slip"])


def test_steady_state_step_heats_the_fault(tmp_path):
    """heatEquationType = steadyState: A dT = setRhs - H J Q with the
    steady problem's own sign convention, so the zero-width shear zone's
    flux warms the fault; the result does not depend on dt or Tn."""
    P, text = _transient_problem(tmp_path, 31, extra={"withFrictionalHeating": "yes",
                                                      "heatEquationType": "steadyState"})
    he = HeatEquation(P, text)
    Nz = P["Nz"]
    T1 = he.be(np.full(Nz, 1e-9), np.full(Nz, 30.0), he.Tamb.copy(), 1e9)
    d1 = he.dT.reshape(P["Ny"], Nz).copy()
    T2 = he.be(np.full(Nz, 1e-9), np.full(Nz, 30.0), he.Tamb + 1.0, 5.0)
    assert np.all(d1[0, 1:-1] > 0) and np.all(d1[0, 1:-1] > d1[5, 1:-1])
    assert np.array_equal(T1, T2)


def _pl_thermal_problem(tmp_path, extra):
    from scycle_b200.configs import make_pl_problem
    e = {"kVals": "[2 2]", "kDepths": "[0 30]", "rhoVals": "[3 3]", "rhoDepths": "[0 30]",
         "cVals": "[900 900]", "cDepths": "[0 30]", "withRadioHeatGeneration": "no",
         "maxEffVisc": "1e12", "maxDeltaT": "1e7"}
    e.update(extra)
    path = make_pl_problem(str(tmp_path), Ny=21, Nz=21, extra=e)
    text = open(path).read()
    from oracle.powerlaw import build_pl_problem
    return build_pl_problem(text), text


def test_uncoupled_power_law_thermal_keeps_the_mechanical_path(tmp_path):
    """The power-law driver, uncoupled and without heat sources: RK43_WBE
    takes the RK43 path (the explicit rates do not see the temperature) and
    the temperature stays at the geotherm."""
    from oracle.heat import PLThermal
    from oracle.powerlaw import PowerLawQD
    extra = {"thermalCoupling": "uncoupled", "timeIntegrator": "RK43_WBE", "withFrictionalHeating": "no",
             "withViscShearHeating": "no"}
    P, text = _pl_thermal_problem(tmp_path / "th", extra)
    th = PLThermal(P, text)
    th.integrate(max_steps=10)
    Pm, _ = _pl_thermal_problem(tmp_path / "me", dict(extra, timeIntegrator="RK43"))
    me = PowerLawQD(Pm)
    me.integrate(max_steps=10)
    assert [h["t"] for h in th.history] == [h["t"] for h in me.history]
    assert np.array_equal(th.history[-1]["gVxy"], me.history[-1]["gVxy"])
    assert not np.any(th.he.dT)


def test_coupled_power_law_thermal_run(tmp_path):
    """Coupled with viscous and frictional heating: the material's
    temperature starts at the heat equation's geotherm and follows it one
    step behind."""
    from oracle.heat import PLThermal
    extra = {"thermalCoupling": "coupled", "timeIntegrator": "RK32_WBE", "withFrictionalHeating": "yes",
             "withViscShearHeating": "yes"}
    P, text = _pl_thermal_problem(tmp_path, extra)
    th = PLThermal(P, text)
    T0 = th.T.copy()
    assert np.array_equal(T0, th.he.T)
    seen = []
    orig = th.imex_after

    def after(t, dt, dvar):
        seen.append(th.he.T.copy())
        orig(t, dt, dvar)
    th.imex_after = after
    th.integrate(max_steps=8)
    assert np.max(np.abs(th.he.dT)) > 0
    assert np.array_equal(th.T, seen[-1])


def test_power_law_thermal_with_steady_state_guess(tmp_path):
    """The shape of the reference's thermal example (power law, the
    steady-state initial guess, coupled heat equation, RK43_WBE): the
    steady-state iteration sees the heat equation's geotherm as the
    material temperature, and the coupled run advances."""
    from oracle.heat import PLThermal
    extra = {"thermalCoupling": "coupled", "timeIntegrator": "RK43_WBE", "withFrictionalHeating": "yes",
             "withViscShearHeating": "yes", "guessSteadyStateICs": "1"}
    P, text = _pl_thermal_problem(tmp_path, extra)
    th = PLThermal(P, text)
    th.integrate(max_steps=5)
    assert 1 < th.ss_its < P["ss"]["maxSSIts_effVisc"]
    assert len(th.history) == 6 and np.all(np.isfinite(th.history[-1]["slipVel"]))


def test_surface_heat_flux_of_a_linear_geotherm(tmp_path):
    """computeHeatFlux: 1e9 k dT/dz, exact for the linear geotherm."""
    P, text = _transient_problem(tmp_path, 21)
    he = HeatEquation(P, text)
    Nz = P["Nz"]
    he.be(np.zeros(Nz), np.zeros(Nz), he.Tamb.copy(), 1.0)
    assert np.allclose(he.kTz_z0, 1e9 * 2.0 * 450.0 / 30.0, rtol=1e-10, atol=0)
