"""The thermal quasi-dynamic driver on the device against the oracle (GPU).

thermalCoupling uncoupled / coupled with RK32_WBE / RK43_WBE: the RK stages
with a strict acceptance test, then after every accepted step one
backward-Euler step of the heat equation (HeatEquation::be_transient, or
be_steadyState) with the new slip velocity and shear stress; coupled, the
fault's temperature is the heat equation's of the step before, and the
flash-heating state law reads it.  The oracle (oracle/heat.py: QDThermal)
replays the device's attempts; slip, slip velocity, state, shear stress,
the temperature field, its change T - Tamb (the heat step's unknown) and the
weakening velocity agree to 1e-9.
"""
import numpy as np
import pytest

from oracle.heat import QDThermal
from oracle.problem import build_qd_problem
from scycle_b200.configs import make_qd_problem

pytestmark = pytest.mark.gpu

REL = 1e-9
BASE = {"kVals": "[2 2]", "kDepths": "[0 30]", "cVals": "[900 900]", "cDepths": "[0 30]", "TVals": "[283 733]",
        "TDepths": "[0 30]", "withRadioHeatGeneration": "no", "thermalCoupling": "uncoupled",
        "timeIntegrator": "RK32_WBE", "heatEquationType": "transient", "withFrictionalHeating": "no",
        "withViscShearHeating": "no", "maxDeltaT": "1e7", "kspTol_heateq": "1e-14"}


def _nrel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _run(tmp_path, extra, steps, n=21, grid="constantGridSpacing", prestress=None):
    from scycle_b200.configs import write_petsc_vec
    from scycle_b200.qd import QD
    kw = dict(Ny=n, Nz=n, grid=grid, name="th", extra=dict(BASE, **extra))
    if grid == "variableGridSpacing":
        kw["stretch_beta"] = 1.5
    path = make_qd_problem(str(tmp_path), **kw)
    if prestress is not None:
        write_petsc_vec(path[:-len(".in")] + "_in_prestress", prestress + np.linspace(0.0, 0.5, n))
    text = open(path).read()
    dev = QD.from_in(path, solve_rtol=1e-14, exact_jacobian=False)
    dev.record_attempts(True)
    dev.integrate_begin_from_in()
    st = dev.integrate_steps(steps)
    ora = QDThermal(build_qd_problem(text), text, keep_history=False)
    rk = ora.integrate(max_steps=steps, replay=dev.attempts())
    assert st.step_count == rk.stepCount == steps
    assert abs(st.t - rk.currT) <= 1e-12 * abs(rk.currT)
    f = ora.fault
    errs = {"slip": _nrel(dev.field("slip"), f.slip), "slipVel": _nrel(dev.field("slipVel"), f.slipVel),
            "psi": _nrel(dev.field("psi"), f.psi), "tauP": _nrel(dev.field("tauP"), f.tauP),
            "T": _nrel(dev.field("T"), ora.he.T)}
    # the heat step's unknown itself (T - Tamb is far smaller than T here)
    if np.any(ora.he.dT):
        errs["dT"] = _nrel(dev.field("dT"), ora.he.dT)
    else:
        errs["dT"] = float(np.max(np.abs(dev.field("dT"))))
    return dev, ora, errs


def test_uncoupled_without_sources_keeps_the_geotherm(tmp_path):
    dev, ora, errs = _run(tmp_path, {}, 20)
    assert max(errs.values()) <= REL, errs
    assert np.array_equal(ora.he.T, ora.he.Tamb) and errs["dT"] == 0.0


@pytest.mark.parametrize("integrator", ["RK32_WBE", "RK43_WBE"])
def test_coupled_frictional_and_flash_heating_match_oracle(tmp_path, integrator):
    extra = {"thermalCoupling": "coupled", "withFrictionalHeating": "yes", "stateLaw": "flashHeating",
             "TwVals": "[1000 1000]", "TwDepths": "[0 30]", "timeIntegrator": integrator}
    dev, ora, errs = _run(tmp_path, extra, 15, prestress=26.0)
    assert max(errs.values()) <= REL, errs
    assert np.max(np.abs(ora.he.dT)) > 0  # the run heated the fault
    assert _nrel(dev.field("Vw"), ora.fault.Vw) <= REL


def test_shear_zone_of_finite_width_on_the_stretched_grid(tmp_path):
    """A Gaussian shear zone (wVals, m) puts the frictional heat into the
    body; on the stretched grid the body source enters the step."""
    extra = {"thermalCoupling": "coupled", "withFrictionalHeating": "yes", "wVals": "[500 500]",
             "wDepths": "[0 30]"}
    dev, ora, errs = _run(tmp_path, extra, 12, grid="variableGridSpacing", prestress=26.0)
    assert max(errs.values()) <= REL, errs
    assert np.max(np.abs(ora.he.dT)) > 0


def test_steady_state_heat_step(tmp_path):
    extra = {"thermalCoupling": "coupled", "withFrictionalHeating": "yes", "heatEquationType": "steadyState"}
    dev, ora, errs = _run(tmp_path, extra, 10, prestress=26.0)
    assert max(errs.values()) <= REL, errs
