"""The library's reader of the heat-equation settings and its initial
geotherm against the oracle (CPU: the loader needs no GPU).

The C++ loader behind scy_qd_create_from_in computes the initial
steady-state geotherm of HeatEquation (computeInitialSteadyStateTemp,
heatEquation.cpp:525-683) column by column on the host; it must agree with
the oracle's assembled solve to rounding, on constant and stretched grids,
with heat production and with the mantle adiabat below a lithosphere of
Nz_lab nodes.
"""
import ctypes as C

import numpy as np
import pytest

from oracle.heat import HeatEquation
from oracle.problem import build_qd_problem
from scycle_b200 import _lib as S
from scycle_b200.configs import make_qd_problem

THERMAL = {"thermalCoupling": "uncoupled", "timeIntegrator": "RK32_WBE", "kVals": "[2 2]", "kDepths": "[0 30]",
           "cVals": "[900 900]", "cDepths": "[0 30]", "TVals": "[283 733]", "TDepths": "[0 30]",
           "withRadioHeatGeneration": "no"}


def _field(path, name):
    L = S.lib()
    n = C.c_long()
    S.check(L.scy_in_problem_field(path.encode(), name.encode(), None, 0, C.byref(n)))
    out = np.empty(n.value)
    S.check(L.scy_in_problem_field(path.encode(), name.encode(), S.as_dptr(out), n.value, C.byref(n)))
    return out


def _case(tmp_path, n, grid, extra):
    kw = dict(Ny=n, Nz=n, grid=grid, name="th", extra=dict(THERMAL, **extra))
    if grid == "variableGridSpacing":
        kw["stretch_beta"] = 1.5
    path = make_qd_problem(str(tmp_path), **kw)
    text = open(path).read()
    return path, HeatEquation(build_qd_problem(text), text)


@pytest.mark.parametrize("grid", ["constantGridSpacing", "variableGridSpacing"])
@pytest.mark.parametrize("extra", [
    {},
    {"withRadioHeatGeneration": "yes", "he_A0Vals": "[0.8 0.2]", "he_A0Depths": "[0 30]", "he_Lrad": "10"},
    {"Nz_lab": "17", "TVals": "[283 1200 1200.5 1250]", "TDepths": "[0 20 20.001 30]"},
    {"kVals": "[2 3.5]", "kDepths": "[0 30]"},
], ids=["linear", "radiogenic", "adiabat", "k_varies"])
def test_initial_geotherm_matches_oracle(tmp_path, grid, extra):
    path, he = _case(tmp_path, 25, grid, extra)
    for nm, ref in (("Tamb", he.Tamb), ("T", he.T), ("heat_k", he.k), ("heat_c", he.c), ("heat_rho", he.rho),
                    ("Qrad", he.Qrad)):
        got = _field(path, nm)
        assert got.shape == ref.shape, nm
        assert np.max(np.abs(got - ref)) <= 1e-12 * max(np.max(np.abs(ref)), 1.0), nm


def test_heat_settings_errors(tmp_path):
    bad = make_qd_problem(str(tmp_path / "a"), Ny=9, Nz=9, name="bad",
                          extra=dict(THERMAL, timeIntegrator="RK32"))
    n = C.c_long()
    assert S.lib().scy_in_problem_field(bad.encode(), b"Tamb", None, 0, C.byref(n)) != 0
    assert b"RK32_WBE" in S.lib().scy_get_last_error()
    bad2 = make_qd_problem(str(tmp_path / "b"), Ny=9, Nz=9, name="bad2", state_law="flashHeating")
    assert S.lib().scy_in_problem_field(bad2.encode(), b"Tamb", None, 0, C.byref(n)) != 0
