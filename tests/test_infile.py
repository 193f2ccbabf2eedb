"""The product's C++ input loader vs the oracle's problem builder (CPU only)."""
import os

import numpy as np
import pytest

from oracle.problem import build_qd_problem
from scycle_b200 import _lib as S
from scycle_b200.configs import make_qd_problem
from scycle_b200.qd import inspect_in
from tests.test_oracle import ex2_text

FIELDS = {"y": "y", "z": "z", "mu": "mu", "rho": "rho", "cs": "cs", "a": "a", "b": "b", "sN": "sN", "Dc": "Dc",
          "psi": "psi", "locked": "locked", "prestress": "prestress", "bcL": "bcL0", "bcRShift": "bcRShift"}


def _compare(path):
    P = build_qd_problem(open(path).read())
    c = inspect_in(path)
    for k, pk in FIELDS.items():
        assert np.allclose(c[k], P[pk], rtol=1e-15, atol=0), k
    eta = np.sqrt(np.abs(P["mu_f"] * P["rho_f"])) / P["faultTypeScale"]
    assert np.allclose(c["eta"], eta, rtol=1e-15, atol=0)
    d = P["domain"]
    g = c["grid"]
    assert (g["order"], g["Ny"], g["Nz"], g["Ly"], g["Lz"]) == (d["order"], d["Ny"], d["Nz"], d["Ly"], d["Lz"])
    assert g["grid_type"] == (0 if d["gridSpacingType"] == "constantGridSpacing" else 1)
    bc = P["bc"]
    assert [g["bcR"], g["bcT"], g["bcL"], g["bcB"]] == [S.BC[bc[k]] for k in "RTLB"]
    s = P["driver"]
    o = c["ode"]
    assert o["method"] == {"RK32": 0, "RK43": 1}[s["timeIntegrator"]]
    assert (o["tol"], o["max_dt"], o["init_dt"], o["t0"], o["t1"]) == \
        (s["timeStepTol"], s["maxDeltaT"], s["initDeltaT"], s["initTime"], s["maxTime"])
    assert o["max_steps"] == s["maxStepCount"]
    assert o["err_keys"] == [{"psi": 0, "slip": 1}[k] for k in s["timeIntInds"]]
    assert c["guess_ss"] == s["guessSteadyStateICs"]
    assert c["fault_type_scale"] == P["faultTypeScale"]
    return c, P


def test_loader_constant_grid(tmp_path):
    _compare(make_qd_problem(str(tmp_path), Ny=41, Nz=37, years=5))


def test_loader_stretched_grid_with_files(tmp_path):
    c, P = _compare(make_qd_problem(str(tmp_path), Ny=33, Nz=45, grid="variableGridSpacing", state_law="slipLaw",
                                    stretch_beta=2.0, dc_lognormal=True, integrator="RK43"))
    assert c["state_law"] == 1
    assert np.ptp(c["Dc"]) > 0   # the per-node Dc file was read


def test_loader_reference_example_ex2(tmp_path):
    p = tmp_path / "ex2.in"
    p.write_text(ex2_text())
    c, P = _compare(str(p))
    assert c["guess_ss"] == 1 and c["ode"]["method"] == 1
    assert c["grid"]["grid_type"] == 1


def test_loader_rejects_out_of_path_inputs(tmp_path):
    p = make_qd_problem(str(tmp_path), Ny=21, Nz=21)
    text = open(p).read()
    for bad in ("momentumBalanceType = quasidynamic_and_dynamic", "timeIntegrator = RK32_WBE",
                "bulkDeformationType = powerLaw", "stateLaw = flashHeating"):
        q = tmp_path / "bad.in"
        q.write_text(text + bad + "\n")
        with pytest.raises(S.ScyError):
            inspect_in(str(q))


def test_loader_rejects_truncated_binary(tmp_path):
    p = make_qd_problem(str(tmp_path), Ny=21, Nz=21)
    psi = [l for l in open(p) if l.startswith("inputDir")][0].split(" = ")[1].strip() + "psi"
    data = open(psi, "rb").read()
    open(psi, "wb").write(data[:-8])
    with pytest.raises(S.ScyError):
        inspect_in(p)


def test_pl_ensemble_files_load(tmp_path):
    """The power-law ensemble writes one loadable input per instance: sizes
    in thirds, b perturbed around the depth profile by about 0.002, and a
    geotherm gradient per instance."""
    from scycle_b200.configs import pl_ensemble_c3
    from scycle_b200.qd import inspect_in
    paths = pl_ensemble_c3(str(tmp_path), n_inst=6, sizes=(33, 41))
    assert len(paths) == 6
    sizes, dev, grads = [], [], set()
    for p in paths:
        info = inspect_in(p, fields=("b",))
        sizes.append(info["grid"]["Ny"])
        z = np.arange(info["grid"]["Nz"]) / (info["grid"]["Nz"] - 1.0) * 30.0
        dev.append(info["b"] - np.interp(z, [0, 12, 17, 30], [0.015, 0.015, 0.005, 0.005]))
        txt = open(p).read()
        assert "bulkDeformationType = powerLaw" in txt
        grads.add([l for l in txt.splitlines() if l.startswith("TVals")][0])
    assert sizes == [33, 33, 33, 41, 41, 41]
    assert 0.0005 < np.std(np.concatenate(dev)) < 0.005
    assert len(grads) == 6
