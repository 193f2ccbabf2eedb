"""Power-law viscoelastic quasi-dynamic driver on the GPU vs the oracle.

The oracle (oracle/powerlaw.py) restates StrikeSlip_PowerLaw_qd with
PowerLaw's dislocation creep.  The GPU driver reads the same input file
(bulkDeformationType = powerLaw) through scy_qd_create_from_in.  d_dt is
compared at states with nonzero viscous strain, then adaptive RK43 runs with
the oracle replaying the device's attempt sequence; tolerance 1e-9 relative
(norm-wise) on every integrated and derived field.
"""
import numpy as np
import pytest

from oracle.powerlaw import PowerLawQD, build_pl_problem
from scycle_b200.configs import make_pl_problem

pytestmark = pytest.mark.gpu

REL = 1e-9


def _nrel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _problem(tmp_path, grid="constantGridSpacing", n=41, nz=37, **kw):
    extra = {"maxDeltaT": "1e6"}
    extra.update(kw.pop("extra", {}))
    args = dict(Ny=n, Nz=nz, grid=grid, extra=extra)
    if grid == "variableGridSpacing":
        args["stretch_beta"] = 1.5
    args.update(kw)
    return make_pl_problem(str(tmp_path), **args)


def _device(path):
    from scycle_b200.qd import QD
    return QD.from_in(path, solve_rtol=1e-14, solve_max_its=2000)


@pytest.mark.parametrize("grid", ["constantGridSpacing", "variableGridSpacing"])
def test_pl_d_dt_matches_oracle(tmp_path, grid):
    path = _problem(tmp_path, grid)
    P = build_pl_problem(open(path).read())
    ora = PowerLawQD(P, keep_history=False)
    dev = _device(path)
    assert dev.state_size() == 2 * dev.N + 2 * dev.Nz
    rng = np.random.default_rng(5)
    N, Nz = dev.N, dev.Nz
    var = ora.initiate_integrand()
    # a state with viscous strain and a loaded fault
    var["gVxy"] = rng.normal(0, 1e-4, N)
    var["gVxz"] = rng.normal(0, 1e-4, N)
    var["slip"] = var["slip"] + np.linspace(0.0, 2.0, Nz)
    t = 3.0e8
    ref = ora.d_dt(t, {k: v.copy() for k, v in var.items()})
    vec = np.concatenate([var["gVxy"], var["gVxz"], var["psi"], var["slip"]])
    from scycle_b200 import _lib as S
    dev.integrate_begin_from_in()
    S.check(S.lib().scy_qd_set_state(dev.h, S.as_dptr(np.ascontiguousarray(vec)), 0))
    import ctypes as C
    import torch
    v = torch.from_numpy(vec).cuda()
    out = torch.empty_like(v)
    torch.cuda.synchronize()
    S.check(S.lib().scy_qd_d_dt(dev.h, t, C.c_void_p(v.data_ptr()), C.c_void_p(out.data_ptr())))
    o = out.cpu().numpy()
    got = {"gVxy": o[:N], "gVxz": o[N:2 * N], "psi": o[2 * N:2 * N + Nz], "slip": o[2 * N + Nz:]}
    for k in ("gVxy", "gVxz", "psi", "slip"):
        assert _nrel(got[k], ref[k]) <= REL, k
    assert _nrel(dev.field("sdev"), ora.sdev) <= REL
    assert _nrel(dev.field("effVisc"), ora.effVisc) <= REL
    assert _nrel(dev.field("sxy"), ora.sxy) <= REL
    assert _nrel(dev.field("sxz"), ora.sxz) <= REL
    assert _nrel(dev.field("tauP"), ora.fault.tauP) <= REL


@pytest.mark.parametrize("grid,control", [("constantGridSpacing", "PID"), ("variableGridSpacing", "P")])
def test_pl_integrate_replay_matches_oracle(tmp_path, grid, control):
    """RK43 over 80 steps (viscous strains growing from zero)."""
    path = _problem(tmp_path, grid, extra={"timeControlType": control})
    dev = _device(path)
    dev.record_attempts(True)
    dev.integrate_begin_from_in()
    st = dev.integrate_steps(80)
    att = dev.attempts()
    P = build_pl_problem(open(path).read())
    ora = PowerLawQD(P)
    rk = ora.integrate(max_steps=80, replay=att)
    assert st.step_count == rk.stepCount == 80
    assert abs(st.t - rk.currT) <= 1e-12 * rk.currT
    h = ora.history[-1]
    for k in ("gVxy", "psi", "slip", "slipVel", "tauP"):
        assert _nrel(dev.field(k), h[k]) <= REL, k
    # gVxz grows from sxz = mu (Dz u - gVxz), which cancels where u hardly
    # varies in z; its error is measured against the viscous strain's size
    gz = dev.field("gVxz")
    assert np.linalg.norm(gz - h["gVxz"]) <= REL * max(np.linalg.norm(h["gVxz"]), np.linalg.norm(h["gVxy"]))
    assert _nrel(dev.field("sdev"), h["sdev"]) <= REL
    assert _nrel(dev.field("surfDisp"), h["surfDisp"]) <= REL
    assert np.abs(dev.field("gVxy")).max() > 0


def test_pl_free_running_decisions(tmp_path):
    """Without replay both controllers take the same accept/reject decisions
    and step sizes (to the error estimate's round-off)."""
    path = _problem(tmp_path)
    dev = _device(path)
    dev.record_attempts(True)
    dev.integrate_begin_from_in()
    dev.integrate_steps(40)
    att = dev.attempts()
    P = build_pl_problem(open(path).read())
    ora = PowerLawQD(P, keep_history=False)
    rec = []
    ora.integrate(max_steps=40, record=rec)
    assert [a for _, a in att] == [a for _, a in rec]
    assert np.allclose([d for d, _ in att], [d for d, _ in rec], rtol=1e-6)


@pytest.mark.parametrize("grid", ["constantGridSpacing", "variableGridSpacing"])
def test_pl_steady_state_guess_matches_oracle(tmp_path, grid):
    """guessSteadyStateICs = 1 with the power-law material: the
    effective-viscosity iteration (an operator with mu = effVisc built for
    every iteration, solved and differentiated on the device, damped in
    log10) gives the oracle's initial state (viscous strains -sxy/mu at
    initTime 0, steady-state psi, zero slip) and the same first rates.
    With a viscosity cap of 1e12 GPa s the operator's contrast is about five
    decades and the oracle's answer is stable to rounding, so the bar is
    1e-8."""
    path = _problem(tmp_path, grid, n=25, nz=25, extra={"guessSteadyStateICs": "1", "maxEffVisc": "1e12"})
    P = build_pl_problem(open(path).read())
    ora = PowerLawQD(P, keep_history=False)
    var = ora.initiate_integrand()
    assert 1 < ora.ss_its < P["ss"]["maxSSIts_effVisc"]
    dev = _device(path)
    dev.integrate_begin_from_in()
    for nm in ("gVxy", "gVxz", "psi", "slip"):
        assert _nrel(dev.field(nm), var[nm]) <= 1e-8, nm
    d0 = ora.d_dt(P["driver"]["initTime"], {k: v.copy() for k, v in var.items()})
    assert _nrel(dev.field("slipVel"), d0["slip"]) <= 1e-8
    assert _nrel(dev.field("tauP"), ora.fault.tauP) <= 1e-8


@pytest.mark.parametrize("grid,n", [("constantGridSpacing", 25), ("variableGridSpacing", 25),
                                    ("constantGridSpacing", 61)])
def test_pl_steady_state_guess_at_the_default_viscosity_cap(tmp_path, grid, n):
    """guessSteadyStateICs = 1 at the reference's default cap maxEffVisc =
    1e30 (powerLaw.cpp:757): the effective viscosity spans about fourteen
    decades and is far from a product a(y) b(z), and the steady velocity is
    ill-conditioned enough that the oracle's own answer moves between plain
    and refined direct solves (its spread).  The device (block Cholesky
    factorisation of every iteration's operator with defect correction from
    double-double residuals) must land within ten times that spread of the
    oracle, with the same number of viscosity iterations give or take one
    (the stopping test compares a relative change with 1e-3)."""
    path = _problem(tmp_path, grid, n=n, nz=n, extra={"guessSteadyStateICs": "1", "maxEffVisc": "1e30"})
    P = build_pl_problem(open(path).read())
    runs = []
    for refine in (0, 2):
        o = PowerLawQD(P, keep_history=False, refine=refine)
        var = o.initiate_integrand()
        d0 = o.d_dt(P["driver"]["initTime"], {k: v.copy() for k, v in var.items()})
        runs.append((o, dict(var, slipVel=d0["slip"], tauP=o.fault.tauP.copy())))
    (ora, ref), (_, fine) = runs
    assert ora.effVisc.max() / ora.effVisc.min() > 1e12
    dev = _device(path)
    dev.integrate_begin_from_in()
    its, err, cg = dev.steady_state_info()
    assert abs(its - ora.ss_its) <= 1, (its, ora.ss_its)
    assert err < P["ss"]["atolSS_effVisc"]
    tr = dev.steady_state_trace()
    assert tr.shape == (its, 5) and np.all(tr[:, 0] >= 1)  # every iteration corrected its velocity
    assert np.all(tr[:, 2] <= 1e-12)  # to the solve tolerance (relative, double-double residual)
    for nm in ("gVxy", "gVxz", "psi", "slip", "slipVel", "tauP"):
        spread = _nrel(fine[nm], ref[nm])
        e = _nrel(dev.field(nm), ref[nm])
        assert e <= max(1e-8, 10.0 * spread), (nm, e, spread)
