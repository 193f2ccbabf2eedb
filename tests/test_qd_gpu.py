"""Quasi-dynamic d_dt and adaptive RK integration on the device vs the oracle (GPU).

The oracle (oracle/qd.py) restates StrikeSlip_LinearElastic_qd with a direct
sparse solve.  Integration parity replays the device's own attempt sequence
(step sizes and accept decisions) in the oracle, so the PID controller cannot
amplify round-off into different step sequences; tolerance 1e-9 relative on
slip, slip velocity, state, shear stress and surface displacement.
"""
import numpy as np
import pytest

from oracle.problem import build_qd_problem
from oracle.qd import QDLinearElastic
from scycle_b200.configs import make_qd_problem

pytestmark = pytest.mark.gpu

REL = 1e-9
SOLVE_RTOL = 1e-14  # elliptic solves converged far below the parity tolerance


def _rel(a, b, floor=0.0):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), floor + 1e-300)))


def _nrel(a, b):
    """Norm-wise relative difference (for fields that cross zero)."""
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _problem(tmp_path, n=41, law="agingLaw", integrator="RK32", grid="constantGridSpacing", prestress=None, **kw):
    p = make_qd_problem(str(tmp_path), Ny=n, Nz=n, state_law=law, integrator=integrator, grid=grid,
                        stretch_beta=2.0 if grid == "variableGridSpacing" else None, **kw)
    P = build_qd_problem(open(p).read())
    if prestress is not None:
        P["prestress"] = np.full(P["Nz"], prestress) + np.linspace(0, 0.5, P["Nz"])
    return P


@pytest.mark.parametrize("law,grid,prestress,exact", [
    ("agingLaw", "constantGridSpacing", 20.0, True), ("agingLaw", "constantGridSpacing", 26.5, False),
    ("agingLaw", "constantGridSpacing", 26.5, True),
    ("slipLaw", "constantGridSpacing", 28.0, True), ("agingLaw", "variableGridSpacing", 26.5, True),
    ("slipLaw", "variableGridSpacing", 29.0, False)])
def test_d_dt_matches_oracle(tmp_path, law, grid, prestress, exact):
    """exact=False reproduces the reference's Newton derivative and iteration
    path; exact=True converges to the same root in fewer iterations."""
    from scycle_b200.qd import QD
    P = _problem(tmp_path, law=law, grid=grid, prestress=prestress)
    ora = QDLinearElastic(P, keep_history=False)
    dev = QD(P, solve_rtol=SOLVE_RTOL, exact_jacobian=exact)
    rng = np.random.default_rng(3)
    for t in (0.0, 3.0e7, 1.1e9):
        psi = P["psi"] + 1e-3 * rng.standard_normal(P["Nz"])
        slip = 0.05 * rng.random(P["Nz"])
        fo = ora.d_dt(t, {"psi": psi, "slip": slip})
        fd = dev.d_dt(t, psi, slip)
        assert _rel(fd["slip"], fo["slip"], 1e-30) <= REL
        assert _rel(fd["psi"], fo["psi"], 1e-12) <= REL
        for nm, ref in (("tauQSP", ora.fault.tauQSP), ("tauP", ora.fault.tauP), ("strength", ora.fault.strength)):
            assert _rel(dev.field(nm), ref, 1e-9) <= REL, nm
        assert _nrel(dev.field("surfDisp"), ora.u[::P["Nz"]]) <= REL


@pytest.mark.parametrize("law,exact", [("agingLaw", False), ("slipLaw", True)])
def test_fault_d_dt_alone_matches_oracle(tmp_path, law, exact):
    """Fault_qd::d_dt on its own (scy_qd_fault_d_dt): given the body's shear
    stress on the fault, the slip velocity from the friction root, the state
    rate, tauQS, tauP and strength as the oracle's FaultQD.d_dt gives them;
    and with the stress the full d_dt computed, the full d_dt's fault rates."""
    from scycle_b200.qd import QD
    P = _problem(tmp_path, law=law, prestress=26.5)
    ora = QDLinearElastic(P, keep_history=False)
    dev = QD(P, solve_rtol=SOLVE_RTOL, exact_jacobian=exact)
    rng = np.random.default_rng(11)
    Nz = P["Nz"]
    psi = P["psi"] + 1e-3 * rng.standard_normal(Nz)
    slip = 0.05 * rng.random(Nz)
    full = dev.d_dt(2.0e8, psi, slip)
    tau_body = dev.field("sxy")[:Nz]
    alone = dev.fault_d_dt(psi, slip, tau_body)
    assert _rel(alone["slip"], full["slip"], 1e-30) <= 1e-12
    assert _rel(alone["psi"], full["psi"], 1e-12) <= 1e-12
    v_start = dev.field("slipVel")  # the root finds start from the current slip velocity
    tau = tau_body + rng.normal(0.0, 0.05, Nz)  # any stress, not only a solve's
    alone = dev.fault_d_dt(psi, slip, tau)
    f = ora.fault
    f.update_fields({"psi": psi, "slip": slip})
    f.slipVel = v_start.copy()
    V_ref, dpsi_ref = f.d_dt(tau)
    assert _rel(alone["slip"], V_ref, 1e-30) <= REL
    assert _rel(alone["psi"], dpsi_ref, 1e-12) <= REL
    for nm, r in (("tauQSP", f.tauQSP), ("tauP", f.tauP), ("strength", f.strength)):
        assert _rel(dev.field(nm), r, 1e-9) <= REL, nm


@pytest.mark.parametrize("integrator,law,steps", [("RK32", "agingLaw", 60), ("RK43", "slipLaw", 30)])
def test_integrate_replay_matches_oracle(tmp_path, integrator, law, steps):
    from scycle_b200.qd import QD
    P = _problem(tmp_path, n=33, law=law, integrator=integrator, prestress=26.0)
    dev = QD(P, solve_rtol=SOLVE_RTOL)
    ora = QDLinearElastic(P, keep_history=False)
    dev.record_attempts(True)
    dev.integrate_begin(ora.min_dt, max_steps=steps)
    st = dev.integrate_steps(steps)
    att = dev.attempts()
    rk = ora.integrate(max_steps=steps, replay=att)
    assert st.step_count == rk.stepCount == steps
    assert abs(st.t - rk.currT) <= 1e-12 * abs(rk.currT)
    f = ora.fault
    assert _rel(dev.field("slip"), f.slip, 1e-12) <= REL
    assert _rel(dev.field("psi"), f.psi) <= REL
    assert _rel(dev.field("slipVel"), f.slipVel, 1e-30) <= REL
    assert _rel(dev.field("tauP"), f.tauP, 1e-9) <= REL
    assert _nrel(dev.field("surfDisp"), ora.u[::P["Nz"]]) <= REL


def test_integrate_free_running_matches_oracle_decisions(tmp_path):
    """Without replay the device takes the same accept/reject decisions as the oracle."""
    from scycle_b200.qd import QD
    P = _problem(tmp_path, n=25, prestress=26.0)
    dev = QD(P, solve_rtol=SOLVE_RTOL)
    ora = QDLinearElastic(P, keep_history=False)
    dev.record_attempts(True)
    dev.integrate_begin(ora.min_dt, max_steps=40)
    dev.integrate_steps(40)
    rec = []
    ora.integrate(max_steps=40, record=rec)
    att = dev.attempts()
    assert [a[1] for a in att] == [r[1] for r in rec]
    # step sizes follow from the embedded error estimate, a difference of two
    # nearly equal solutions, so they agree to fewer digits than the states
    assert np.allclose([a[0] for a in att], [r[0] for r in rec], rtol=1e-6, atol=0)


def _ex2_like(tmp_path, n=41, integrator="RK43"):
    from tests.test_oracle import ex2_text
    text = ex2_text().replace("Ny = 151", "Ny = %d" % n).replace("Nz = 151", "Nz = %d" % n)
    text = text.replace("timeIntegrator = RK43", "timeIntegrator = %s" % integrator)
    p = tmp_path / "ex2_small.in"
    p.write_text(text + "stride1D = 0\nstride2D = 0\n")
    return str(p)


@pytest.mark.parametrize("integrator", ["RK43", "RK32"])
def test_reference_example_from_input_file(tmp_path, integrator):
    """The reference's examples/ex2.in settings (steady-state initial guess,
    stretched grid, aging law) on a 41x41 grid, loaded by the C++ reader."""
    from scycle_b200.qd import QD
    path = _ex2_like(tmp_path, integrator=integrator)
    P = build_qd_problem(open(path).read())
    ora = QDLinearElastic(P, keep_history=False)
    dev = QD.from_in(path, solve_rtol=SOLVE_RTOL)
    dev.record_attempts(True)
    dev.integrate_begin_from_in()
    st = dev.integrate_steps(25)
    rk = ora.integrate(max_steps=25, replay=dev.attempts())
    assert st.step_count == rk.stepCount == 25
    f = ora.fault
    assert _rel(dev.field("slip"), f.slip, 1e-12) <= REL
    assert _rel(dev.field("psi"), f.psi) <= REL
    assert _rel(dev.field("slipVel"), f.slipVel, 1e-30) <= REL
    assert _rel(dev.field("tauP"), f.tauP, 1e-9) <= REL
    assert _nrel(dev.field("surfDisp"), ora.u[::P["Nz"]]) <= REL


@pytest.mark.parametrize("integrator", ["RK32", "RK43"])
def test_response_mode_matches_oracle(tmp_path, integrator):
    """Fault stress from the precomputed discrete fault response (Nz + 2
    solves) instead of a solve per stage: same states as the oracle's direct
    solves to the parity tolerance."""
    from scycle_b200.qd import QD
    path = _ex2_like(tmp_path, n=33, integrator=integrator)
    P = build_qd_problem(open(path).read())
    ora = QDLinearElastic(P, keep_history=False)
    dev = QD.from_in(path, solve_rtol=SOLVE_RTOL)
    dev.set_mode("response")
    dev.record_attempts(True)
    dev.integrate_begin_from_in()
    st = dev.integrate_steps(30)
    rk = ora.integrate(max_steps=30, replay=dev.attempts())
    assert st.step_count == rk.stepCount == 30
    f = ora.fault
    assert _rel(dev.field("slip"), f.slip, 1e-12) <= REL
    assert _rel(dev.field("psi"), f.psi) <= REL
    assert _rel(dev.field("slipVel"), f.slipVel, 1e-30) <= REL
    assert _rel(dev.field("tauP"), f.tauP, 1e-9) <= REL
    assert _nrel(dev.field("surfDisp"), ora.u[::P["Nz"]]) <= REL
    assert _nrel(dev.field("u"), ora.u) <= REL


def test_response_mode_d_dt_matches_solve_mode(tmp_path):
    from scycle_b200.qd import QD
    P = _problem(tmp_path, n=45, law="slipLaw", grid="variableGridSpacing", prestress=27.0)
    a = QD(P, solve_rtol=SOLVE_RTOL)
    b = QD(P, solve_rtol=SOLVE_RTOL)
    b.set_mode("response")
    rng = np.random.default_rng(11)
    for t in (0.0, 5.0e8):
        psi = P["psi"] + 1e-3 * rng.standard_normal(P["Nz"])
        slip = 0.05 * rng.random(P["Nz"])
        fa, fb = a.d_dt(t, psi, slip), b.d_dt(t, psi, slip)
        assert _rel(fb["slip"], fa["slip"], 1e-30) <= REL
        assert _rel(fb["psi"], fa["psi"], 1e-12) <= REL
        assert _rel(b.field("tauQSP"), a.field("tauQSP"), 1e-9) <= REL
