"""Quasi-dynamic / fully dynamic cycles on the GPU against the oracle.

The oracle (oracle/qdfd.py) restates strikeSlip_linearElastic_qd_fd; the GPU
driver runs the same input file through scy_cycle_*.

Earthquake nucleation is an instability: a relative difference d in the
state grows roughly like the slip velocity itself (from 1e-9 to 1 m/s), so
two correct FP64 implementations that start 1e-13 apart end an event about
1e-3 apart (the oracle shows this against itself, see
``_oracle_sensitivity``).  The parity gates are therefore:

* wave-equation phases restarted from the oracle's state (scy_cycle_set_fd_state)
  match step by step to 1e-9 and switch back at the same step;
* quasi-dynamic phases replaying the oracle's attempt sequence stay within
  1e3 times the oracle's own divergence from a 1e-13 perturbation (and within
  1e-9 while that is smaller), and switch to the wave equation at the same step;
* free-running event times agree within 1% (event recurrence).
"""
import numpy as np
import pytest

from scycle_b200.configs import make_qdfd_problem
from oracle.qdfd import build_qdfd_problem, QDFDLinearElastic

pytestmark = pytest.mark.gpu

REL = 1e-9
FIELDS = ("slip", "slipVel", "psi", "tauP", "tauQSP", "surfDisp")


def _nrel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _oracle(path, stop_at=None, replay=None, perturb=0.0, snapshots=None):
    P = build_qdfd_problem(open(path).read())
    m = QDFDLinearElastic(P)
    if perturb:
        orig = m.solve_ss
        m.solve_ss = lambda: orig() * (1.0 + perturb)
    if snapshots is not None:
        def snap(mm, var, prev):
            f = mm.ffd
            snapshots.append(dict(t=mm.currTime, step=mm.stepCount, allowed=mm.allowed,
                                  var={k: v.copy() for k, v in var.items()},
                                  prev={k: v.copy() for k, v in prev.items()},
                                  u0=mm.u0.copy(), slip0=f.slip0.copy(), tau0=f.tau0.copy(),
                                  slipVel=f.slipVel.copy()))
        m.on_fd_start = snap
    rec = []
    m.integrate_cycles(record=rec, replay=replay, stop_at_step=stop_at)
    return m, rec, {h["step"]: h for h in m.history}


def _gpu(path, rec=None, batch=None, mode=None):
    from scycle_b200.cycle import Cycle
    c = Cycle.from_in(path, solve_rtol=1e-14, solve_max_its=2000)
    if rec is not None:
        c.force_attempts(rec)
    if batch:
        c.set_fd_batch(batch)
    if mode:
        c.set_mode(mode)
    c.begin_from_in()
    return c


def _compare(c, h, tag, bound=None):
    for f in FIELDS:
        e = _nrel(c.field(f), h[f])
        b = REL if bound is None else bound[f]
        assert e <= b, "%s %s rel err %.3e > %.3e" % (tag, f, e, b)


@pytest.fixture(scope="module")
def three_cycles(tmp_path_factory):
    """41x41 constant grid, P step control, leaving the wave equation once R
    falls below 1e-3 after passing 0.01: three full cycles in ~360 steps."""
    d = tmp_path_factory.mktemp("cyc3")
    path = make_qdfd_problem(str(d), Ny=41, Nz=41, cycles=3, years=1000.0,
                             extra={"limit_fd": "0.01", "timeControlType": "P"})
    snaps = []
    m, rec, hist = _oracle(path, snapshots=snaps)
    return path, m, rec, hist, snaps


def _fd_phase_check(path, m, hist, snap, n_max=None, every=1):
    """Restart the GPU at the oracle's state at the start of a wave phase
    and compare every `every`-th step until the oracle leaves the phase."""
    c = _gpu(path)
    c.set_fd_state(snap["t"], snap["step"], snap["allowed"], snap["var"], snap["prev"], snap["u0"],
                   snap["slip0"], snap["tau0"], snap["slipVel"])
    k0 = snap["step"]
    end = [s["step"] for s in m.switches if s["to"] == "qd" and s["step"] > k0]
    last = end[0] if end else max(hist)
    if n_max:
        last = min(last, k0 + n_max)
    step = k0
    for k in range(k0 + 1, last + 1):
        if (k - k0) % every and k != last:
            continue
        st = c.run(k - step)
        step = k
        assert st.step_count == k
        assert abs(st.t - hist[k]["t"]) <= 1e-12 * abs(hist[k]["t"])
        assert hist[k]["phase"] == "fd"
        _compare(c, hist[k], "wave step %d" % k)
    if end and end[0] == last:
        sw = c.switches()
        assert sw and sw[-1]["step"] == last and sw[-1]["to"] == "qd"
    return c


def test_cycle_wave_phases_restarted(three_cycles):
    path, m, rec, hist, snaps = three_cycles
    assert [s["to"] for s in m.switches] == ["fd", "qd"] * 3
    assert len(snaps) == 3
    for snap in snaps:
        _fd_phase_check(path, m, hist, snap)


def test_cycle_wave_phase_variable_grid(tmp_path):
    """Stretched grid: the wave update carries Jinv, the fault stress qy."""
    path = make_qdfd_problem(str(tmp_path), Ny=41, Nz=37, cycles=2, years=1000.0, grid="variableGridSpacing",
                             stretch_beta=1.5, extra={"limit_fd": "0.01", "timeControlType": "P"})
    snaps = []
    m, rec, hist = _oracle(path, stop_at=200, snapshots=snaps)
    assert snaps
    _fd_phase_check(path, m, hist, snaps[0])


def test_cycle_long_wave_phase(tmp_path):
    """61x61: the first event never reaches limit_fd, so the wave phase runs
    on; 1500 steps compared every 50."""
    path = make_qdfd_problem(str(tmp_path), Ny=61, Nz=61, cycles=2, years=1000.0)
    snaps = []
    m, rec, hist = _oracle(path, stop_at=116 + 1500, snapshots=snaps)
    assert snaps and len(m.switches) == 1
    _fd_phase_check(path, m, hist, snaps[0], n_max=1500, every=50)


def _oracle_sensitivity(path, rec, ref_hist, stop_at):
    """The oracle's own divergence (per step and field) when its steady-state
    initial slip is perturbed by 1e-13 and the same attempts are replayed."""
    _, _, h1 = _oracle(path, stop_at=stop_at, replay=rec, perturb=1e-13)
    return {k: {f: _nrel(h1[k][f], ref_hist[k][f]) for f in FIELDS} for k in ref_hist if k in h1}


def test_cycle_quasi_dynamic_replay(three_cycles):
    """Replaying the oracle's attempts from the start: within 1e3 x the
    oracle's own sensitivity (>= 1e-9), same switch step into the first
    event."""
    path, m, rec, hist, snaps = three_cycles
    first = m.switches[0]["step"]
    sens = _oracle_sensitivity(path, rec, hist, first + 1)
    c = _gpu(path, rec)
    step = 0
    for k in sorted(set([1, 2, 5, 10, 20, 40, 60, 80, first - 1, first, first + 1])):
        st = c.run(k - step)
        step = k
        assert st.step_count == k
        bound = {f: max(REL, 1e3 * sens[k][f]) for f in FIELDS}
        _compare(c, hist[k], "step %d" % k, bound)
    sw = c.switches()
    assert sw[0]["step"] == first and sw[0]["to"] == "fd"
    assert abs(sw[0]["t"] - m.switches[0]["t"]) <= 1e-12 * m.switches[0]["t"]


def _event_times(switches):
    return [s["t"] for s in switches if s["to"] == "fd"]


@pytest.mark.parametrize("mode", ["solve", "response"])
def test_cycle_event_recurrence_free_running(three_cycles, mode):
    """Both integrators choose their own steps: the three events start at the
    oracle's times within 1% of the recurrence interval."""
    path, m, rec, hist, snaps = three_cycles
    c = _gpu(path, mode=mode)
    st = c.run(10 ** 6)
    assert st.done == 1
    assert st.cycle_count == m.cycleCount
    to = _event_times(m.switches)
    tg = _event_times(c.switches())
    assert len(tg) == len(to) == 3
    assert abs(tg[0] - to[0]) <= 1e-6 * to[0]
    for i in range(1, 3):
        ro, rg = to[i] - to[i - 1], tg[i] - tg[i - 1]
        assert abs(rg - ro) <= 0.01 * ro, (i, rg, ro)


def test_cycle_graph_batch_invariance(three_cycles):
    """Results do not depend on how many wave steps one graph launch holds."""
    path, m, rec, hist, snaps = three_cycles
    snap = snaps[0]
    out = {}
    for batch in (1, 7, 64):
        c = _gpu(path, batch=batch)
        c.set_fd_state(snap["t"], snap["step"], snap["allowed"], snap["var"], snap["prev"], snap["u0"],
                       snap["slip0"], snap["tau0"], snap["slipVel"])
        st = c.run(11)
        assert st.step_count == snap["step"] + 11
        out[batch] = {f: c.field(f) for f in FIELDS + ("u",)}
    for f in out[1]:
        assert np.array_equal(out[1][f], out[7][f]), f
        assert np.array_equal(out[1][f], out[64][f]), f


def test_cycle_fused_step_matches_two_launches(three_cycles):
    """The fused wave + fault launch gives bitwise the results of the
    two-launch form, through the switch back to the quasi-dynamic phase."""
    path, m, rec, hist, snaps = three_cycles
    snap = snaps[0]
    out = {}
    for fused in (True, False):
        c = _gpu(path)
        c.set_fd_fused(fused)
        c.set_fd_state(snap["t"], snap["step"], snap["allowed"], snap["var"], snap["prev"], snap["u0"],
                       snap["slip0"], snap["tau0"], snap["slipVel"])
        end = [s["step"] for s in m.switches if s["to"] == "qd" and s["step"] > snap["step"]][0]
        st = c.run(end - snap["step"])
        assert st.step_count == end and c.switches()[-1]["step"] == end
        out[fused] = {f: c.field(f) for f in FIELDS + ("u",)}
    for f in out[True]:
        assert np.array_equal(out[True][f], out[False][f]), f


def test_cycle_pid_restart_rule(tmp_path):
    """PID control: each phase starts a fresh integrator with no error
    history, so past step 4 its first step-size update is 0 * inf = NaN and
    the 5x growth cap decides (first quasi-dynamic step after the return from
    the wave equation)."""
    path = make_qdfd_problem(str(tmp_path), Ny=41, Nz=41, cycles=3, years=1000.0, extra={"limit_fd": "0.01"})
    m, rec, hist = _oracle(path, stop_at=126)
    back = [s for s in m.switches if s["to"] == "qd"]
    assert back and back[0]["step"] == 125
    h = hist[126]
    assert h["new_dt"] == pytest.approx(5 * h["dt"], rel=1e-15)
    c = _gpu(path, rec)
    st = c.run(125)
    assert st.step_count == 125
    if c.switches()[-1]["step"] == 125:  # the GPU left the wave phase at the same step
        st = c.run(1)
        assert st.step_count == 126 and st.phase == 0
        assert st.new_dt == pytest.approx(5 * st.dt, rel=1e-15)
