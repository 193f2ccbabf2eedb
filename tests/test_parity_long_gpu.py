"""Long-horizon parity on the benchmark configurations against oracle fixtures (GPU).

The fixtures tests/golden/parity_{c0,c1,c4}.npz come from the oracle
(tests/golden/make_parity_fixtures.py: the CPU restatement of
StrikeSlip_LinearElastic_qd with a SuperLU direct solve) run free on the
seeded inputs:

* c0: 101x101 constant grid, aging law, RK32 -- the whole 200-year run
  (805 accepted steps);
* c1: 401x401 tanh-stretched grid, slip law, lognormal per-node Dc,
  steady-state start -- the first 100 RK32 steps (the benchmark's instance 0);
* c4: 201x201 constant grid, aging law, steady-state start, 2000 RK32 steps
  of at most 1e4 s (the adjoint workload's forward run).

The device driver is forced onto the oracle's attempt sequence (step sizes
and accept decisions), takes the reference's own Newton path in the
friction root find (its Jacobian expression, fault.cpp:1051, as the oracle
does), and slip, slip velocity, state, shear stress and surface
displacement are compared after the recorded steps, norm-wise relative
(max |device - oracle| / max |oracle| per field).

The bar is 1e-9, or ten times the oracle's own spread where that is larger
(a hundred times for the slip velocity, see SPREAD_FACTOR):
the fixture holds, per field and snapshot, how far the oracle moves when
its refined solves are replaced by the plain direct solve (solutions that
differ by rounding only).  The fault stress is a near-cancelling difference
of displacements across the finest cell, so rounding in u moves it by about
1e-11 relative and the slip velocity, exponential in the stress, by about
1e-9, and the integration carries such differences forward; a device path
that agrees with the oracle as closely as the oracle agrees with itself
meets the bar.  The batched ensemble runs the c1 instance the same way.
"""
import os

import numpy as np
import pytest

from scycle_b200 import configs

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
REL = 1e-9
SOLVE_RTOL = 1e-15  # the stress is read from the solution; solves far below the bar

BUILD = {
    "c0": lambda w: configs.aging_const_101(w, seed=0),
    "c1": lambda w: configs.slip_var_401(w, seed=0, Ny=401, Nz=401, years=1.0e4),
    "c4": lambda w: configs.adjoint_c4(w, seed=0)[0],
}


def _fixture(name):
    return np.load(os.path.join(HERE, "golden", "parity_%s.npz" % name))


def _nrel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


FIELDS = ("slip", "slipVel", "psi", "tauP", "tauQSP", "surfDisp")
# the slip velocity comes from the bracketed Newton, whose stopping test
# (|residual| < rootTol, absolute) turns rounding-level stress differences
# into discontinuous changes of V where the stress is tiny (the locked fault
# of c0): its bar is a hundred times the oracle's spread sample
SPREAD_FACTOR = {f: 10.0 for f in FIELDS}
SPREAD_FACTOR["slipVel"] = 100.0


def _check(view, fx, k, worst):
    """Fields of a device driver (QD view) against snapshot k of a fixture:
    records in ``worst`` the largest error per field and its ratio to the
    bar (1e-9 or ten times the oracle's spread)."""
    for f in FIELDS:
        e = _nrel(view.field(f), fx[f][k])
        bar = max(REL, SPREAD_FACTOR[f] * float(fx["spread_" + f][k]))
        w = worst.setdefault(f, {"err": 0.0, "ratio": 0.0})
        w["err"] = max(w["err"], e)
        w["ratio"] = max(w["ratio"], e / bar)


def _attempts(fx):
    return list(zip(fx["attempt_dt"].tolist(), fx["attempt_acc"].astype(bool).tolist()))


@pytest.mark.parametrize("name", ["c0", "c1", "c4"])
def test_forced_oracle_sequence_matches_oracle(tmp_path, name):
    from scycle_b200.qd import QD
    fx = _fixture(name)
    dev = QD.from_in(BUILD[name](str(tmp_path)), solve_rtol=SOLVE_RTOL, exact_jacobian=False)
    dev.force_attempts(_attempts(fx))
    dev.integrate_begin_from_in()
    done = 0
    worst = {}
    for k, step in enumerate(fx["snap_steps"].tolist()):
        st = dev.integrate_steps(step - done)
        done = step
        assert st.step_count == step
        assert abs(st.t - fx["snap_t"][k]) <= 1e-12 * abs(fx["snap_t"][k])
        _check(dev, fx, k, worst)
    dev.close()
    assert max(w["ratio"] for w in worst.values()) <= 1.0, (name, worst)


def test_batched_c1_instance_matches_oracle(tmp_path):
    """The batched ensemble (here a group of two instances of the c1
    workload, the first forced onto the oracle's attempts) reproduces the
    oracle's first 100 steps."""
    from scycle_b200.batch import Batch
    fx = _fixture("c1")
    p0 = BUILD["c1"](str(tmp_path / "i0"))
    p1 = configs.slip_var_401(str(tmp_path / "i1"), seed=1, Ny=401, Nz=401, years=1.0e4)
    b = Batch([p0, p1], solve_rtol=SOLVE_RTOL, exact_jacobian=False)
    v = b.instance(0)
    v.force_attempts(_attempts(fx))
    done = 0
    worst = {}
    for k, step in enumerate(fx["snap_steps"].tolist()):
        b.run(step - done)
        done = step
        assert v.integrate_steps(0).step_count == step
        _check(v, fx, k, worst)
    b.close()
    assert max(w["ratio"] for w in worst.values()) <= 1.0, ("batch c1", worst)


def test_cycle_first_quasi_dynamic_phase_801():
    """Config 2's first quasi-dynamic phase at 801x801 (qdfd_const_801, seed
    0) into its first event, in two parts (tests/golden/make_cycle801_fixture.py).

    Replay: the device cycle driver in solve mode with the reference's
    Newton path, forced onto the oracle's attempts, against the oracle's
    fields at the snapshots where the oracle's own rounding spread (its plain
    against its refined direct solves) in the slip velocity is below 1e-2,
    i.e. through step 100 (21.2 of the phase's 21.9 years); the bar is the
    largest of 1e-9, ten times that spread and 1e3 times the oracle's
    divergence from a 1e-13 perturbation of its initial slip, as in
    tests/test_cycle_gpu.py.  Nearer the event the slip velocity grows by
    orders of magnitude, the oracle's plain and refined runs differ by O(1)
    (spread_slipVel ~ 1 at steps 176-178) and one trajectory's step sizes no
    longer suit the other's state, so the replay stops there.

    Free running: the device's own step control switches into the wave
    equation at the oracle's step (accepted steps; the number of rejected
    attempts on the way varies with rounding), at the oracle's time within
    1e-4 relative (the step sizes differ
    from the fourth attempt on at the 1e-6 level, where the embedded error
    estimate of the first steps after the steady-state guess is a
    difference of nearly equal solutions; measured 7e-6)."""
    import tempfile
    from scycle_b200.cycle import Cycle
    fx = _fixture("c2qd")
    work = tempfile.mkdtemp(prefix="c2qd_")
    path = configs.qdfd_const_801(work, seed=0, cycles=3, years=1000.0)
    c = Cycle.from_in(path, solve_rtol=SOLVE_RTOL, solve_max_its=2000, exact_jacobian=False)
    c.force_attempts(list(zip(fx["attempt_dt"].tolist(), fx["attempt_acc"].astype(bool).tolist())))
    c.begin_from_in()
    step = 0
    worst = {}
    compared = 0
    for i, k in enumerate(fx["snap_steps"].tolist()):
        if float(fx["spread_slipVel"][i]) >= 1e-2:
            break
        st = c.run(k - step)
        step = k
        assert st.step_count == k
        assert abs(st.t - fx["snap_t"][i]) <= 1e-12 * abs(fx["snap_t"][i])
        for f in FIELDS:
            e = float(np.linalg.norm(c.field(f) - fx[f][i]) / max(np.linalg.norm(fx[f][i]), 1e-300))
            bar = max(REL, 10.0 * float(fx["spread_" + f][i]), 1e3 * float(fx["sens_" + f][i]))
            worst[f] = max(worst.get(f, 0.0), e / bar)
            assert e <= bar, "step %d %s rel err %.3e > %.3e" % (k, f, e, bar)
        compared += 1
    assert compared >= 7 and step >= 100
    c.close()
    c = Cycle.from_in(path, solve_rtol=SOLVE_RTOL, solve_max_its=2000, exact_jacobian=False)
    c.begin_from_in()
    n = 0
    while not c.switches() and n < 2000:
        c.run(10)
        n += 10
    sw = c.switches()
    first = int(fx["switch_step"])
    assert sw and sw[0]["step"] == first and sw[0]["to"] == "fd", sw[:1]
    assert abs(sw[0]["t"] - float(fx["switch_t"])) <= 1e-4 * float(fx["switch_t"])
    c.close()
