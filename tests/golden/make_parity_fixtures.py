"""Generates the long-horizon parity fixtures tests/golden/parity_*.npz.

For each workload the oracle (oracle/qd.py: the CPU restatement of
StrikeSlip_LinearElastic_qd with a SuperLU direct solve) integrates the
seeded input free-running, recording every RK attempt (step size, accept
decision) and the fault state after selected accepted steps.  The GPU parity
tests force the device driver onto the same attempt sequence (north star:
identical inputs and an identical forced step sequence) and compare slip,
slip velocity, state, shear stress and surface displacement at those steps.

Workloads (inputs from scycle_b200/configs.py, seed 0):
  c0  aging_const_101: 101x101 constant grid, aging law, RK32, the whole
      200-year run (it ends after 805 steps: with no steady-state start the
      fault stays locked, V below 1e-30 m/s)
  c1  slip_var_401: 401x401 stretched grid, slip law, lognormal Dc,
      steady-state start, RK32, 100 steps (the benchmark's instance 0)
  c4  adjoint_c4: 201x201, aging law, steady-state start, 2000 RK32 steps of
      at most 1e4 s (the adjoint workload's forward run)

Beside the trajectory each fixture holds the oracle's own spread at
rounding level (spread_<field>): the same attempts replayed with the plain
direct solve instead of the refined one.  The fault stress is a
near-cancelling difference of displacements across the finest cell, so
FP64 rounding in u alone moves it by about 1e-11 relative, and the slip
velocity, exponential in the stress, by about 1e-9; two FP64 solutions
that differ only in rounding drift apart at that rate.

    python tests/golden/make_parity_fixtures.py [c0 c1 c4]
"""
import os
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.problem import build_qd_problem  # noqa: E402
from oracle.qd import QDLinearElastic  # noqa: E402
from scycle_b200 import configs  # noqa: E402

FIELDS = ("slip", "slipVel", "psi", "tauP", "tauQSP", "surfDisp")

WORKLOADS = {
    "c0": dict(steps=2000, snaps=(1, 10, 100, 200, 400, 600, 800),
               make=lambda w: configs.aging_const_101(w, seed=0)),
    "c1": dict(steps=100, snaps=(1, 10, 50, 100),
               make=lambda w: configs.slip_var_401(w, seed=0, Ny=401, Nz=401, years=1.0e4)),
    "c4": dict(steps=2000, snaps=(1, 10, 100, 500, 1000, 2000),
               make=lambda w: configs.adjoint_c4(w, seed=0)[0]),
}


def make(name):
    spec = WORKLOADS[name]
    work = tempfile.mkdtemp(prefix="scy_fix_")
    path = spec["make"](work)
    P = build_qd_problem(open(path).read())
    t0 = time.time()
    # one step of extended-precision refinement per solve: the fixture holds
    # the discrete solution to rounding, not a direct solve's forward error
    ora = QDLinearElastic(P, keep_history=True, refine=1)
    rec = []
    rk = ora.integrate(max_steps=spec["steps"], record=rec)
    el = time.time() - t0
    hist = {h["step"]: h for h in ora.history}
    snaps = sorted(set([s for s in spec["snaps"] if s in hist] + [rk.stepCount]))
    out = {"attempt_dt": np.array([r[0] for r in rec]), "attempt_acc": np.array([int(r[1]) for r in rec], np.int8),
           "snap_steps": np.array(snaps), "snap_t": np.array([hist[s]["t"] for s in snaps]),
           "steps": np.array(rk.stepCount), "stage_evals": np.array(rk.stage_evals),
           "oracle_seconds": np.array(el)}
    for f in FIELDS:
        out[f] = np.array([hist[s][f] for s in snaps])
    # the oracle's own spread at rounding level: the same attempts replayed
    # with the plain direct solve (no refinement), whose solutions differ from
    # the refined ones by rounding only; per field and snapshot, the
    # norm-wise relative difference max|a - b| / max|b|
    t1 = time.time()
    ora2 = QDLinearElastic(P, keep_history=True, refine=0)
    ora2.integrate(max_steps=spec["steps"], replay=rec)
    hist2 = {h["step"]: h for h in ora2.history}
    for f in FIELDS:
        out["spread_" + f] = np.array([np.max(np.abs(hist2[s][f] - hist[s][f])) / max(np.max(np.abs(hist[s][f])), 1e-300)
                                       for s in snaps])
    print("%s: spread run %.1f s; spread at the last snapshot: %s" % (
        name, time.time() - t1, {f: float(out["spread_" + f][-1]) for f in FIELDS}))
    np.savez_compressed(os.path.join(HERE, "parity_%s.npz" % name), **out)
    print("%s: %d steps, %d attempts, t = %.6g s, %.1f s of oracle time" % (name, rk.stepCount, len(rec), rk.currT, el))


if __name__ == "__main__":
    for nm in sys.argv[1:] or sorted(WORKLOADS):
        make(nm)
