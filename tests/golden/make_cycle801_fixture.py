"""Generates tests/golden/parity_c2qd.npz: the first quasi-dynamic phase of
the 801x801 cycle workload (qdfd_const_801, seed 0: order-4 constant grid
over 30 km, aging law, RK43, steady-state start, switch to the wave equation
when max(eta V / tau) passes 1e-3) up to and including the switch into the
first event.

The oracle (oracle/qdfd.py: the CPU restatement of
strikeSlip_linearElastic_qd_fd with a SuperLU direct solve) integrates the
phase free-running, recording every RK attempt (step size, accept decision)
and the fault and surface fields after selected steps; its run stops when
the wave-equation phase would begin (after the single quasi-dynamic step of
size deltaT_fd that prepares it).  The GPU test forces the device cycle
driver onto the same attempts and compares the fields at those steps and
the switch step.

Beside the trajectory the fixture holds two measures of the oracle's own
uncertainty.  sens_<field>: the same attempts replayed with the
steady-state initial slip perturbed by 1e-13; nucleation amplifies such a
perturbation roughly like the slip velocity grows, so near the switch two
correct FP64 implementations differ far above rounding.  spread_<field>:
the same attempts replayed with every direct solve refined once in
extended precision; the fault stress is a near-cancelling difference of
displacements across the finest cell (37.5 m here), so FP64 rounding in u
moves the slip velocity by about 1e-8 relative at this size.  The test's
bar is the largest of 1e-9, ten times the spread and 1e3 times the
sensitivity (as in tests/test_cycle_gpu.py and tests/golden/parity_*.npz).

SuperLU factorises the 641,601-unknown operator once (about a minute, 4 GB)
and takes about half a second per solve; the phase and its two replays take
about fifty minutes on one core.

    python tests/golden/make_cycle801_fixture.py
"""
import os
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.qdfd import build_qdfd_problem, QDFDLinearElastic  # noqa: E402
from scycle_b200.configs import qdfd_const_801  # noqa: E402

FIELDS = ("slip", "slipVel", "psi", "tauP", "tauQSP", "surfDisp")


class _FirstPhase(QDFDLinearElastic):
    """The driver stopped where its first wave-equation phase would start."""

    def integrate_fd(self):
        self.hard_stop = True


def _run(path, replay=None, perturb=0.0, refine=0):
    P = build_qdfd_problem(open(path).read())
    m = _FirstPhase(P, refine=refine)
    if perturb:
        orig = m.solve_ss
        m.solve_ss = lambda: orig() * (1.0 + perturb)
    rec = []
    m.integrate_cycles(record=rec, replay=replay)
    return m, rec, {h["step"]: h for h in m.history}


def main():
    work = tempfile.mkdtemp(prefix="c2qd_")
    path = qdfd_const_801(work, seed=0, cycles=3, years=1000.0)
    t0 = time.time()
    m, rec, hist = _run(path)
    first = m.switches[0]["step"]
    print("oracle: switch to the wave equation at step %d (t = %.6e s), %d attempts, %.0f s"
          % (first, m.switches[0]["t"], len(rec), time.time() - t0), flush=True)
    snaps = sorted(set([1, 2, 5, 10, 20, 50, 100] + list(range(200, first, 100)) + [first - 1, first, first + 1]))
    snaps = [k for k in snaps if k in hist]
    t0 = time.time()
    _, _, h1 = _run(path, replay=rec, perturb=1e-13)
    print("perturbed replay: %.0f s" % (time.time() - t0), flush=True)
    t0 = time.time()
    _, _, h2 = _run(path, replay=rec, refine=1)
    print("refined replay: %.0f s" % (time.time() - t0), flush=True)
    out = {"attempt_dt": np.array([d for d, _ in rec]), "attempt_acc": np.array([a for _, a in rec], dtype=np.int8),
           "snap_steps": np.array(snaps), "snap_t": np.array([hist[k]["t"] for k in snaps]),
           "switch_step": np.array(first), "switch_t": np.array(m.switches[0]["t"])}
    for f in FIELDS:
        out[f] = np.array([hist[k][f] for k in snaps])
        out["sens_" + f] = np.array([np.linalg.norm(h1[k][f] - hist[k][f]) / max(np.linalg.norm(hist[k][f]), 1e-300)
                                     for k in snaps])
        out["spread_" + f] = np.array([np.linalg.norm(h2[k][f] - hist[k][f]) / max(np.linalg.norm(hist[k][f]), 1e-300)
                                       for k in snaps])
    dst = os.path.join(HERE, "parity_c2qd.npz")
    np.savez_compressed(dst, **out)
    print("wrote", dst, os.path.getsize(dst), "bytes")


if __name__ == "__main__":
    main()
