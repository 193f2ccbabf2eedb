"""Checkpoint / restart of the quasi-dynamic driver (enableCheckpointing) on the GPU.

The reference writes chkpt_* files at step 0, every `interval` steps and at
the end, stops the run there, and a new run of the same input file restarts
from them, appending to the output files.  Two runs of six steps each must
give the state of one uninterrupted twelve-step run.
"""
import os

import numpy as np
import pytest

from scycle_b200.configs import make_qd_problem, write_petsc_vec

pytestmark = pytest.mark.gpu


def _nrel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _problem(d, ckpt):
    n = 25
    extra = {"stride1D": "1"}
    if ckpt:
        extra.update({"enableCheckpointing": "1", "interval": "6"})
    path = make_qd_problem(str(d), Ny=n, Nz=n, integrator="RK32", name="ck", extra=extra)
    write_petsc_vec(path[:-len(".in")] + "_in_prestress", 26.0 + np.linspace(0.0, 0.5, n))
    return path, str(d / "ck_out_")


def test_checkpoint_restart_continues_the_run(tmp_path):
    from scycle_b200.qd import QD
    os.makedirs(tmp_path / "a")
    os.makedirs(tmp_path / "b")
    path, out = _problem(tmp_path / "a", True)
    run1 = QD.from_in(path, solve_rtol=1e-14)
    run1.integrate_begin_from_in()
    st = run1.integrate_steps(100)
    assert st.done == 2 and st.step_count == 6
    run1.close()
    assert int(open(out + "ckptNumber").read()) == 2  # step 0 and step 6
    assert int(open(out + "chkpt_stepCount").read()) == 6
    run2 = QD.from_in(path, solve_rtol=1e-14)
    run2.record_attempts(True)
    run2.integrate_begin_from_in()
    st2 = run2.integrate_steps(100)
    assert st2.done == 2 and st2.step_count == 12
    # the same problem without checkpoints, twelve steps
    ref_path, ref_out = _problem(tmp_path / "b", False)
    ref = QD.from_in(ref_path, solve_rtol=1e-14)
    ref.record_attempts(True)
    ref.integrate_begin_from_in()
    sr = ref.integrate_steps(12)
    assert sr.step_count == 12
    assert abs(st2.t - sr.t) <= 1e-12 * sr.t
    for nm in ("slip", "psi", "slipVel", "tauP", "surfDisp"):
        assert _nrel(run2.field(nm), ref.field(nm)) <= 1e-9, nm
    ar, a2 = ref.attempts(), run2.attempts()
    tail = ar[len(ar) - len(a2):]
    assert [a for _, a in a2] == [a for _, a in tail]
    assert np.allclose([d for d, _ in a2], [d for d, _ in tail], rtol=1e-9, atol=0)
    # output appended across the restart; the restart writes its start (step 6) again
    run2.flush_output()
    ref.flush_output()
    t = np.loadtxt(out + "med_time1D.txt")
    tr = np.loadtxt(ref_out + "med_time1D.txt")
    assert t.size == 14 and tr.size == 13
    assert t[6] == t[7]
    assert np.allclose(np.delete(t, 7), tr, rtol=1e-12, atol=0)
