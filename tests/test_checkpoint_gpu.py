"""Checkpoint / restart of the quasi-dynamic driver (enableCheckpointing) on the GPU.

The reference writes chkpt_* files at step 0, every `interval` steps and at
the end, stops the run there, and a new run of the same input file restarts
from them, appending to the output files.  With the extension key
ckptContinueSteps = 1 the restart keeps the step count and error history,
so two runs of six steps each must give the state of one uninterrupted
twelve-step run.  Without it the restart behaves as the reference's does
(step count and error history from zero); that path is compared with the
oracle restarted from the device's own checkpoint files.
"""
import os

import numpy as np
import pytest

from scycle_b200.configs import make_qd_problem, write_petsc_vec

pytestmark = pytest.mark.gpu


def _nrel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _problem(d, ckpt, cont=True):
    n = 25
    extra = {"stride1D": "1"}
    if ckpt:
        extra.update({"enableCheckpointing": "1", "interval": "6"})
        if cont:
            extra["ckptContinueSteps"] = "1"  # extension: keep step count and error history
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


def test_checkpoint_files_and_restart_match_the_oracle(tmp_path):
    """The device's chkpt_* files after six steps hold the oracle's state
    after the same six attempts (read with the oracle's PETSc reader), and a
    run restarted from those files matches the oracle restarted from them
    (reference restart semantics: step count and error history from zero)."""
    import glob
    import shutil

    from oracle.checkpoint import read_checkpoint, restart_problem
    from oracle.problem import build_qd_problem
    from oracle.qd import QDLinearElastic
    from scycle_b200.qd import QD
    os.makedirs(tmp_path / "a")
    path, out = _problem(tmp_path / "a", True, cont=False)
    P = build_qd_problem(open(path).read())
    run1 = QD.from_in(path, solve_rtol=1e-14, exact_jacobian=False)
    run1.record_attempts(True)
    run1.integrate_begin_from_in()
    st = run1.integrate_steps(100)
    assert st.done == 2 and st.step_count == 6
    att1 = run1.attempts()
    run1.close()
    # the run's checkpoint files (outputDir is a prefix) before the restart rewrites them
    saved = str(tmp_path / "ckpt6") + "/ck_"
    os.makedirs(os.path.dirname(saved))
    for f in glob.glob(out + "*"):
        shutil.copy(f, saved + os.path.basename(f)[len(os.path.basename(out)):])
    ck = read_checkpoint(saved)
    assert ck["ckptNumber"] == 2 and ck["chkpt_stepCount"] == 6
    ora = QDLinearElastic(P, keep_history=False)
    rk = ora.integrate(max_steps=6, replay=att1)
    f = ora.fault
    assert abs(ck["chkpt_currT"] - rk.currT) <= 1e-12 * rk.currT
    for nm, ref in (("slip", f.slip), ("slipVel", f.slipVel), ("psi", f.psi), ("tau", f.tauP), ("tauQS", f.tauQSP),
                    ("prestress", f.prestress), ("sNEff", f.sN), ("momBal_bcL", ora.bcL), ("momBal_bcR", ora.bcR),
                    ("momBal_bcRShift", ora.bcRShift)):
        assert _nrel(ck[nm], ref) <= 1e-9, nm
    # the step-size controller's numbers follow from embedded error
    # estimates (differences of nearly equal solutions): fewer digits
    assert np.allclose([ck["chkpt_currErr"], ck["chkpt_prevErr"], ck["chkpt_deltaT"]],
                       [rk.errA[0], rk.errA[1], rk.newDeltaT], rtol=1e-6, atol=0)
    # restart: the device from its files, the oracle from the same files
    run2 = QD.from_in(path, solve_rtol=1e-14, exact_jacobian=False)
    run2.record_attempts(True)
    run2.integrate_begin_from_in()
    st2 = run2.integrate_steps(100)
    assert st2.done == 2 and st2.step_count == 6  # counted from 0 again, stops at the next checkpoint
    assert int(open(out + "ckptNumber").read()) == 4  # rewritten at the restart, then at its step 6
    ora2 = QDLinearElastic(restart_problem(P, ck), keep_history=False)
    rk2 = ora2.integrate(max_steps=6, replay=run2.attempts())
    assert rk2.stepCount == 6
    assert abs(st2.t - rk2.currT) <= 1e-12 * rk2.currT
    f2 = ora2.fault
    for nm, ref in (("slip", f2.slip), ("psi", f2.psi), ("slipVel", f2.slipVel), ("tauP", f2.tauP),
                    ("surfDisp", ora2.u[::P["Nz"]])):
        assert _nrel(run2.field(nm), ref) <= 1e-9, nm
    run2.close()
