"""Stride output of the quasi-dynamic driver (scy_qd_set_output) on the GPU.

The reference's timeMonitor writes PETSc-binary Vec records and
med_time / med_dt text files every stride1D / stride2D steps and at step 0;
here the files are read back and compared with the oracle's states at the
same steps (the oracle replaying the device's attempts).
"""
import numpy as np
import pytest

from oracle.infile import read_petsc_vecs
from oracle.problem import build_qd_problem
from oracle.qd import QDLinearElastic
from scycle_b200.configs import make_qd_problem, write_petsc_vec

pytestmark = pytest.mark.gpu

REL = 1e-9


def _nrel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def test_stride_output_files(tmp_path):
    from scycle_b200.qd import QD
    n = 25
    path = make_qd_problem(str(tmp_path), Ny=n, Nz=n, integrator="RK32", name="out",
                           extra={"stride1D": "2", "stride2D": "3"})
    write_petsc_vec(path[:-len(".in")] + "_in_prestress", 26.0 + np.linspace(0.0, 0.5, n))
    prefix = str(tmp_path / "out_out_")
    dev = QD.from_in(path, solve_rtol=1e-14)
    dev.record_attempts(True)
    dev.integrate_begin_from_in()
    dev.integrate_steps(9)
    dev.flush_output()
    P = build_qd_problem(open(path).read())
    ora = QDLinearElastic(P)
    ora.integrate(max_steps=9, replay=dev.attempts())
    hist = {h["step"]: h for h in ora.history}
    steps1, steps2 = [0, 2, 4, 6, 8], [0, 3, 6, 9]
    t1 = np.loadtxt(prefix + "med_time1D.txt")
    d1 = np.loadtxt(prefix + "med_dt1D.txt")
    assert t1.size == len(steps1) and np.loadtxt(prefix + "med_time2D.txt").size == len(steps2)
    for k, s in enumerate(steps1):
        assert abs(t1[k] - hist[s]["t"]) <= 1e-12 * max(abs(hist[s]["t"]), 1.0)
    taken = dev.step_sizes()
    for k, s in enumerate(steps1[1:], 1):
        assert d1[k] == pytest.approx(taken[s - 1], rel=1e-15)
    recs = {nm: read_petsc_vecs(prefix + nm) for nm in ("slip", "slipVel", "psi", "tauP", "surfDisp", "momBal_bcR",
                                                          "momBal_bcRShift", "momBal_bcL", "sNEff")}
    for nm in recs:
        assert len(recs[nm]) == len(steps1), nm
    for k, s in enumerate(steps1):
        assert _nrel(recs["slip"][k], hist[s]["slip"]) <= REL
        assert _nrel(recs["psi"][k], hist[s]["psi"]) <= REL
        if s > 0:  # rates and stresses of step 0 are written before the first d_dt
            assert _nrel(recs["slipVel"][k], hist[s]["slipVel"]) <= REL
            assert _nrel(recs["tauP"][k], hist[s]["tauP"]) <= REL
            assert _nrel(recs["surfDisp"][k], hist[s]["surfDisp"]) <= REL
    # the first record of momBal_bcRShift holds bcRShift, the later ones bcR
    assert np.array_equal(recs["momBal_bcRShift"][0], np.asarray(P["bcRShift"], dtype=np.float64))
    for k in range(1, len(steps1)):
        assert np.array_equal(recs["momBal_bcRShift"][k], recs["momBal_bcR"][k])
    assert np.allclose(recs["sNEff"][1], P["sN"])
    u = read_petsc_vecs(prefix + "momBal_u")
    sxy = read_petsc_vecs(prefix + "momBal_sxy")
    assert len(u) == len(sxy) == len(steps2)
    assert _nrel(u[2][::n], hist[6]["surfDisp"]) <= REL
    # mu Dy u on the fault row is the fault's quasi-static stress before the prestress
    assert _nrel(sxy[2][:n] + P["prestress"], hist[6]["tauQSP"]) <= REL
