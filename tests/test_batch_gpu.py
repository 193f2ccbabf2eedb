"""Batched ensemble (scy_batch_*) on the GPU.

Every instance of a batch keeps its own adaptive step control; its stage
solves run inside shared launches (one CUDA graph per round).  Parity: each
instance against the oracle replaying that instance's attempt sequence
(1e-9 relative, as for the single-instance driver), results independent of
how the rounds are launched (graph or direct, concurrent streams or one),
and the FP32-preconditioned form against the FP64 form.
"""
import numpy as np
import pytest

from oracle.powerlaw import PowerLawQD, build_pl_problem
from oracle.problem import build_qd_problem
from oracle.qd import QDLinearElastic
from scycle_b200.configs import make_pl_problem, make_qd_problem, write_petsc_vec

pytestmark = pytest.mark.gpu

REL = 1e-9
SOLVE_RTOL = 1e-14
FIELDS = ("slip", "psi", "slipVel", "tauP", "surfDisp")


def _nrel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _with_prestress(path, nz, level):
    """inputDir/prestress (Fault::loadFieldsFromFiles, fault.cpp:128-129):
    a fault loaded to about `level` MPa, so that slip velocities and stresses
    are far from the root finder's absolute tolerance (1e-12 MPa)."""
    write_petsc_vec(path[:-len(".in")] + "_in_prestress", level + np.linspace(0.0, 0.5, nz))
    return path


def _le_paths(tmp_path, integrator="RK32"):
    """Five instances in two operator groups, given interleaved: 33 x 33
    constant grid, aging law, prestressed (seeds 0-2), and 41 x 37 stretched
    grid, slip law, lognormal Dc, steady-state initial guess (seeds 3-4)."""
    a = [_with_prestress(make_qd_problem(str(tmp_path / ("a%d" % s)), Ny=33, Nz=33, seed=s, integrator=integrator,
                                         name="a"), 33, 26.0 + 0.2 * s) for s in range(3)]
    b = [make_qd_problem(str(tmp_path / ("b%d" % s)), Ny=41, Nz=37, seed=s, integrator=integrator, name="b",
                         grid="variableGridSpacing", stretch_beta=2.0, state_law="slipLaw", dc_lognormal=True,
                         guess_ss=1) for s in (3, 4)]
    return [a[0], b[0], a[1], b[1], a[2]]


def _batch(paths, **kw):
    from scycle_b200.batch import Batch
    args = dict(solve_rtol=SOLVE_RTOL)
    args.update(kw)
    return Batch(paths, **args)


@pytest.mark.parametrize("integrator", ["RK32", "RK43"])
def test_batch_linear_elastic_matches_oracle(tmp_path, integrator):
    paths = _le_paths(tmp_path, integrator)
    b = _batch(paths)
    assert b.n_groups == 2 and b.group_of == [0, 1, 0, 1, 0]
    for i in range(b.n):
        b.instance(i).record_attempts(True)
    st = b.run(30)
    assert st.instance_steps == 30 * b.n
    assert st.rounds >= 30
    for i, path in enumerate(paths):
        q = b.instance(i)
        att = q.attempts()
        P = build_qd_problem(open(path).read())
        ora = QDLinearElastic(P, keep_history=False)
        rk = ora.integrate(max_steps=30, replay=att)
        qs = q.integrate_steps(0)
        assert qs.step_count == rk.stepCount == 30
        assert abs(qs.t - rk.currT) <= 1e-12 * rk.currT
        f = ora.fault
        ref = {"slip": f.slip, "psi": f.psi, "slipVel": f.slipVel, "tauP": f.tauP, "surfDisp": ora.u[::P["Nz"]]}
        for nm in FIELDS:
            assert _nrel(q.field(nm), ref[nm]) <= REL, (i, nm)


def test_batch_launch_forms_agree(tmp_path):
    """Graph or direct launches, concurrent group streams or one stream:
    bitwise the same states and the same step sequences."""
    paths = _le_paths(tmp_path)
    out = {}
    for form in ((True, True), (False, True), (True, False)):
        b = _batch(paths, graphs=form[0], concurrent=form[1], cg_its=3)
        for i in range(b.n):
            b.instance(i).record_attempts(True)
        b.run(12)
        out[form] = [({nm: b.instance(i).field(nm) for nm in FIELDS + ("u",)}, b.instance(i).attempts())
                     for i in range(b.n)]
        b.close()
    ref = out[(True, True)]
    for form, res in out.items():
        for i in range(len(ref)):
            assert res[i][1] == ref[i][1], (form, i)
            for nm in ref[i][0]:
                assert np.array_equal(res[i][0][nm], ref[i][0][nm]), (form, i, nm)


def test_batch_matches_single_instance_runs(tmp_path):
    """An instance of a batch takes the steps it takes alone: the same
    accept / reject decisions and, with the batch's attempts forced on the
    single-instance driver, the same states.  (The step sizes themselves
    are not compared: right after the steady-state guess the embedded error
    estimate is a difference of two solutions that agree to round-off, so
    solves converged to the same tolerance but by different iterations give
    step sizes a few percent apart.)"""
    from scycle_b200.qd import QD
    paths = _le_paths(tmp_path)
    b = _batch(paths)
    for i in range(b.n):
        b.instance(i).record_attempts(True)
    b.run(25)
    for i, path in enumerate(paths):
        ab = b.instance(i).attempts()
        q = QD.from_in(path, solve_rtol=SOLVE_RTOL)
        q.record_attempts(True)
        q.integrate_begin_from_in()
        q.integrate_steps(25)
        aq = q.attempts()
        assert [a for _, a in ab] == [a for _, a in aq]
        q = QD.from_in(path, solve_rtol=SOLVE_RTOL)
        q.force_attempts(ab)
        q.integrate_begin_from_in()
        q.integrate_steps(25)
        for nm in ("slip", "psi", "slipVel", "tauP"):
            assert _nrel(b.instance(i).field(nm), q.field(nm)) <= REL, (i, nm)


def test_batch_mixed_precision_against_fp64(tmp_path):
    """FP32 fast-diagonalisation preconditioner inside FP64 CG: the FP64
    batch's attempt sequence replayed gives states within 1e-9."""
    paths = _le_paths(tmp_path)
    b64 = _batch(paths)
    for i in range(b64.n):
        b64.instance(i).record_attempts(True)
    b64.run(30)
    att = [b64.instance(i).attempts() for i in range(b64.n)]
    ref = [{nm: b64.instance(i).field(nm) for nm in FIELDS} for i in range(b64.n)]
    b32 = _batch(paths, precision="mixed")
    for i in range(b32.n):
        b32.instance(i).force_attempts(att[i])
    b32.run(30)
    for i in range(b32.n):
        for nm in FIELDS:
            assert _nrel(b32.instance(i).field(nm), ref[i][nm]) <= REL, (i, nm)


def test_batch_power_law_matches_oracle(tmp_path):
    """Three power-law instances (two operator groups: 33 x 33 with two
    geotherms, 41 x 37), RK43 over 25 steps, oracle replaying each
    instance's attempts."""
    mk = lambda s, ny, nz, grad: _with_prestress(
        make_pl_problem(str(tmp_path / ("p%d" % s)), Ny=ny, Nz=nz, seed=s, grad=grad, extra={"maxDeltaT": "1e6"}),
        nz, 26.0 + 0.3 * s)
    paths = [mk(0, 33, 33, 15.0), mk(1, 41, 37, 20.0), mk(2, 33, 33, 30.0)]
    b = _batch(paths)
    assert b.n_groups == 2
    for i in range(b.n):
        b.instance(i).record_attempts(True)
    b.run(25)
    for i, path in enumerate(paths):
        q = b.instance(i)
        ora = PowerLawQD(build_pl_problem(open(path).read()))
        rk = ora.integrate(max_steps=25, replay=q.attempts())
        assert rk.stepCount == 25
        h = ora.history[-1]
        for nm in ("gVxy", "psi", "slip", "slipVel", "tauP"):
            assert _nrel(q.field(nm), h[nm]) <= REL, (i, nm)
        assert np.linalg.norm(q.field("gVxz") - h["gVxz"]) <= REL * max(np.linalg.norm(h["gVxz"]),
                                                                         np.linalg.norm(h["gVxy"]))
        assert _nrel(q.field("sdev"), h["sdev"]) <= REL
        assert np.abs(q.field("gVxy")).max() > 0


def test_batch_rejects_mixed_drivers(tmp_path):
    from scycle_b200._lib import ScyError
    paths = [make_qd_problem(str(tmp_path / "le"), Ny=33, Nz=33, integrator="RK43"),
             make_pl_problem(str(tmp_path / "pl"), Ny=33, Nz=33)]
    with pytest.raises(ScyError, match="same driver"):
        _batch(paths)


def test_batch_state_io(tmp_path):
    """State and fault-field transfer of the whole batch: concatenated in
    instance order, and a state written back unchanged leaves the run as it
    was."""
    paths = _le_paths(tmp_path)
    b1, b2 = _batch(paths, cg_its=3), _batch(paths, cg_its=3)
    for b in (b1, b2):
        b.run(5)
    assert b1.state_size() == sum(b1.instance(i).state_size() for i in range(b1.n))
    vel = b1.fault_field("slipVel")
    parts = np.split(vel, np.cumsum([b1.instance(i).Nz for i in range(b1.n)])[:-1])
    for i in range(b1.n):
        assert np.array_equal(parts[i], b1.instance(i).field("slipVel"))
    state = np.concatenate([np.concatenate([b1.instance(i).field("psi"), b1.instance(i).field("slip")])
                            for i in range(b1.n)])
    b1.set_states(state)
    b1.run(5)
    b2.run(5)
    assert np.array_equal(b1.fault_field("slip"), b2.fault_field("slip"))
    assert np.array_equal(b1.fault_field("psi"), b2.fault_field("psi"))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_banded_preconditioner_matches_dense(tmp_path, precision):
    """The preconditioner as z-transform GEMMs with banded Cholesky solves
    along y is the four-GEMM fast diagonalisation in another form: with the
    same attempts forced, the states agree within 1e-9, and one (FP64) or
    two (FP32) iterations per stage solve still reach the tolerance."""
    paths = _le_paths(tmp_path)
    bd = _batch(paths, precision=precision, fd_dense=True)
    for i in range(bd.n):
        bd.instance(i).record_attempts(True)
    sd = bd.run(20)
    att = [bd.instance(i).attempts() for i in range(bd.n)]
    bb = _batch(paths, precision=precision)
    for i in range(bb.n):
        bb.instance(i).force_attempts(att[i])
    sb = bb.run(20)
    assert sb.cg_its <= sd.cg_its + 1
    for i in range(bb.n):
        for nm in FIELDS:
            assert _nrel(bb.instance(i).field(nm), bd.instance(i).field(nm)) <= REL, (i, nm)


def test_batch_sweep_wait_timeout_is_reported_and_recoverable(tmp_path):
    """The banded sweeps' data waits are bounded: with a test hook
    withholding each block's first chunk copy (a wait that nothing
    completes) and the limit lowered to 64 polls, the waits run out, the
    blocks mark their instances (status bit 4) and still await the copies
    they did issue, the batch repeats the round three times and then reports
    SCY_ERR_TIMEOUT (no hang, no fault).  With the hook cleared the same
    batch carries on and gives what an undisturbed batch gives."""
    from scycle_b200 import _lib as S
    paths = _le_paths(tmp_path)
    b = _batch(paths)
    ref = _batch(paths)
    b.run(2)
    ref.run(3)
    S.check(S.lib().scy_batch_set_sweep_test(b.h, 64, 1))
    with pytest.raises(S.ScyError) as ei:
        b.run(1)
    assert "pipeline wait" in str(ei.value)
    S.check(S.lib().scy_batch_set_sweep_test(b.h, 1 << 18, 0))
    b.run(1)
    for i in range(len(paths)):
        for f in FIELDS:
            assert _nrel(b.instance(i).field(f), ref.instance(i).field(f)) <= 1e-12, (i, f)
    b.close()
    ref.close()
