"""Oracle of the quasi-dynamic / fully dynamic cycle driver, and the C++
host-side set-up of the fully dynamic phase, on the CPU."""
import math

import numpy as np
import pytest

from oracle import fault as F
from oracle.ode import AdaptiveRK
from oracle.qdfd import build_qdfd_problem, penalty_ay, qdfd_settings
from scycle_b200.configs import make_qdfd_problem


def test_settings_defaults_and_check_input():
    s = qdfd_settings("")
    assert s["trigger_qd2fd"] == 1e-3 and s["trigger_fd2qd"] == 1e-3
    assert s["limit_fd"] == 0.1 and s["limit_qd"] == 1e-8
    assert s["limit_stride_fd"] == pytest.approx(0.01)
    assert s["minDeltaT"] == 1e-3 and s["maxNumCycles"] == 1000
    # limit_fd below trigger_qd2fd is raised to 10 * trigger_qd2fd
    s = qdfd_settings("limit_fd = 1e-4\ntrigger_qd2fd = 1e-3\n")
    assert s["limit_fd"] == pytest.approx(1e-2)
    # limit_qd is compared with trigger_fd2qd but reset from trigger_qd2fd
    s = qdfd_settings("limit_qd = 5e-3\ntrigger_fd2qd = 1e-3\ntrigger_qd2fd = 2e-2\n")
    assert s["limit_qd"] == pytest.approx(2e-3)


def test_penalty_vector_index_quirk():
    """computePenaltyVectors advances its index only for iy = 0 rows: the
    damping of the R and B boundaries collapses onto entries Nz-1 and Nz."""
    Ny, Nz = 7, 5
    cs = np.full(Ny * Nz, 2.0)
    ay = penalty_ay(Ny, Nz, 0.1, 0.2, "outGoingCharacteristics", "freeSurface", "symmFault",
                    "outGoingCharacteristics", cs)
    nz = np.nonzero(ay)[0]
    assert list(nz) == [Nz - 1, Nz]
    assert ay[Nz - 1] == pytest.approx(2.0 * 0.5 / 0.2)          # B corner of row 0
    assert ay[Nz] == pytest.approx(2.0 * (0.5 / 0.1 + 0.5 / 0.2))  # last node: R and B
    # with T outgoing too, entry 0 also picks up the T damping of node 0
    ay = penalty_ay(Ny, Nz, 0.1, 0.2, "outGoingCharacteristics", "outGoingCharacteristics", "symmFault",
                    "outGoingCharacteristics", cs)
    assert ay[0] == pytest.approx(2.0 * 0.5 / 0.2)


def test_vel_fd_residual_derivative():
    """The fully dynamic velocity residual's Jacobian is exact."""
    rng = np.random.default_rng(1)
    for _ in range(20):
        V = 10 ** rng.uniform(-6, 0)
        Phi = rng.uniform(-3, 3)
        fp, sN, psi, a = rng.uniform(0.05, 0.3), 50.0, rng.uniform(0.5, 0.8), 0.01
        f, J = F.resid_vel_fd(V, Phi, fp, sN, psi, a, 1e-6)
        h = 1e-6 * V
        fd = (F.resid_vel_fd(V + h, Phi, fp, sN, psi, a, 1e-6)[0] - F.resid_vel_fd(V - h, Phi, fp, sN, psi, a,
                                                                                    1e-6)[0]) / (2 * h)
        assert J == pytest.approx(fd, rel=1e-5)


@pytest.mark.parametrize("law", ["agingLaw", "slipLaw"])
def test_state_fd_residual_derivative(law):
    rng = np.random.default_rng(2)
    for _ in range(20):
        st, pp = rng.uniform(0.4, 0.8), rng.uniform(0.4, 0.8)
        V = 10 ** rng.uniform(-9, 0)
        args = (pp, V, 0.01, 0.015, 0.6, 1e-6, 0.008, 0.01)
        f, J = F.resid_state_fd(law, st, *args)
        h = 1e-7
        fd = (F.resid_state_fd(law, st + h, *args)[0] - F.resid_state_fd(law, st - h, *args)[0]) / (2 * h)
        assert J == pytest.approx(fd, rel=1e-5)


def test_fd_fault_update_balances_friction():
    """After Fault_fd::d_dt, a sliding node satisfies the discrete momentum
    balance V + fricPen * strength(V) = |Phi| at the root."""
    Nz = 16
    rng = np.random.default_rng(3)
    fq = F.FaultQD(np.linspace(0, 10, Nz), np.full(Nz, 0.01), np.full(Nz, 0.015), np.full(Nz, 50.0),
                   np.full(Nz, 0.008), rng.uniform(0.5, 0.6, Nz), np.full(Nz, 32.04), np.full(Nz, 2.67))
    ff = F.FaultFD(fq, np.full(Nz, 2.67), np.full(Nz, 0.2), 2.0)
    ff.slip0 = np.zeros(Nz)
    ff.tau0 = np.full(Nz, 30.0)
    ff.d2u = rng.normal(0, 1, Nz)
    ff.slipVel = np.full(Nz, 1e-3)
    var = {"psi": fq.psi.copy(), "slip": rng.uniform(0, 1e-3, Nz)}
    prev = {"psi": fq.psi.copy(), "slip": var["slip"] - 1e-5}
    dt = 0.01
    ff.d_dt(dt, var, prev)
    ff.uPrev = (prev["slip"] - ff.slip0) / 2.0
    u = (var["slip"] - ff.slip0) / 2.0
    ff.u, u_new = u, ff.u
    ff.set_phi(dt)
    V = ff.slipVel
    mv = V >= 1e-14
    s = F.strength_psi(fq.sN, var["psi"], np.abs(V), fq.a, fq.v0)
    res = np.abs(V) + ff.fricPen * s - np.abs(ff.Phi)
    assert np.all(np.abs(res[mv]) < 1e-9 * np.abs(ff.Phi[mv]) + 1e-10)


def test_rk_restart_growth_cap():
    """A fresh PID integrator past step 4 has errA = [0, 0]: the ratio is
    0 * inf = NaN, std::min keeps 5 dt, so the first update grows 5x."""
    rk = AdaptiveRK("RK43", 10, 1e9, 0.1, "PID")
    rk.set_time_step_bounds(1e-3, 1e10)
    rk.set_initial_step_count(100)
    assert rk.maxNumSteps == 110
    rk.stepCount = 101
    assert rk.compute_step_size(3e-9) == pytest.approx(0.5)
    rk.errA = [3e-9, 0.0]  # second update: ratio = inf, cap again
    assert rk.compute_step_size(3e-9) == pytest.approx(0.5)
    rk.errA = [3e-9, 2e-9]
    assert math.isfinite(rk.compute_step_size(3e-9))


def test_cpp_cycle_setup_matches_oracle(tmp_path):
    """The C++ loader's cycle settings, CFL step and penalty vector equal the
    oracle's (constant and stretched grids)."""
    from scycle_b200.cycle import inspect_cycle_in
    from oracle.qdfd import QDFDLinearElastic
    cases = [dict(Ny=41, Nz=41, name="c"),
             dict(Ny=33, Nz=29, grid="variableGridSpacing", stretch_beta=2.0, name="v",
                  extra={"CFL": "0.5", "limit_fd": "0.005"})]
    for kw in cases:
        path = make_qdfd_problem(str(tmp_path), **kw)
        info = inspect_cycle_in(path)
        P = build_qdfd_problem(open(path).read())
        m = QDFDLinearElastic(P, keep_history=False)
        assert info["dt_fd"] == pytest.approx(m.deltaT_fd, rel=1e-15)
        assert np.array_equal(np.nonzero(info["ay"])[0], np.nonzero(m.ay)[0])
        assert np.allclose(info["ay"], m.ay, rtol=1e-15, atol=0)
        for k in ("trigger_qd2fd", "trigger_fd2qd", "limit_qd", "limit_fd"):
            assert info[k] == pytest.approx(P["fd"][k], rel=1e-15), k
        assert info["max_num_cycles"] == P["fd"]["maxNumCycles"]


def test_cfl_step_801():
    """801x801 on 30 km with cs = sqrt(32.04/2.67): dt = gcfl * dy / cs."""
    gcfl = 0.7071 / math.sqrt(1.4498)
    dt = gcfl * (30.0 / 800.0) / math.sqrt(32.04 / 2.67)
    assert dt == pytest.approx(0.006357222828, rel=1e-9)
