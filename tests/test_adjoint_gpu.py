"""Discrete adjoint of the RK32 integration (scy_adj_*) on the GPU.

The gradient of the misfit with respect to a, b and Dc at every fault node
is checked against central finite differences of the device's own forward
map (h = 1e-6 relative, random directions, 1e-5 relative agreement), against
central differences of the oracle's forward map (the restated reference,
replaying the same step sizes), for independence of the checkpoint interval,
and through the torch.autograd binding.
"""
import numpy as np
import pytest

from oracle.problem import build_qd_problem
from oracle.qd import QDLinearElastic
from scycle_b200.configs import make_qd_problem, write_petsc_vec

pytestmark = pytest.mark.gpu

SOLVE_RTOL = 1e-14
STEPS = 30


def _problem(tmp_path, n=25, law="agingLaw"):
    path = make_qd_problem(str(tmp_path), Ny=n, Nz=n, state_law=law, integrator="RK32", name="adj")
    write_petsc_vec(path[:-len(".in")] + "_in_prestress", 26.0 + np.linspace(0.0, 0.5, n))
    return path


def _setup(path, steps=STEPS, ck=10):
    """Accepted steps of an adaptive run, targets from perturbed parameters,
    and an adjoint at the unperturbed ones."""
    from scycle_b200.adjoint import Adjoint
    from scycle_b200.qd import QD, inspect_in
    run = QD.from_in(path, solve_rtol=SOLVE_RTOL)
    run.record_attempts(True)
    run.integrate_begin_from_in()
    run.integrate_steps(steps)
    dts = run.step_sizes()
    assert len(dts) == steps
    q = QD.from_in(path, solve_rtol=SOLVE_RTOL)
    q.integrate_begin_from_in()
    adj = Adjoint(q, checkpoint_every=ck)
    adj.set_steps(dts)
    f = inspect_in(path, fields=("a", "b", "Dc"))
    base = (f["a"], f["b"], f["Dc"])
    rng = np.random.default_rng(3)
    pert = (base[0] * (1 + 0.02 * rng.standard_normal(q.Nz)), base[1] * (1 + 0.02 * rng.standard_normal(q.Nz)),
            base[2] * (1 + 0.05 * rng.standard_normal(q.Nz)))
    adj.set_params(*pert)
    adj.forward()
    ts, tv = adj.observations()
    adj.set_params(*base)
    ws, wv = 1.0 / np.mean(ts ** 2), 1.0 / np.mean(tv ** 2)
    adj.set_targets(ts, tv, ws, wv)
    return adj, base, dts, (ts, tv, ws, wv)


def _directions(base, k, seed=7):
    rng = np.random.default_rng(seed)
    return [tuple(p * rng.standard_normal(p.size) for p in base) for _ in range(k)]


@pytest.mark.parametrize("law", ["agingLaw", "slipLaw"])
def test_adjoint_matches_device_finite_differences(tmp_path, law):
    adj, base, dts, _ = _setup(_problem(tmp_path, law=law))
    J, ga, gb, gd = adj.gradient()
    assert J > 0
    h = 1e-6
    for d in _directions(base, 3):
        adj.set_params(*[p + h * q for p, q in zip(base, d)])
        jp = adj.forward()
        adj.set_params(*[p - h * q for p, q in zip(base, d)])
        jm = adj.forward()
        fd = (jp - jm) / (2 * h)
        an = ga @ d[0] + gb @ d[1] + gd @ d[2]
        assert abs(fd - an) <= 1e-5 * max(abs(fd), abs(an)), (fd, an)
    adj.set_params(*base)


def test_adjoint_checkpoint_interval_independent(tmp_path):
    path = _problem(tmp_path)
    g = []
    for ck in (4, 7, 40):
        adj, base, dts, _ = _setup(path, ck=ck)
        g.append(adj.gradient())
    for other in g[1:]:
        assert abs(other[0] - g[0][0]) <= 1e-12 * abs(g[0][0])
        for a, b in zip(other[1:], g[0][1:]):
            assert np.abs(a - b).max() <= 1e-8 * np.abs(b).max()


def test_adjoint_matches_oracle_finite_differences(tmp_path):
    """Central differences of the oracle (the restated reference) replaying
    the same step sizes, with the device's targets."""
    path = _problem(tmp_path)
    adj, base, dts, (ts, tv, ws, wv) = _setup(path, steps=20)
    J, ga, gb, gd = adj.gradient()
    P = build_qd_problem(open(path).read())

    def J_oracle(params):
        Q = dict(P)
        Q["a"], Q["b"], Q["Dc"] = [np.array(p) for p in params]
        ora = QDLinearElastic(Q)
        ora.integrate(max_steps=len(dts), replay=[(d, True) for d in dts])
        h = ora.history[1:]
        return sum(ws * np.sum((e["surfDisp"] - ts[n]) ** 2) + wv * np.sum((e["slipVel"] - tv[n]) ** 2)
                   for n, e in enumerate(h))

    assert abs(J_oracle(base) - J) <= 1e-6 * J
    h = 1e-6
    for d in _directions(base, 2, seed=11):
        fd = (J_oracle([p + h * q for p, q in zip(base, d)]) - J_oracle([p - h * q for p, q in zip(base, d)])) / (2 * h)
        an = ga @ d[0] + gb @ d[1] + gd @ d[2]
        assert abs(fd - an) <= 1e-5 * max(abs(fd), abs(an)), (fd, an)


def test_adjoint_torch_binding_and_knots(tmp_path):
    """J and its gradient through torch.autograd, with a, b and Dc given by
    knot values on a depth profile (piecewise linear, as setVec)."""
    import torch
    from scycle_b200.adjoint import knot_matrix, misfit_function
    path = _problem(tmp_path)
    adj, base, dts, _ = _setup(path, steps=15)
    z = np.arange(adj.Nz) / (adj.Nz - 1.0) * 30.0
    depths = np.linspace(0.0, 30.0, 8)
    Pm = torch.tensor(knot_matrix(z, depths))
    knots = [torch.tensor(np.interp(depths, z, p), requires_grad=True) for p in base]
    f = misfit_function()
    vals = [Pm @ k for k in knots]
    J = f.apply(vals[0], vals[1], vals[2], adj)
    J.backward()
    adj.set_params(*[v.detach().numpy() for v in vals])
    J2, ga, gb, gd = adj.gradient()
    assert abs(J.item() - J2) <= 1e-12 * J2
    for k, g in zip(knots, (ga, gb, gd)):
        assert np.allclose(k.grad.numpy(), Pm.numpy().T @ g, rtol=1e-12, atol=0)
