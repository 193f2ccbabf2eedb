"""The seeded synthetic workloads that stand in for the benchmark's
configurations (scycle_b200/configs.py), read back through the oracle's
.in reader and checked against their stated shapes and distributions:
101^2 aging law on a constant grid; 401^2 slip law on a tanh-stretched grid
with a per-node lognormal Dc (mean 8 mm, sigma_ln 0.2); the power-law
ensemble of three grid sizes with a linear geotherm of gradient U(15, 30)
K/km and a - b perturbed by a Gaussian random field of std 0.002 and
correlation length 2 km; the 201^2 adjoint workload with a, b and Dc given at
40 depth knots each (120 parameters)."""
import os
import re

import numpy as np

from oracle.problem import build_qd_problem
from scycle_b200.configs import aging_const_101, pl_ensemble_c3, slip_var_401, tanh_stretch


def _problem(path):
    return build_qd_problem(open(path).read())


def test_aging_const_101(tmp_path):
    P = _problem(aging_const_101(str(tmp_path), seed=5))
    assert P["Ny"] == P["Nz"] == 101
    assert P["fault"]["stateLaw"] == "agingLaw"
    z = P["z"].reshape(101, 101)[0]
    np.testing.assert_allclose(np.diff(z), 0.3, rtol=1e-12)
    np.testing.assert_allclose(P["a"], 0.010)
    np.testing.assert_allclose(P["b"], np.interp(z, [0, 12, 17, 30], [0.015, 0.015, 0.005, 0.005]), atol=1e-15)
    psi = P["psi"]
    assert abs(psi.mean() - 0.6) < 3e-5 and 0.7e-4 < psi.std() < 1.3e-4


def test_slip_var_401(tmp_path):
    P = _problem(slip_var_401(str(tmp_path), seed=3))
    Ny, Nz = P["Ny"], P["Nz"]
    assert Ny == Nz == 401
    assert P["fault"]["stateLaw"] == "slipLaw"
    y = P["y"].reshape(Ny, Nz)[:, 0]
    z = P["z"].reshape(Ny, Nz)[0]
    np.testing.assert_allclose(y, tanh_stretch(401, 30.0, 2.0), atol=1e-12)
    np.testing.assert_allclose(z, tanh_stretch(401, 30.0, 2.0), atol=1e-12)
    assert np.diff(z)[0] < np.diff(z)[-1] / 3  # clustered at the fault and the surface
    ln = np.log(P["Dc"])
    assert abs(ln.std() - 0.2) < 0.03
    assert abs(np.exp(ln.mean() + 0.5 * ln.var()) - 0.008) < 5e-4
    # seeds differ: another instance has another Dc
    Q = _problem(slip_var_401(str(tmp_path / "other"), seed=4))
    assert not np.allclose(Q["Dc"], P["Dc"])


def test_pl_ensemble_sizes_geotherm_and_ab_field(tmp_path):
    paths = pl_ensemble_c3(str(tmp_path), n_inst=9)
    sizes, grads, deltas = [], [], []
    for p in paths:
        P = _problem(p)
        n = P["Nz"]
        sizes.append(n)
        text = open(p).read()
        assert re.search(r"bulkDeformationType = powerLaw", text)
        tv = [float(v) for v in re.search(r"TVals = \[([^\]]*)\]", text).group(1).split()]
        grads.append((tv[1] - tv[0]) / 30.0)
        z = P["z"].reshape(P["Ny"], n)[0]
        b0 = np.interp(z, [0.0, 12.0, 17.0, 30.0], [0.015, 0.015, 0.005, 0.005])
        assert os.path.exists(p[:-len(".in")] + "_in_b")
        deltas.append((z, b0 - P["b"]))
    assert sizes == [101] * 3 + [201] * 3 + [301] * 3
    assert all(15.0 <= g <= 30.0 for g in grads) and len(set(np.round(grads, 9))) == len(grads)
    d_all = np.concatenate([d for _, d in deltas])
    assert 0.0014 < d_all.std() < 0.0026 and abs(d_all.mean()) < 0.001
    # correlation: neighbours 0.1 km apart (301 nodes over 30 km) move together,
    # points 10 km apart do not
    c_near, c_far = [], []
    for z, d in deltas:
        if len(z) != 301:
            continue
        c_near.append(np.mean(d[:-1] * d[1:]))
        c_far.append(np.mean(d[:-100] * d[100:]))
    assert np.mean(c_near) > 0.8 * d_all.var()
    assert abs(np.mean(c_far)) < 0.3 * d_all.var()


def test_adjoint_c4_knots(tmp_path):
    from scycle_b200.configs import C4_DEPTHS, adjoint_c4
    path, K, knots = adjoint_c4(str(tmp_path))
    P = _problem(path)
    assert P["Ny"] == P["Nz"] == 201 and P["fault"]["stateLaw"] == "agingLaw"
    assert K.shape == (201, 40) and len(C4_DEPTHS) == 40 and sum(len(k) for k in knots) == 120
    # the piecewise-linear map from the 40 knots reproduces the fields it wrote,
    # and every row of it is a partition of unity
    np.testing.assert_allclose(K.sum(axis=1), 1.0, atol=1e-14)
    for nm, k in zip(("a", "b", "Dc"), knots):
        np.testing.assert_allclose(P[nm], K @ k, rtol=1e-14, atol=1e-16)
    assert P["driver"]["timeIntegrator"] == "RK32"
