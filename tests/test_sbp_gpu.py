"""Device SBP-SAT operators and elliptic solve vs the oracle (GPU)."""
import itertools

import numpy as np
import pytest

from oracle.sbp2d import SbpOps as OracleSbp

pytestmark = pytest.mark.gpu

BCS = [("Dirichlet", "Neumann", "Dirichlet", "Neumann"), ("Neumann", "Dirichlet", "Neumann", "Dirichlet"),
       ("Dirichlet", "Dirichlet", "Dirichlet", "Dirichlet")]


def _case(order, grid, Ny, Nz, seed=0, compat="fullyCompatible", bcs=BCS[0]):
    rng = np.random.default_rng(seed)
    Ly, Lz = 30.0, 24.0
    q = np.repeat(np.arange(Ny) / (Ny - 1), Nz)
    r = np.tile(np.arange(Nz) / (Nz - 1), Ny)
    var = grid == "variableGridSpacing"
    y = Ly * np.sinh(2 * q) / np.sinh(2) if var else None
    z = Lz * (r + 0.2 * r * r) / 1.2 if var else None
    mu = 32.04 + 2 * rng.random(Ny * Nz)
    from scycle_b200.sbp import SbpOps
    dev = SbpOps(order, Ny, Nz, Ly, Lz, mu, grid=grid, y=y, z=z, compat=compat, bcs=bcs)
    ora = OracleSbp(order, Ny, Nz, Ly, Lz, mu, grid=grid, y=y, z=z, compat=compat, bcs=bcs)
    return dev, ora, rng


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("order,grid,bcs,shape", list(itertools.product(
    (2, 4), ("constantGridSpacing", "variableGridSpacing"), BCS, [(37, 45), (101, 67)])))
def test_apply_A_matches_oracle(order, grid, bcs, shape):
    dev, ora, rng = _case(order, grid, *shape, bcs=bcs)
    x = rng.standard_normal(dev.N)
    out = dev.apply("A", x).cpu().numpy()
    assert _rel(out, ora.A @ x) <= 1e-13


@pytest.mark.parametrize("grid,bcs", list(itertools.product(("constantGridSpacing", "variableGridSpacing"), BCS[:2])))
def test_apply_A_separable_interior(grid, bcs):
    """Constant mu: the interior tiles use the composed 9-point stencils
    built from the 1D coefficient arrays (grid large enough for such tiles)."""
    Ny, Nz = 129, 161
    Ly, Lz = 30.0, 24.0
    q = np.repeat(np.arange(Ny) / (Ny - 1), Nz)
    r = np.tile(np.arange(Nz) / (Nz - 1), Ny)
    var = grid == "variableGridSpacing"
    y = Ly * np.sinh(2 * q) / np.sinh(2) if var else None
    z = Lz * (r + 0.2 * r * r) / 1.2 if var else None
    mu = np.full(Ny * Nz, 32.04)
    from scycle_b200.sbp import SbpOps
    dev = SbpOps(4, Ny, Nz, Ly, Lz, mu, grid=grid, y=y, z=z, bcs=bcs)
    ora = OracleSbp(4, Ny, Nz, Ly, Lz, mu, grid=grid, y=y, z=z, bcs=bcs)
    x = np.random.default_rng(7).standard_normal(Ny * Nz)
    out = dev.apply("A", x).cpu().numpy()
    assert _rel(out, ora.A @ x) <= 1e-13
    # a smooth field: the operator's cancellation exposes rounding differences
    xs = np.sin(q * 3.0) * np.cos(r * 2.0) + 0.1 * q
    out = dev.apply("A", xs).cpu().numpy()
    ref = ora.A @ xs
    assert np.linalg.norm(out - ref) <= 1e-12 * np.linalg.norm(ref)


@pytest.mark.parametrize("order,grid", list(itertools.product((2, 4), ("constantGridSpacing", "variableGridSpacing"))))
def test_first_derivative_ops(order, grid):
    dev, ora, rng = _case(order, grid, 41, 29)
    x = rng.standard_normal(dev.N)
    checks = {"Dy": ora.Dy_Iz @ x, "Dz": ora.Iy_Dz @ x, "muxDy": ora.muxDy(x), "muxDz": ora.muxDz(x),
              "Dyxmu": ora.Dy_Iz @ (ora.mu_vec * x), "Dzxmu": ora.Iy_Dz @ (ora.mu_vec * x),
              "H": ora.H @ x, "Hinv": ora.Hinv @ x}
    for op, ref in checks.items():
        assert _rel(dev.apply(op, x).cpu().numpy(), ref) <= 1e-13, op


@pytest.mark.parametrize("order,grid,bcs", list(itertools.product((2, 4), ("constantGridSpacing", "variableGridSpacing"), BCS)))
def test_set_rhs_matches_oracle(order, grid, bcs):
    dev, ora, rng = _case(order, grid, 33, 41, bcs=bcs)
    bcL, bcR = rng.standard_normal(41), rng.standard_normal(41)
    bcT, bcB = rng.standard_normal(33), rng.standard_normal(33)
    out = dev.set_rhs(bcL, bcR, bcT, bcB).cpu().numpy()
    assert _rel(out, ora.set_rhs(bcL, bcR, bcT, bcB)) <= 1e-13


@pytest.mark.parametrize("order,grid,precision,precond", list(itertools.product(
    (2, 4), ("constantGridSpacing", "variableGridSpacing"), ("fp64", "mixed"), ("mg", "fd"))))
def test_solve_matches_direct_solve(order, grid, precision, precond):
    import scipy.sparse.linalg as spla
    dev, ora, rng = _case(order, grid, 101, 81)
    bcL = np.linspace(0, 1, 81) ** 2
    bcR = np.full(81, 0.3)
    rhs = ora.set_rhs(bcL, bcR, np.zeros(101), np.zeros(101))
    ref = spla.spsolve(ora.A.tocsc(), rhs)
    u, st = dev.solve(rhs, rtol=1e-12, max_its=300, precision=precision, precond=precond)
    assert st.converged
    assert _rel(u.cpu().numpy(), ref) <= 1e-9


@pytest.mark.parametrize("rpt,grid,mu_kind", list(itertools.product(
    (1, 2, 4), ("constantGridSpacing", "variableGridSpacing"), ("constant", "one_column"))))
def test_full_form_every_rows_per_thread(monkeypatch, rpt, grid, mu_kind):
    """The full-form operator kernels (one 17-point stencil per row and per
    column, line classes, 9-point interior tiles) at 1, 2 and 4 output rows
    per thread (SCY_FULL_RPT, read when the operator is built): A x, and a
    CG solve whose matrix-vector products and residuals run through them,
    against the oracle.  mu is constant, or constant but for one column (an
    exceptional y line)."""
    import scipy.sparse.linalg as spla
    from scycle_b200.sbp import SbpOps
    monkeypatch.setenv("SCY_FULL_RPT", str(rpt))
    Ny, Nz = 137, 163
    Ly, Lz = 30.0, 24.0
    q = np.repeat(np.arange(Ny) / (Ny - 1), Nz)
    r = np.tile(np.arange(Nz) / (Nz - 1), Ny)
    var = grid == "variableGridSpacing"
    y = Ly * np.sinh(2 * q) / np.sinh(2) if var else None
    z = Lz * (r + 0.2 * r * r) / 1.2 if var else None
    mu = np.full(Ny * Nz, 32.04)
    if mu_kind == "one_column":
        mu.reshape(Ny, Nz)[:, Nz // 3] = 27.5
    dev = SbpOps(4, Ny, Nz, Ly, Lz, mu, grid=grid, y=y, z=z)
    ora = OracleSbp(4, Ny, Nz, Ly, Lz, mu, grid=grid, y=y, z=z)
    x = np.random.default_rng(rpt).standard_normal(Ny * Nz)
    assert _rel(dev.apply("A", x).cpu().numpy(), ora.A @ x) <= 1e-13
    rhs = ora.set_rhs(np.linspace(0, 1, Nz) ** 2, np.full(Nz, 0.3), np.zeros(Ny), np.zeros(Ny))
    ref = spla.spsolve(ora.A.tocsc(), rhs)
    u, st = dev.solve(rhs, rtol=1e-12, max_its=400, precond="mg")
    assert st.converged
    assert _rel(u.cpu().numpy(), ref) <= 1e-9


@pytest.mark.parametrize("precision", ("fp64", "mixed"))
def test_fast_diagonalisation_on_separable_stretched_grid(precision):
    """Constant mu, y(iy) and z(iz) stretched independently: the separable part
    is exact except for the mu3 column, so CG converges in a few iterations."""
    import scipy.sparse.linalg as spla
    from scycle_b200.configs import tanh_stretch
    from scycle_b200.sbp import SbpOps
    Ny, Nz = 121, 97
    y = np.repeat(tanh_stretch(Ny, 30.0, 2.0), Nz)
    z = np.tile(tanh_stretch(Nz, 24.0, 2.0), Ny)
    mu = np.full(Ny * Nz, 32.04)
    dev = SbpOps(4, Ny, Nz, 30.0, 24.0, mu, grid="variableGridSpacing", y=y, z=z)
    ora = OracleSbp(4, Ny, Nz, 30.0, 24.0, mu, grid="variableGridSpacing", y=y, z=z)
    rhs = ora.set_rhs(np.linspace(0, 1, Nz) ** 2, np.full(Nz, 0.3), np.zeros(Ny), np.zeros(Ny))
    ref = spla.spsolve(ora.A.tocsc(), rhs)
    u, st = dev.solve(rhs, rtol=1e-13, max_its=100, precision=precision, precond="fd")
    assert st.converged and st.iterations <= (12 if precision == "fp64" else 20)
    assert _rel(u.cpu().numpy(), ref) <= 1e-10


def test_fast_diagonalisation_of_a_product_shear_modulus():
    """mu = a(y) b(z) (here b spans two decades, a a factor three): the
    fast diagonalisation fits log mu as alpha(y) + beta(z) and weights the
    two directions' operators and masses by the fitted factors, which makes
    it exact for a product up to the mu3 column, so CG needs few
    iterations where the plain averages of mu would not be close."""
    import scipy.sparse.linalg as spla
    from scycle_b200.sbp import SbpOps
    Ny, Nz = 81, 73
    yy = np.linspace(0.0, 1.0, Ny)[:, None]
    zz = np.linspace(0.0, 1.0, Nz)[None, :]
    mu = (32.04 * (1.0 + 2.0 * yy) * 10.0 ** (2.0 * zz ** 2)).ravel()
    dev = SbpOps(4, Ny, Nz, 30.0, 24.0, mu)
    ora = OracleSbp(4, Ny, Nz, 30.0, 24.0, mu)
    rhs = ora.set_rhs(np.linspace(0, 1, Nz), np.full(Nz, 0.3), np.zeros(Ny), np.zeros(Ny))
    ref = spla.spsolve(ora.A.tocsc(), rhs)
    u, st = dev.solve(rhs, rtol=1e-12, max_its=200, precond="fd")
    assert st.converged and st.iterations <= 40, st.iterations
    assert _rel(u.cpu().numpy(), ref) <= 1e-9


def test_change_bc_types_rebuilds_operator():
    dev, ora, rng = _case(4, "constantGridSpacing", 45, 37)
    dev.change_bc_types("Neumann", "Neumann", "Neumann", "Neumann")
    ora.change_bc_types("Neumann", "Neumann", "Neumann", "Neumann")
    x = rng.standard_normal(dev.N)
    assert _rel(dev.apply("A", x).cpu().numpy(), ora.A @ x) <= 1e-13


def test_solve_warm_start_converges_immediately():
    dev, ora, rng = _case(4, "constantGridSpacing", 65, 65)
    rhs = ora.set_rhs(np.ones(65), np.zeros(65), np.zeros(65), np.zeros(65))
    u, st = dev.solve(rhs, rtol=1e-11)
    u2, st2 = dev.solve(rhs, u0=u, rtol=1e-11)
    # one batch of iterations runs before the first read-back; from a
    # converged start it changes nothing
    assert st2.iterations <= 1 and st2.converged
    # the extra iteration may still improve an rtol-1e-11 solution slightly
    assert np.abs(u2.cpu().numpy() - u.cpu().numpy()).max() <= 1e-9 * np.abs(u.cpu().numpy()).max()
