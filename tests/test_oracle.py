"""Pins of the oracle against the reference's own known answers and fixtures (CPU).

* TestRoots known-answer residual (reference source/rootFinder.cpp:12-24)
* the manufactured solution of LinearElastic (source/linearElastic.cpp:1049-1128):
  convergence rates of the assembled SBP-SAT operator
* SBP identities the 1D operators are built to satisfy (source/spmat.cpp)
* the reference's example input examples/ex2.in and PETSc-binary vector
  examples/ex3_z, through tests/golden/reference_examples.json
"""
import json
import os

import numpy as np
import pytest
import scipy.sparse.linalg as spla

from oracle.fault import compute_vel_qd, known_answer_resid
from oracle.infile import load_vector_double, load_vector_string, parse_lines, read_petsc_vecs, set_vec, write_petsc_vec
from oracle.sbp1d import sbp_spmat, sbp_spmat4
from oracle.sbp2d import SbpOps

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_examples.json")))


def test_test_roots_known_answer():
    # TestRoots: 0.015*50*asinh(V/2e-6*exp(0.6/0.015)) + 0.5*12*V - tauQS = 0
    tau = 0.75 * (3.000075e+01 - 9.999920e-06)
    one = np.ones(1)
    V, its, conv = compute_vel_qd(one * 1e-3, one * tau, one * 6.0, one * 50.0, one * 0.6, one * 0.015, one * 0.0,
                                  1e-6, 1e-9, root_tol=1e-12)
    assert conv
    root = GOLDEN["test_roots"]["root"]
    assert abs(V[0] - root) <= 1e-10 * root
    assert abs(known_answer_resid(V[0])) <= 1e-12


def _mms(order, n, grid):
    Ny = Nz = n
    Ly = Lz = 2.0
    q = np.repeat(np.arange(Ny) / (Ny - 1), Nz)
    r = np.tile(np.arange(Nz) / (Nz - 1), Ny)
    if grid == "constantGridSpacing":
        y, z, yy, zz = q * Ly, r * Lz, None, None
    else:
        y = Ly * np.sinh(2 * q) / np.sinh(2)
        z = r * Lz
        yy, zz = y, z
    mu = np.sin(y) * np.sin(z) + 30
    op = SbpOps(order, Ny, Nz, Ly, Lz, mu, grid=grid, y=yy, z=zz)
    uA = np.cos(y) * np.sin(z)
    # zzmms_uSource: mu*(u_yy+u_zz) + mu_y*u_y + mu_z*u_z
    f = mu * (-2 * np.cos(y) * np.sin(z)) + np.cos(y) * np.sin(z) * (-np.sin(y) * np.sin(z)) \
        + np.sin(y) * np.cos(z) * np.cos(y) * np.cos(z)
    yL, yR = np.zeros(Nz), np.full(Nz, Ly)
    zc = z[:Nz]
    ys = y[::Nz]
    bcL = np.cos(yL) * np.sin(zc)
    bcR = np.cos(yR) * np.sin(zc)
    bcT = (np.sin(ys) * np.sin(0.0) + 30) * np.cos(ys) * np.cos(0.0)
    bcB = (np.sin(ys) * np.sin(Lz) + 30) * np.cos(ys) * np.cos(Lz)
    rhs = op.set_rhs(bcL, bcR, bcT, bcB)
    Hf = op.H @ f
    if grid != "constantGridSpacing":
        Hf = op.yq_vec * op.zr_vec * Hf
    u = spla.spsolve(op.A.tocsc(), rhs + Hf)
    return np.sqrt(np.mean((u - uA) ** 2)), op


@pytest.mark.parametrize("order,grid,rate", [(2, "constantGridSpacing", 1.9), (4, "constantGridSpacing", 3.3),
                                             (2, "variableGridSpacing", 1.8), (4, "variableGridSpacing", 3.1)])
def test_mms_convergence(order, grid, rate):
    e = [_mms(order, n, grid)[0] for n in (21, 41, 81)]
    rates = np.log2(np.array(e[:-1]) / np.array(e[1:]))
    assert rates.min() >= rate, rates


@pytest.mark.parametrize("order", [2, 4])
def test_operator_is_symmetric(order):
    _, op = _mms(order, 21, "variableGridSpacing")
    A = op.A
    assert abs(A - A.T).max() <= 1e-12 * abs(A).max()


@pytest.mark.parametrize("order,n", [(2, 11), (4, 13), (4, 30)])
def test_sbp_identities(order, n):
    h = 0.37
    o = sbp_spmat(order, n, 1.0 / h)
    Q = o["H"] @ o["D1"]
    B = np.zeros((n, n)); B[0, 0] = -1; B[-1, -1] = 1
    assert np.abs(Q + Q.T - B).max() <= 1e-12
    x = np.arange(n) * h
    for p in range(order // 2 + 1):
        assert np.abs(o["D1"] @ x ** p - p * x ** max(p - 1, 0) * (p > 0)).max() <= 1e-9
    if order == 4:
        D3, D4, C3, C4 = sbp_spmat4(n, 1.0 / h)
        assert np.all(np.abs(D4 @ x ** 3) <= 1e-9)   # 4th differences annihilate cubics


def test_in_parser_semantics():
    assert load_vector_double("[0.010 0.010] # comment") == [0.01, 0.01]
    assert load_vector_double("[5]") == []                 # single entry: the loop never runs
    assert load_vector_double("[1  2]") == [1.0, 0.0, 2.0]  # doubled space reads an empty entry
    assert load_vector_string("[psi slip]") == ["psi", "slip"]
    assert load_vector_string("[slip]") == ["slip"]
    rows = list(parse_lines("Ny = 201 # points\nLy = 30\n"))
    assert rows[0] == ("Ny", "201", "201 # points") and rows[1][1] == "30"


def test_set_vec_interpolates_and_extrapolates():
    z = np.array([0.0, 6.0, 12.0, 14.5, 17.0, 30.0, 40.0])
    v = set_vec(z, [0.015, 0.015, 0.005, 0.005], [0, 12, 17, 30])
    assert np.allclose(v, [0.015, 0.015, 0.015, 0.01, 0.005, 0.005, 0.005])
    w = set_vec(np.array([-1.0, 5.0, 12.0]), [1.0, 2.0], [0.0, 10.0])
    assert np.allclose(w, [1.0, 1.5, 2.2])


def test_petsc_binary_round_trip(tmp_path):
    p = str(tmp_path / "v")
    v = np.linspace(-3, 7, 101)
    write_petsc_vec(p, v)
    write_petsc_vec(p, 2 * v, append=True)
    r = read_petsc_vecs(p)
    assert len(r) == 2 and np.array_equal(r[0], v) and np.array_equal(r[1], 2 * v)
    raw = open(p, "rb").read()
    assert raw[:4] == (1211214).to_bytes(4, "big") and raw[4:8] == (101).to_bytes(4, "big")


def test_ex3_z_fixture_describes_a_column_major_z_grid():
    g = GOLDEN["ex3_z"]
    assert g["records"] == 1 and g["n"] == g["ny_guess"] * g["nz_guess"]
    assert g["min"] == 0.0 and g["max"] == 500.0
    # z restarts at 0 at every new y row: entry nz-1 is Lz and entry nz is 0
    assert g["col_first"][1] == 500.0 and g["col_first"][2] == 0.0
    assert g["first"][0] == 0.0 and all(np.diff(g["first"]) > 0)


def ex2_text(tmp_path=None):
    """The settings of examples/ex2.in rebuilt as an input file."""
    lines = []
    for var, kind, val in GOLDEN["ex2_settings"]:
        if kind == "list":
            lines.append("%s = [%s]" % (var, " ".join(str(x) for x in val)))
        else:
            lines.append("%s = %s" % (var, val))
    return "\n".join(lines) + "\n"


def test_ex2_settings_through_the_oracle():
    from oracle.problem import build_qd_problem
    P = build_qd_problem(ex2_text())
    d = P["domain"]
    assert (d["Ny"], d["Nz"], d["Ly"], d["Lz"]) == (151, 151, 100.0, 30.0)
    assert d["gridSpacingType"] == "variableGridSpacing"   # bCoordTrans > 0 forces it
    assert P["driver"]["guessSteadyStateICs"] == 1 and P["driver"]["timeIntegrator"] == "RK43"
    assert P["driver"]["timeIntInds"] == ["psi", "slip"]
    zf = P["z"][:151]
    assert np.isclose(P["a"][0], 0.0135) and np.isclose(np.interp(11.0, zf, P["a"]), 0.03, rtol=1e-3)
    y = P["y"][::151]
    assert np.isclose(y[-1], 100.0) and np.isclose(y[75], 100 * np.sinh(2.5) / np.sinh(5))
