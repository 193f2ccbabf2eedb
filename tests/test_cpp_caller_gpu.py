"""A compiled C++ caller of the library (tests/cpp/adapter_driver.cpp through
include/scycle_b200.hpp, the reference's SbpOps interface and a whole
driver over the C ABI) against the Python binding of the same calls and
against the oracle.  The compile check runs without a GPU."""
import os
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIBDIR = os.path.join(ROOT, "scycle_b200")


def _build(tmp_path):
    exe = str(tmp_path / "adapter_driver")
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(cuda, "include"), os.path.join(HERE, "cpp", "adapter_driver.cpp"),
           "-L", LIBDIR, "-lscycle_b200", "-L", os.path.join(cuda, "lib64"), "-lcudart",
           "-Wl,-rpath," + LIBDIR, "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_cpp_caller_compiles(tmp_path):
    from scycle_b200 import build
    build.build(verbose=False)
    exe = _build(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr


@pytest.mark.gpu
def test_cpp_caller_sbp_ops_matches_binding_and_oracle(tmp_path):
    import scipy.sparse.linalg as spla
    from oracle.sbp2d import SbpOps as OracleSbp
    from scycle_b200.sbp import SbpOps
    exe = _build(tmp_path)
    Ny, Nz = 45, 37
    out = str(tmp_path / "sbp.bin")
    r = subprocess.run([exe, "sbp", str(Ny), str(Nz), out], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    N = Ny * Nz
    got = np.fromfile(out, dtype=np.float64).reshape(5, N)
    mu = (32.04 + 0.01 * np.arange(Ny)[:, None] + 0.0 * np.arange(Nz)[None, :]).ravel()
    x = np.sin(0.1 * np.arange(N))
    dev = SbpOps(4, Ny, Nz, 30.0, 30.0, mu)
    for row, op in zip(got[:4], ("muxDy", "Dz", "A", "H")):
        assert np.array_equal(row, dev.apply(op, x).cpu().numpy()), op
    ora = OracleSbp(4, Ny, Nz, 30.0, 30.0, mu)
    rhs = ora.set_rhs(np.ones(Nz), np.full(Nz, 0.5), np.zeros(Ny), np.zeros(Ny))
    ref = spla.spsolve(ora.A.tocsc(), rhs)
    assert np.linalg.norm(got[4] - ref) <= 1e-9 * np.linalg.norm(ref)
    assert np.linalg.norm(got[2] - ora.A @ x) <= 1e-13 * np.linalg.norm(ora.A @ x)


@pytest.mark.gpu
def test_cpp_caller_driver_matches_binding(tmp_path):
    from scycle_b200.configs import make_qd_problem
    from scycle_b200.qd import QD
    exe = _build(tmp_path)
    path = make_qd_problem(str(tmp_path / "p"), Ny=33, Nz=33, seed=2, name="cpp")
    out = str(tmp_path / "qd.bin")
    r = subprocess.run([exe, "qd", path, "20", out], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = np.fromfile(out, dtype=np.float64).reshape(3, 33)
    q = QD.from_in(path, solve_rtol=1e-12, solve_max_its=300)
    q.integrate_begin_from_in()
    st = q.integrate_steps(20)
    assert st.step_count == 20
    for row, f in zip(got, ("slip", "slipVel", "psi")):
        assert np.array_equal(row, q.field(f)), f
