"""scy_sbp_solve_noalloc: the elliptic solve for callers that cannot allocate.

Some callers cannot call cudaMalloc between time steps: their device memory
is owned by another allocator (a framework's caching pool, a memory manager
that reserved the device up front), or they cannot afford the device
synchronisation an allocation may imply.  This entry point allocates
nothing: its work vectors sit in a fixed array inside the library, which
limits it to grids of at most 65,536 nodes.

The test calls it through the C ABI twice in a row (the array keeps the
previous call's contents, which the second call must not depend on) and
compares each result with scy_sbp_solve's on the same input, to the
tolerance the other solver tests use.  It is collected last so that a run
stopping at the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from oracle.sbp2d import SbpOps as OracleSbp
from scycle_b200 import _lib as S

pytestmark = pytest.mark.gpu


def _solve(fn, sbp, rhs_dev, torch, u0=None, check_every=1, atol=0.0):
    u = torch.zeros_like(rhs_dev) if u0 is None else u0.clone()
    o = S.SolveOpts(1e-12, atol, 5000, S.PREC["fp64"], 0 if u0 is None else 1, check_every)
    st = S.SolveStats()
    torch.cuda.synchronize()
    S.check(fn(sbp.h, C.c_void_p(rhs_dev.data_ptr()), C.c_void_p(u.data_ptr()), C.byref(o), C.byref(st)))
    torch.cuda.synchronize()
    assert st.converged
    # success means the true residual met the target
    assert st.rnorm <= max(1e-12 * st.bnorm, atol) * (1 + 1e-6)
    return u.cpu().numpy()


def test_noalloc_solve_matches_allocating_solve_twice():
    import torch
    from scycle_b200.sbp import SbpOps
    n = 101
    rng = np.random.default_rng(7)
    mu = 32.04 + rng.random(n * n)
    sbp = SbpOps(4, n, n, 30.0, 30.0, mu)
    ora = OracleSbp(4, n, n, 30.0, 30.0, mu)
    L = S.lib()
    for k in range(2):
        bcL = rng.random(n) * (k + 1)
        rhs = ora.set_rhs(bcL, np.full(n, 0.3 * k), np.zeros(n), np.zeros(n))
        rhs_dev = torch.from_numpy(rhs).cuda()
        ref = _solve(L.scy_sbp_solve, sbp, rhs_dev, torch)
        got = _solve(L.scy_sbp_solve_noalloc, sbp, rhs_dev, torch)
        assert np.abs(got - ref).max() <= 1e-9 * np.abs(ref).max()


def test_noalloc_solve_rejects_grids_beyond_its_limit():
    import torch
    from scycle_b200.sbp import SbpOps
    n = 257  # 66,049 nodes > 65,536
    sbp = SbpOps(4, n, n, 30.0, 30.0, np.full(n * n, 32.04))
    rhs = torch.zeros(n * n, dtype=torch.float64, device="cuda")
    u = torch.zeros_like(rhs)
    o = S.SolveOpts(1e-12, 0.0, 10, 0, 0, 1)
    st = S.SolveStats()
    status = S.lib().scy_sbp_solve_noalloc(sbp.h, C.c_void_p(rhs.data_ptr()), C.c_void_p(u.data_ptr()),
                                           C.byref(o), C.byref(st))
    assert status == 1
    assert b"at most 65536" in S.lib().scy_get_last_error()


def test_noalloc_solve_warm_start_check_interval_and_zero_rhs():
    """A warm start (nonzero_guess = 1) checked every 5 iterations gives the
    allocating solve's answer from the same start; a zero right-hand side
    with atol = 0 returns u = 0 from a nonzero start."""
    import torch
    from scycle_b200.sbp import SbpOps
    n = 65
    rng = np.random.default_rng(11)
    mu = 32.04 + rng.random(n * n)
    sbp = SbpOps(4, n, n, 30.0, 30.0, mu)
    ora = OracleSbp(4, n, n, 30.0, 30.0, mu)
    L = S.lib()
    rhs = ora.set_rhs(rng.random(n), np.full(n, 0.2), np.zeros(n), np.zeros(n))
    rhs_dev = torch.from_numpy(rhs).cuda()
    exact = _solve(L.scy_sbp_solve, sbp, rhs_dev, torch)
    u0 = torch.from_numpy(exact * (1.0 + 1e-3 * rng.standard_normal(n * n))).cuda()
    ref = _solve(L.scy_sbp_solve, sbp, rhs_dev, torch, u0=u0, check_every=5)
    got = _solve(L.scy_sbp_solve_noalloc, sbp, rhs_dev, torch, u0=u0, check_every=5)
    assert np.abs(got - ref).max() <= 1e-9 * np.abs(ref).max()
    zero = torch.zeros_like(rhs_dev)
    got0 = _solve(L.scy_sbp_solve_noalloc, sbp, zero, torch, u0=u0)
    assert np.all(got0 == 0.0)


def test_noalloc_solve_leaves_device_memory_unchanged():
    """After one warm-up call (which may load the module on the device),
    further calls change the device's free memory by nothing."""
    import torch
    from scycle_b200.sbp import SbpOps
    n = 81
    rng = np.random.default_rng(3)
    mu = np.full(n * n, 32.04)
    sbp = SbpOps(4, n, n, 30.0, 30.0, mu)
    ora = OracleSbp(4, n, n, 30.0, 30.0, mu)
    L = S.lib()
    rhs_dev = torch.from_numpy(ora.set_rhs(rng.random(n), np.zeros(n), np.zeros(n), np.zeros(n))).cuda()
    u = torch.zeros_like(rhs_dev)
    o = S.SolveOpts(1e-12, 0.0, 5000, S.PREC["fp64"], 0, 1)
    st = S.SolveStats()
    call = lambda: S.check(L.scy_sbp_solve_noalloc(sbp.h, C.c_void_p(rhs_dev.data_ptr()), C.c_void_p(u.data_ptr()),
                                                    C.byref(o), C.byref(st)))
    call()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        call()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
