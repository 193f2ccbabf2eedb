"""Ensemble sharding over ranks by cost (CPU; world size 2 over gloo).

An ensemble of independent runs is split over ranks by the estimated cost
of each instance (grid size x stage solves) with the largest-first rule;
each rank integrates its share and rank 0 gathers the per-instance results
in the caller's order.  Here the runner is the oracle on CPU, so the whole
path -- split, per-rank runs, gather, reordering -- is checked without a
GPU: the gathered results must equal a single-process run bit for bit.
"""
import os
import socket
import tempfile

import numpy as np
import pytest

from scycle_b200 import configs
from scycle_b200.ensemble import imbalance, instance_cost, partition, run_ensemble


def test_partition_balances_mixed_grid_sizes(tmp_path):
    """128 power-law instances of 101^2 / 201^2 / 301^2 (the ensemble
    configuration's mix) over 2, 4 and 8 ranks."""
    sizes = [101] * 43 + [201] * 43 + [301] * 42
    paths = []
    for i, n in enumerate(sizes):
        p = tmp_path / ("i%03d.in" % i)
        p.write_text("Ny = %d\nNz = %d\ntimeIntegrator = RK43\n" % (n, n))
        paths.append(str(p))
    costs = [instance_cost(p) for p in paths]
    assert costs[-1] > costs[0] > 0
    for world in (2, 4, 8):
        shares = partition(costs, world)
        assert sorted(i for s in shares for i in s) == list(range(len(paths)))
        assert imbalance(costs, shares) <= 1.02, (world, imbalance(costs, shares))
    # deterministic: every rank computes the same split
    assert partition(costs, 8) == partition(list(costs), 8)


def test_partition_of_fewer_instances_than_ranks():
    shares = partition([3.0, 1.0], 4)
    assert shares == [[0], [1], [], []]


def _oracle_runner(nsteps):
    def run(paths):
        from oracle.problem import build_qd_problem
        from oracle.qd import QDLinearElastic
        out = []
        for p in paths:
            P = build_qd_problem(open(p).read())
            ora = QDLinearElastic(P, keep_history=False)
            rk = ora.integrate(max_steps=nsteps)
            out.append({"t": rk.currT, "slip": ora.fault.slip.copy(), "slipVel": ora.fault.slipVel.copy(),
                        "psi": ora.fault.psi.copy()})
        return out
    return run


def _make_paths(work):
    paths = []
    for i, n in enumerate((17, 25, 21, 25, 17, 29)):
        paths.append(configs.make_qd_problem(os.path.join(work, "m%d" % i), Ny=n, Nz=n, seed=i,
                                             integrator="RK32" if i % 2 else "RK43"))
    return paths


def _rank_main(rank, world, port, paths, out):
    import torch.distributed as dist
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        res = run_ensemble(paths, _oracle_runner(6), dist=dist, steps=6)
        if rank == 0:
            np.save(out, np.array(res, dtype=object), allow_pickle=True)
    finally:
        dist.destroy_process_group()


def test_two_ranks_gather_equals_single_process():
    import multiprocessing as mp
    work = tempfile.mkdtemp(prefix="scy_ens_")
    paths = _make_paths(work)
    ref = run_ensemble(paths, _oracle_runner(6))
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    out = os.path.join(work, "gathered.npy")
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, paths, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = list(np.load(out, allow_pickle=True))
    # the split really spreads the work: both ranks own instances
    shares = partition([instance_cost(p, 6) for p in paths], 2)
    assert all(shares)
    assert len(got) == len(ref)
    for a, b in zip(got, ref):
        assert a["t"] == b["t"]
        for k in ("slip", "slipVel", "psi"):
            assert np.array_equal(a[k], b[k]), k
