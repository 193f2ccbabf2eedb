"""The CPU reference arm of bench.py: the oracle over several instances in
rounds of one instance per worker, with untimed warm-up steps before the
timed ones in the same integration."""
import importlib
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    # imported by name, so that the pool's spawned workers find its functions
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    return importlib.import_module("bench")


def test_reference_pool_counts_only_the_timed_steps():
    bench = _bench()
    steps, warm = 3, 2
    r = bench.oracle_on_all_cores("c1", steps, n=25, max_workers=2, instances=3, warm=warm)
    assert r["instances"] == 3 and r["rounds"] == 2 and r["workers"] == 2
    # RK32: three evaluations per accepted step (the first stage reuses the
    # last one), more for rejected attempts; the initial evaluation belongs
    # to the warm-up
    assert r["stage_solves"] >= 3 * steps * 3
    assert r["stage_solves"] % 3 == 0
    assert r["timed_s_sum_of_rounds"] >= r["timed_s_max"] > 0
    assert r["value"] == pytest.approx(r["stage_solves"] / r["timed_s_sum_of_rounds"])
    # without a warm-up the initial evaluation is timed too
    r0 = bench.oracle_on_all_cores("c1", steps, n=25, max_workers=1, instances=1)
    assert r0["stage_solves"] % 3 == 1 and r0["rounds"] == 1


def test_both_arms_share_the_workload_config():
    bench = _bench()

    class A:
        batch, n = 32, 401

    cfg = bench.batch_config(A, 1)
    assert cfg["instances_per_gpu"] == 32 and cfg["Ny"] == cfg["Nz"] == 401
    assert cfg["workload"] == bench.BATCH_WORKLOAD % 32
    assert "solver" not in cfg and "l2" not in cfg
