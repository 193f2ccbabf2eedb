"""An ensemble of independent runs spread over ranks (one process per GPU).

The reference runs one ``StrikeSlip_*_qd`` per process; an ensemble of runs
(different friction profiles, geotherms, grid sizes) has no exchange between
its members, so it shards by instance with no data-path collective: each
rank integrates its share as one batch (``scy_batch_*``) and the per-instance
results are gathered on rank 0 at the end.

The share of each rank comes from a cost estimate per instance,

    cost = Ny * Nz * (Nz + 64) * stages per step * steps,

the work of one stage solve (the two dense z transforms of the
preconditioner, Nz multiply-adds per node each, plus the node-local
kernels, about 64 node operations' worth) times the stage solves the run
is expected to take (3 per RK32 step, 6 per RK43 step).  ``partition``
assigns instances largest-first to the least-loaded rank (the LPT rule), so
an ensemble of mixed grid sizes (e.g. 101^2 / 201^2 / 301^2) balances
within the largest single instance's cost.
"""
import numpy as np

STAGES_PER_STEP = {"RK32": 3, "RK43": 6, "RK32_WBE": 3, "RK43_WBE": 6}


def read_in_settings(path, keys=("Ny", "Nz", "timeIntegrator")):
    """The few .in settings the cost estimate needs (the reference's
    ``key = value`` lines; later lines win, as in its loaders)."""
    out = {}
    with open(path) as f:
        for line in f:
            line = line.split("#", 1)[0]
            if " = " not in line:
                continue
            k, v = line.split(" = ", 1)
            k, v = k.strip(), v.strip()
            if k in keys:
                out[k] = v
    return out


def instance_cost(path, steps=1):
    s = read_in_settings(path)
    ny, nz = int(s.get("Ny", 1)), int(s.get("Nz", 1))
    stages = STAGES_PER_STEP.get(s.get("timeIntegrator", "RK43"), 6)
    return float(ny) * nz * (nz + 64) * stages * steps


def partition(costs, n_ranks):
    """Instance indices per rank: largest cost first, each to the rank with
    the smallest load so far (ties to the lower rank).  Deterministic, so
    every rank computes the same split without communicating."""
    costs = np.asarray(costs, dtype=np.float64)
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * n_ranks
    share = [[] for _ in range(n_ranks)]
    for i in order:
        r = min(range(n_ranks), key=lambda q: (load[q], q))
        share[r].append(i)
        load[r] += costs[i]
    return [sorted(s) for s in share]


def imbalance(costs, shares):
    """max rank load / mean rank load (1.0 = perfect balance)."""
    loads = [sum(costs[i] for i in s) for s in shares]
    mean = sum(loads) / len(loads)
    return max(loads) / mean if mean > 0 else 1.0


def run_ensemble(paths, runner, dist=None, steps=1):
    """Runs the ensemble ``paths`` with ``runner(list_of_paths) -> list of
    per-instance results`` on this rank's share and returns, on rank 0, the
    results in the order of ``paths`` (None on the other ranks).  Without a
    process group (``dist`` None or world size 1) everything runs here."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return list(runner(list(paths)))
    rank, world = dist.get_rank(), dist.get_world_size()
    shares = partition([instance_cost(p, steps) for p in paths], world)
    mine = shares[rank]
    res = list(runner([paths[i] for i in mine])) if mine else []
    gathered = [None] * world if rank == 0 else None
    dist.gather_object(list(zip(mine, res)), gathered, dst=0)
    if rank != 0:
        return None
    out = [None] * len(paths)
    for part in gathered:
        for i, r in part:
            out[i] = r
    return out


def batch_runner(nsteps, fields=("psi", "slip", "slipVel"), **batch_kw):
    """A runner for ``run_ensemble`` on the GPU: one ``Batch`` of the given
    input files advanced ``nsteps`` accepted steps; per instance the final
    time, step count and the listed fault fields."""
    def run(paths):
        from .batch import Batch
        b = Batch(paths, **batch_kw)
        try:
            b.run(nsteps)
            res = []
            for i in range(b.n):
                v = b.instance(i)
                st = v.integrate_steps(0)
                res.append({"t": st.t, "steps": st.step_count, **{f: v.field(f) for f in fields}})
            return res
        finally:
            b.close()
    return run


__all__ = ["instance_cost", "partition", "imbalance", "run_ensemble", "batch_runner", "read_in_settings"]
