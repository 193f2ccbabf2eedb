"""Operator tables of the device stencil vs the oracle's assembled matrix (CPU only).

scy_grid_host_apply evaluates A*x on the host from exactly the banded tables
and coefficient fields the device kernel reads, so this pins the table
construction (restating source/spmat.cpp and source/sbpOps_m_*Grid.cpp)
without a GPU.
"""
import itertools

import numpy as np
import pytest

from oracle.sbp2d import SbpOps
from scycle_b200 import _lib as S

BCS = [("Dirichlet", "Neumann", "Dirichlet", "Neumann"), ("Neumann", "Dirichlet", "Neumann", "Dirichlet"),
       ("Dirichlet", "Dirichlet", "Dirichlet", "Dirichlet"), ("Neumann", "Neumann", "Dirichlet", "Neumann")]


def _grid(Ny, Nz, Ly, Lz):
    q = np.repeat(np.arange(Ny) / (Ny - 1), Nz)
    r = np.tile(np.arange(Nz) / (Nz - 1), Ny)
    return Ly * np.sinh(2 * q) / np.sinh(2), Lz * (r + 0.1 * r * r) / 1.1


@pytest.mark.parametrize("order,grid,compat,bcs,shape", list(itertools.product(
    (2, 4), ("constantGridSpacing", "variableGridSpacing"), ("fullyCompatible", "compatible"), BCS,
    [(13, 17), (21, 11), (9, 9)])))
def test_host_tables_match_assembled_A(order, grid, compat, bcs, shape):
    Ny, Nz = shape
    rng = np.random.default_rng(Ny * 100 + Nz)
    Ly, Lz = 3.0, 2.0
    y, z = _grid(Ny, Nz, Ly, Lz)
    mu = 30 + rng.random(Ny * Nz)
    var = grid == "variableGridSpacing"
    op = SbpOps(order, Ny, Nz, Ly, Lz, mu, grid=grid, y=y if var else None, z=z if var else None,
                compat=compat, bcs=bcs)
    d, keep = S.grid_desc(order, Ny, Nz, Ly, Lz, mu, grid, y if var else None, z if var else None, compat, bcs)
    x = rng.standard_normal(Ny * Nz)
    a = op.A @ x
    b = S.host_apply(d, x)
    assert np.abs(a - b).max() <= 1e-13 * np.abs(a).max()
    # the per-node cross-stencil form of the batched ensemble: the same operator
    c = S.host_apply(d, x, form="cross")
    assert np.abs(a - c).max() <= 1e-13 * np.abs(a).max()


@pytest.mark.parametrize("grid,bcs,shape,mu_kind", list(itertools.product(
    ("constantGridSpacing", "variableGridSpacing"), BCS, [(17, 17), (25, 19), (40, 33)],
    ("constant", "one_column", "one_row"))))
def test_full_form_matches_assembled_A(grid, bcs, shape, mu_kind):
    """The full form (one 17-point stencil per row and per column, a table
    per class of lines, 9-point on the interior box) that the operator kernels
    apply on separable levels, against the oracle's assembled matrix: constant
    mu (only the corner lines of the flattened-index m3 average are
    exceptional), and mu constant but for one column or one row (one more
    exceptional line)."""
    Ny, Nz = shape
    rng = np.random.default_rng(Ny * 7 + Nz)
    Ly, Lz = 3.0, 2.0
    y, z = _grid(Ny, Nz, Ly, Lz)
    mu = np.full(Ny * Nz, 32.04)
    if mu_kind == "one_column":
        mu.reshape(Ny, Nz)[:, Nz // 3] = 27.5
    elif mu_kind == "one_row":
        mu.reshape(Ny, Nz)[Ny // 3, :] = 27.5
    var = grid == "variableGridSpacing"
    op = SbpOps(4, Ny, Nz, Ly, Lz, mu, grid=grid, y=y if var else None, z=z if var else None, bcs=bcs)
    d, keep = S.grid_desc(4, Ny, Nz, Ly, Lz, mu, grid, y if var else None, z if var else None, "fullyCompatible",
                          bcs)
    x = rng.standard_normal(Ny * Nz)
    a = op.A @ x
    f = S.host_apply(d, x, form="full")
    assert np.abs(a - f).max() <= 1e-13 * np.abs(a).max()


def test_full_form_absent_for_nonseparable_mu():
    d, keep = S.grid_desc(4, 21, 21, 1.0, 1.0, 30 + np.random.default_rng(0).random(21 * 21))
    with pytest.raises(S.ScyError, match="no full form"):
        S.host_apply(d, np.zeros(21 * 21), form="full")


def test_host_apply_rejects_small_order4_grid():
    d, keep = S.grid_desc(4, 8, 12, 1.0, 1.0, np.ones(96))
    with pytest.raises(S.ScyError):
        S.host_apply(d, np.zeros(96))


def test_library_exports_every_declared_symbol():
    import re
    import os
    hdr = open(os.path.join(os.path.dirname(S.HERE), "include", "scycle_b200.h")).read()
    names = set(re.findall(r"\b(scy_[a-z0-9_]+)\s*\(", hdr))
    names -= {n for n in names if n.endswith("_t")}
    assert names
    L = S.lib()
    missing = [n for n in sorted(names) if not hasattr(L, n)]
    assert not missing, missing
