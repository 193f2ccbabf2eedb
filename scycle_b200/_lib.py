"""ctypes binding of libscycle_b200.so (the C ABI in include/scycle_b200.h).

The shared library is built in-tree by ``scycle_b200.build``; loading fails
loudly if it is missing.  Device pointers are passed as integers (e.g.
``tensor.data_ptr()`` of a CUDA tensor).
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libscycle_b200.so")

SCY_OK = 0
STATUS_NAMES = {0: "OK", 1: "ERR_ARG", 2: "ERR_CUDA", 3: "ERR_NOMEM", 4: "ERR_ROOT_NOCONV", 5: "ERR_NONFINITE",
                6: "ERR_CG_NOCONV", 7: "ERR_DT_UNDERFLOW", 8: "ERR_STATE", 9: "ERR_IO", 10: "ERR_TIMEOUT"}
BC = {"Dirichlet": 0, "Neumann": 1}
GRID = {"constantGridSpacing": 0, "variableGridSpacing": 1}
COMPAT = {"fullyCompatible": 0, "compatible": 1}
OPS = {"A": 0, "Dy": 1, "Dz": 2, "muxDy": 3, "muxDz": 4, "H": 5, "Hinv": 6, "Dyxmu": 7, "Dzxmu": 8}
PREC = {"fp64": 0, "mixed": 1, "tf32": 2}
PRECOND = {"auto": 0, "mg": 1, "fd": 2}

dptr = C.POINTER(C.c_double)


class GridDesc(C.Structure):
    _fields_ = [("order", C.c_int), ("Ny", C.c_int), ("Nz", C.c_int), ("Ly", C.c_double), ("Lz", C.c_double),
                ("grid_type", C.c_int), ("compat", C.c_int), ("y", dptr), ("z", dptr), ("mu", dptr),
                ("bcR", C.c_int), ("bcT", C.c_int), ("bcL", C.c_int), ("bcB", C.c_int)]


class SolveOpts(C.Structure):
    _fields_ = [("rtol", C.c_double), ("atol", C.c_double), ("max_its", C.c_int), ("precision", C.c_int),
                ("nonzero_guess", C.c_int), ("check_every", C.c_int), ("precond", C.c_int), ("verify", C.c_int)]


class SolveStats(C.Structure):
    _fields_ = [("iterations", C.c_int), ("converged", C.c_int), ("rnorm0", C.c_double), ("rnorm", C.c_double),
                ("bnorm", C.c_double)]


class ScyError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("%s: %s" % (STATUS_NAMES.get(status, status), msg))
        self.status = status


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libscycle_b200.so is not built (run python -m scycle_b200.build)")
        L = C.CDLL(LIB_PATH)
        L.scy_get_last_error.restype = C.c_char_p
        L.scy_version.restype = C.c_char_p
        vp = C.c_void_p
        L.scy_sbp_create.argtypes = [C.POINTER(GridDesc), C.POINTER(vp)]
        L.scy_sbp_destroy.argtypes = [vp]
        L.scy_sbp_set_stream.argtypes = [vp, vp]
        L.scy_sbp_synchronize.argtypes = [vp]
        L.scy_sbp_change_bc_types.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int]
        L.scy_sbp_apply.argtypes = [vp, C.c_int, vp, vp]
        L.scy_sbp_set_rhs.argtypes = [vp, vp, vp, vp, vp, vp]
        L.scy_sbp_solve.argtypes = [vp, vp, vp, C.POINTER(SolveOpts), C.POINTER(SolveStats)]
        L.scy_sbp_solve_noalloc.argtypes = [vp, vp, vp, C.POINTER(SolveOpts), C.POINTER(SolveStats)]
        L.scy_sbp_info.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.scy_grid_host_apply.argtypes = [C.POINTER(GridDesc), dptr, dptr]
        L.scy_grid_host_apply_cross.argtypes = [C.POINTER(GridDesc), dptr, dptr]
        L.scy_grid_host_apply_full.argtypes = [C.POINTER(GridDesc), dptr, dptr]
        L.scy_ozaki_matmul.argtypes = [vp, C.c_long, C.c_int, C.c_int, dptr, C.c_long, C.c_int, C.c_int, vp,
                                       C.c_long, C.c_int, C.c_int]
        L.scy_launch_count.restype = C.c_longlong
        L.scy_profile_enable.argtypes = [C.c_int]
        L.scy_profile_collect.argtypes = [C.c_int, C.c_int, dptr, C.POINTER(C.c_longlong), dptr]
        _declare_extra(L)
        _lib = L
    return _lib


def _declare_extra(L):
    """Hook for entry points declared by other modules of the package."""
    from . import _lib_ext  # noqa: F401  (adds argtypes for the fault / driver API)
    _lib_ext.declare(L)
    _lib_ext.declare_cycle(L)
    _lib_ext.declare_batch(L)


def check(status):
    if status != SCY_OK:
        raise ScyError(status, lib().scy_get_last_error().decode(errors="replace"))


def as_dptr(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(dptr)


def grid_desc(order, Ny, Nz, Ly, Lz, mu, grid="constantGridSpacing", y=None, z=None, compat="fullyCompatible",
              bcs=("Dirichlet", "Neumann", "Dirichlet", "Neumann")):
    """Builds a GridDesc; returns (desc, keepalive list of arrays)."""
    mu = np.ascontiguousarray(mu, dtype=np.float64)
    keep = [mu]
    d = GridDesc()
    d.order, d.Ny, d.Nz, d.Ly, d.Lz = order, Ny, Nz, Ly, Lz
    d.grid_type = GRID[grid] if isinstance(grid, str) else int(grid)
    d.compat = COMPAT[compat] if isinstance(compat, str) else int(compat)
    d.mu = as_dptr(mu)
    for nm, arr in (("y", y), ("z", z)):
        if arr is not None:
            a = np.ascontiguousarray(arr, dtype=np.float64)
            keep.append(a)
            setattr(d, nm, as_dptr(a))
    b = [BC[x] if isinstance(x, str) else int(x) for x in bcs]
    d.bcR, d.bcT, d.bcL, d.bcB = b
    return d, keep


def host_apply(desc, x, form="stages"):
    """A x on the host: the two-stage form of the device stencil ("stages"),
    the per-node cross-stencil form of the batched ensemble ("cross") or the
    full form with line classes ("full")."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.zeros_like(x)
    f = {"stages": lib().scy_grid_host_apply, "cross": lib().scy_grid_host_apply_cross,
         "full": lib().scy_grid_host_apply_full}[form]
    check(f(C.byref(desc), as_dptr(x), as_dptr(out)))
    return out
