"""Seeded synthetic workloads in the reference's ``.in`` format.

Each builder writes an ``.in`` file plus the PETSc-binary per-node fields it
names under ``inputDir`` (big-endian int32 class id 1211214, int32 length,
big-endian float64 values), exactly what ``Domain``/``Fault`` read with
``loadVecFromInputFile`` (source/genFuncs.cpp:380-410).

Workloads (no public dataset is involved; all inputs are seeded synthetic):

* ``aging_const_101``: order-4 constant grid 101x101 on Ly=Lz=30 km, mu 32.04
  GPa, rho 2.67 g/cm^3, sN 50 MPa, f0 0.6, v0 1e-6 m/s, a 0.010, b 0.015
  above 12 km falling to 0.005 at 17 km, Dc 8 mm, vL 1e-9 m/s, free
  surface / remote loading / symmetric fault, psi = f0 + N(0, 1e-4), RK32
  with absolute tolerance 1e-7 over 200 simulated years.
* ``slip_var_401``: the same friction profile on a 401x401 grid stretched
  toward the fault and the surface (y/z coordinate files), slip law, Dc
  lognormal per node (mean 8 mm, sigma_ln 0.2) supplied as ``inputDir/Dc``.
"""
import os
import struct

import numpy as np

YEAR = 31557600.0
VEC_FILE_CLASSID = 1211214


def write_petsc_vec(path, vec):
    vec = np.asarray(vec, dtype=np.float64)
    with open(path, "wb") as f:
        f.write(struct.pack(">ii", VEC_FILE_CLASSID, vec.size))
        f.write(vec.astype(">f8").tobytes())


_COMMON = """\
# seeded synthetic quasi-dynamic strike-slip problem
order = {order}
Ny = {Ny}
Nz = {Nz}
Ly = {Ly}
Lz = {Lz}
vL = 1e-9
gridSpacingType = {grid}
inputDir = {inputDir}
outputDir = {outputDir}
bulkDeformationType = linearElastic
momentumBalanceType = {mbt}
stateLaw = {stateLaw}
guessSteadyStateICs = {guess}
f0 = 0.6
v0 = 1e-6
DcVals = [0.008 0.008]
DcDepths = [0 {Lz}]
aVals = [0.010 0.010]
aDepths = [0 {Lz}]
bVals = [0.015 0.015 0.005 0.005]
bDepths = [0 12 17 {Lz}]
sNVals = [50 50]
sNDepths = [0 {Lz}]
muVals = [32.04 32.04]
muDepths = [0 {Lz}]
rhoVals = [2.67 2.67]
rhoDepths = [0 {Lz}]
timeIntegrator = {integrator}
timeControlType = PID
stride1D = 0
stride2D = 0
maxStepCount = {maxStepCount}
initTime = 0
maxTime = {maxTime}
initDeltaT = {initDeltaT}
timeStepTol = {tol}
timeIntInds = [psi slip]
"""


def tanh_stretch(n, L, beta):
    """Coordinates 0..L clustered at 0: L*(1 - tanh(beta*(1-q))/tanh(beta))."""
    q = np.arange(n) / (n - 1.0)
    return L * (1.0 - np.tanh(beta * (1.0 - q)) / np.tanh(beta))


def make_qd_problem(workdir, Ny=101, Nz=101, Ly=30.0, Lz=30.0, order=4, seed=0,
                    grid="constantGridSpacing", state_law="agingLaw", integrator="RK32",
                    tol=1e-7, years=200.0, max_steps=100000000, init_dt=1e-3,
                    stretch_beta=None, dc_lognormal=False, name="qd", guess_ss=0,
                    mbt="quasidynamic", extra=None):
    """Write ``<workdir>/<name>.in`` and its inputDir fields; return the .in path."""
    os.makedirs(workdir, exist_ok=True)
    rng = np.random.default_rng(seed)
    input_dir = os.path.join(workdir, name + "_in_")
    out_dir = os.path.join(workdir, name + "_out_")
    text = _COMMON.format(order=order, Ny=Ny, Nz=Nz, Ly=repr(float(Ly)), Lz=repr(float(Lz)), grid=grid,
                          inputDir=input_dir, outputDir=out_dir, stateLaw=state_law,
                          integrator=integrator, maxStepCount=int(max_steps),
                          maxTime=repr(float(years * YEAR)), initDeltaT=repr(float(init_dt)), tol=repr(float(tol)),
                          guess=int(guess_ss), mbt=mbt)
    if extra:
        text += "".join("%s = %s\n" % (k, v) for k, v in extra.items())
    psi = 0.6 + rng.normal(0.0, 1e-4, size=Nz)
    write_petsc_vec(input_dir + "psi", psi)
    # fields a previous problem of the same name may have left behind
    for nm, keep in (("y", stretch_beta is not None), ("z", stretch_beta is not None), ("Dc", dc_lognormal)):
        if not keep and os.path.exists(input_dir + nm):
            os.remove(input_dir + nm)
    if stretch_beta is not None:
        yv = tanh_stretch(Ny, Ly, stretch_beta)
        zv = tanh_stretch(Nz, Lz, stretch_beta)
        write_petsc_vec(input_dir + "y", np.repeat(yv, Nz))
        write_petsc_vec(input_dir + "z", np.tile(zv, Ny))
    if dc_lognormal:
        sig = 0.2
        mu_ln = np.log(0.008) - 0.5 * sig * sig
        write_petsc_vec(input_dir + "Dc", np.exp(rng.normal(mu_ln, sig, size=Nz)))
    path = os.path.join(workdir, name + ".in")
    with open(path, "w") as f:
        f.write(text)
    return path


def make_qdfd_problem(workdir, Ny=801, Nz=801, Ly=30.0, Lz=30.0, seed=0, cycles=3, trigger=1e-3,
                      name="qdfd", integrator="RK43", tol=1e-7, years=1000.0, min_dt=1e-3, **kw):
    """Quasi-dynamic / fully dynamic switching (momentumBalanceType
    quasidynamic_and_dynamic): order-4 constant grid, cs = sqrt(32.04/2.67)
    = 3.464 km/s, switch to the wave equation when max(eta V / tau) exceeds
    ``trigger``, CFL-limited fully dynamic step, ``cycles`` full cycles."""
    extra = {"maxNumCycles": int(cycles), "trigger_qd2fd": repr(float(trigger)),
             "trigger_fd2qd": repr(float(trigger)), "minDeltaT": repr(float(min_dt))}
    extra.update(kw.pop("extra", {}) or {})
    args = dict(Ny=Ny, Nz=Nz, Ly=Ly, Lz=Lz, seed=seed, name=name, integrator=integrator, tol=tol,
                years=years, guess_ss=1, mbt="quasidynamic_and_dynamic", extra=extra)
    args.update(kw)
    return make_qd_problem(workdir, **args)


def qdfd_const_801(workdir, seed=0, **kw):
    """801x801 order-4 constant grid on 30 km, three full cycles."""
    return make_qdfd_problem(workdir, Ny=801, Nz=801, seed=seed, name="qdfd_const_801", **kw)


def make_pl_problem(workdir, Ny=101, Nz=101, Ly=30.0, Lz=30.0, seed=0, A=1e-4, n=3.0, Q=135e3,
                    T0=283.0, grad=25.0, name="pl", integrator="RK43", tol=1e-7, years=1000.0,
                    min_dt=1e-3, max_effvisc=1e30, **kw):
    """Power-law viscoelastic quasi-dynamic problem (bulkDeformationType
    powerLaw): dislocation creep with prefactor A (MPa^-n/s), exponent n,
    activation energy Q (J/mol, B = Q/R in kelvin) and a linear geotherm
    T = T0 + grad*z (grad in K/km)."""
    R = 8.314462618
    extra = {"wDislCreep": "yes", "disl_AVals": "[%r %r]" % (A, A), "disl_ADepths": "[0 %r]" % Lz,
             "disl_BVals": "[%r %r]" % (Q / R, Q / R), "disl_BDepths": "[0 %r]" % Lz,
             "disl_nVals": "[%r %r]" % (n, n), "disl_nDepths": "[0 %r]" % Lz,
             "TVals": "[%r %r]" % (T0, T0 + grad * Lz), "TDepths": "[0 %r]" % Lz,
             "maxEffVisc": repr(float(max_effvisc)), "minDeltaT": repr(float(min_dt))}
    extra.update(kw.pop("extra", {}) or {})
    args = dict(Ny=Ny, Nz=Nz, Ly=Ly, Lz=Lz, seed=seed, name=name, integrator=integrator, tol=tol,
                years=years, mbt="quasidynamic", extra=extra)
    args.update(kw)
    path = make_qd_problem(workdir, **args)
    text = open(path).read().replace("bulkDeformationType = linearElastic", "bulkDeformationType = powerLaw")
    with open(path, "w") as f:
        f.write(text)
    return path


def aging_const_101(workdir, seed=0, **kw):
    args = dict(Ny=101, Nz=101, seed=seed, name="aging_const_101")
    args.update(kw)
    return make_qd_problem(workdir, **args)


def slip_var_401(workdir, seed=0, **kw):
    """401x401 stretched grid, slip law, per-node lognormal Dc; starts from the
    steady-state guess (guessSteadyStateICs = 1) so the run is inside the cycle."""
    args = dict(Ny=401, Nz=401, seed=seed, grid="variableGridSpacing", state_law="slipLaw",
                stretch_beta=2.0, dc_lognormal=True, name="slip_var_401", guess_ss=1)
    args.update(kw)
    return make_qd_problem(workdir, **args)


def pl_ensemble_c3(workdir, n_inst=128, seed=0, sizes=(101, 201, 301), Lz=30.0, sigma_ab=0.002, corr_km=2.0,
                   grad_range=(15.0, 30.0), **kw):
    """Ensemble of power-law viscoelastic instances with dislocation creep
    (A = 1e-4 MPa^-n/s, n = 3, Q = 135 kJ/mol): grid sizes split in thirds
    over ``sizes`` (43/43/42 of 128 for 101^2/201^2/301^2), a linear
    geotherm with gradient ~ U(grad_range) K/km per instance, and a - b
    perturbed by a seeded Gaussian random field on the fault (std
    ``sigma_ab``, squared-exponential correlation length ``corr_km``),
    written as inputDir/b.  Returns the .in paths, grouped by size."""
    rng = np.random.default_rng(seed)
    counts = [n_inst // len(sizes) + (1 if i < n_inst % len(sizes) else 0) for i in range(len(sizes))]
    paths = []
    i = 0
    for n, cnt in zip(sizes, counts):
        z = np.arange(n) / (n - 1.0) * Lz
        d = z[:, None] - z[None, :]
        Lc = np.linalg.cholesky(sigma_ab ** 2 * np.exp(-0.5 * (d / corr_km) ** 2) + 1e-12 * np.eye(n))
        b0 = np.interp(z, [0.0, 12.0, 17.0, Lz], [0.015, 0.015, 0.005, 0.005])
        for _ in range(cnt):
            grad = rng.uniform(*grad_range)
            path = make_pl_problem(os.path.join(workdir, "c3_%03d" % i), Ny=n, Nz=n, Lz=Lz, seed=seed * 1000 + i,
                                   grad=grad, name="pl", **kw)
            # a - b + delta: b - delta on the fault
            write_petsc_vec(path[:-len(".in")] + "_in_b", b0 - Lc @ rng.standard_normal(n))
            paths.append(path)
            i += 1
    return paths


C4_DEPTHS = np.linspace(0.0, 30.0, 40)


def adjoint_c4(workdir, seed=0, n=201, name="c4"):
    """201x201 constant-grid aging-law run of the adjoint workload: steady-
    state initial guess, RK32 steps of at most 1e4 s (the 2000 steps stay
    early in the interseismic period), rootTol 1e-14.  a, b and Dc are
    written as inputDir fields equal to their piecewise-linear interpolation
    from 40 depth knots (the same map the gradient is taken through).
    Returns (path, knot matrix P, [a, b, Dc] knot values)."""
    from .adjoint import knot_matrix
    path = make_qd_problem(workdir, Ny=n, Nz=n, seed=seed, state_law="agingLaw", integrator="RK32", guess_ss=1,
                           name=name, extra={"maxDeltaT": "1e4", "rootTol": "1e-14"})
    z = np.arange(n) / (n - 1.0) * 30.0
    prof = {"a": np.interp(z, [0.0, 30.0], [0.010, 0.010]),
            "b": np.interp(z, [0.0, 12.0, 17.0, 30.0], [0.015, 0.015, 0.005, 0.005]),
            "Dc": np.full(n, 0.008)}
    P = knot_matrix(z, C4_DEPTHS)
    base_k = [np.interp(C4_DEPTHS, z, prof[k]) for k in ("a", "b", "Dc")]
    for nm, k in zip(("a", "b", "Dc"), base_k):
        write_petsc_vec(path[:-len(".in")] + "_in_" + nm, P @ k)
    return path, P, base_k
