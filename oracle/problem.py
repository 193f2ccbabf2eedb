"""Problem set-up from a ``.in`` file (oracle; test infrastructure only).

Restates the settings each reference class reads and the fields it derives:
Domain (source/domain.cpp:8-50, :133-196, :233-262, :352-430), LinearElastic
(source/linearElastic.cpp:8-50, :99-148, :297-323), Fault
(source/fault.cpp:8-141, :200-288), StrikeSlip_LinearElastic_qd
(source/strikeSlip_linearElastic_qd.cpp:7-78, :126-373).  The result is a
plain dict of host arrays consumed by the oracle driver and, in the tests, by
the device path.
"""
import os

import numpy as np

from .infile import (atof, atoi, load_vector_double, load_vector_string, parse_lines,
                     read_petsc_vecs, set_vec)


def _load_vec_file(input_dir, name, n):
    path = input_dir + name
    if os.path.exists(path):
        v = read_petsc_vecs(path)[0]
        if v.size != n:
            raise ValueError("%s holds %d entries, expected %d" % (path, v.size, n))
        return v
    return None


def domain_settings(text):
    """Domain::loadSettings + constructor defaults (domain.cpp:8-16, :133-196, :233-262)."""
    d = dict(inputDir="unspecified_", outputDir="data/", bulkDeformationType="linearElastic",
             momentumBalanceType="quasidynamic", operatorType="matrix-based",
             sbpCompatibilityType="fullyCompatible", gridSpacingType="variableGridSpacing",
             isMMS=0, order=4, Ny=-1, Nz=-1, Ly=-1.0, Lz=-1.0, vL=1e-9, bCoordTrans=-1.0,
             enableCheckpointing=0, interval=10000)
    for var, rhs, _ in parse_lines(text):
        if var == "order": d["order"] = atoi(rhs)
        elif var == "Ny" and d["Ny"] < 0: d["Ny"] = atoi(rhs)
        elif var == "Nz" and d["Nz"] < 0: d["Nz"] = atoi(rhs)
        elif var == "Ly": d["Ly"] = atof(rhs)
        elif var == "Lz": d["Lz"] = atof(rhs)
        elif var == "inputDir": d["inputDir"] = rhs
        elif var == "outputDir": d["outputDir"] = rhs
        elif var == "operatorType": d["operatorType"] = rhs
        elif var == "sbpCompatibilityType": d["sbpCompatibilityType"] = rhs
        elif var == "gridSpacingType": d["gridSpacingType"] = rhs
        elif var == "bulkDeformationType": d["bulkDeformationType"] = rhs
        elif var == "momentumBalanceType": d["momentumBalanceType"] = rhs
        elif var == "isMMS": d["isMMS"] = atoi(rhs)
        elif var == "bCoordTrans": d["bCoordTrans"] = atof(rhs)
        elif var == "vL": d["vL"] = atof(rhs)
        elif var == "enableCheckpointing": d["enableCheckpointing"] = atoi(rhs)
        elif var == "interval": d["interval"] = int(atof(rhs))
    if d["bCoordTrans"] > 0.0:
        d["gridSpacingType"] = "variableGridSpacing"
    return d


def fault_settings(text):
    """Fault::loadSettings + defaults (fault.cpp:8-16, :35-109)."""
    f = dict(stateLaw="agingLaw", f0=0.6, v0=1e-6, sN_cap=1e14, sN_floor=0.0, rootTol=1e-12,
             maxNumIts=10000, fw=0.64, Vw=0.12, D=5.0, tau_c=3.0)
    vecs = {"DcVals", "DcDepths", "sNVals", "sNDepths", "aVals", "aDepths", "bVals", "bDepths",
            "cohesionVals", "cohesionDepths", "muVals", "muDepths", "rhoVals", "rhoDepths",
            "stateVals", "stateDepths", "lockedVals", "lockedDepths", "TwVals", "TwDepths"}
    for k in vecs:
        f[k] = []
    for var, rhs, full in parse_lines(text):
        if var in vecs: f[var] = f[var] + load_vector_double(full)
        elif var == "sN_cap": f["sN_cap"] = atof(rhs)
        elif var == "sN_floor": f["sN_floor"] = atof(rhs)
        elif var == "stateLaw": f["stateLaw"] = rhs
        elif var == "rootTol": f["rootTol"] = atof(rhs)
        elif var == "f0": f["f0"] = atof(rhs)
        elif var == "v0": f["v0"] = atof(rhs)
        elif var in ("fw", "Vw", "D", "tau_c"): f[var] = atof(rhs)  # flash heating (fault.cpp:89-97)
    return f


def material_settings(text):
    """LinearElastic::loadSettings + defaults (linearElastic.cpp:8-16, :99-148)."""
    m = dict(linSolver="MUMPSCHOLESKY", kspTol=1e-10, muVals=[], muDepths=[], rhoVals=[], rhoDepths=[])
    for var, rhs, full in parse_lines(text):
        if var == "linSolver": m["linSolver"] = rhs
        elif var == "kspTol": m["kspTol"] = atof(rhs)
        elif var in ("muVals", "muDepths", "rhoVals", "rhoDepths"): m[var] = m[var] + load_vector_double(full)
    return m


def driver_settings(text):
    """StrikeSlip_LinearElastic_qd::loadSettings + defaults (strikeSlip_linearElastic_qd.cpp:7-20, :126-195)."""
    s = dict(thermalCoupling="no", hydraulicCoupling="no", stateLaw=None, guessSteadyStateICs=0,
             forcingType="no", timeIntegrator="RK43", timeControlType="PID", stride1D=1, stride2D=1,
             maxStepCount=100000000, initTime=0.0, maxTime=1e15, minDeltaT=-1.0, maxDeltaT=1e10,
             initDeltaT=1e-3, timeStepTol=1e-8, timeIntInds=[], scale=[], normType="L2_absolute",
             vL=1e-9, bodyForce=0.0, bcRType="remoteLoading", bcTType="freeSurface",
             bcLType="symmFault", bcBType="freeSurface")
    for var, rhs, full in parse_lines(text):
        if var == "thermalCoupling": s["thermalCoupling"] = rhs
        elif var == "hydraulicCoupling": s["hydraulicCoupling"] = rhs
        elif var == "stateLaw": s["stateLaw"] = rhs
        elif var == "guessSteadyStateICs": s["guessSteadyStateICs"] = atoi(rhs)
        elif var == "forcingType": s["forcingType"] = rhs
        elif var == "timeIntegrator": s["timeIntegrator"] = rhs
        elif var == "timeControlType": s["timeControlType"] = rhs
        elif var == "stride1D": s["stride1D"] = int(atof(rhs))
        elif var == "stride2D": s["stride2D"] = int(atof(rhs))
        elif var == "maxStepCount": s["maxStepCount"] = int(atof(rhs))
        elif var == "initTime": s["initTime"] = atof(rhs)
        elif var == "maxTime": s["maxTime"] = atof(rhs)
        elif var == "minDeltaT": s["minDeltaT"] = atof(rhs)
        elif var == "maxDeltaT": s["maxDeltaT"] = atof(rhs)
        elif var == "initDeltaT": s["initDeltaT"] = atof(rhs)
        elif var == "timeStepTol": s["timeStepTol"] = atof(rhs)
        elif var == "timeIntInds": s["timeIntInds"] = s["timeIntInds"] + load_vector_string(full)
        elif var == "scale": s["scale"] = s["scale"] + load_vector_double(full)
        elif var == "normType": s["normType"] = rhs
        elif var == "vL": s["vL"] = atof(rhs)
        elif var == "bodyForce": s["bodyForce"] = atof(rhs)
        elif var == "momBal_bcR_qd": s["bcRType"] = rhs
        elif var == "momBal_bcT_qd": s["bcTType"] = rhs
        elif var == "momBal_bcL_qd": s["bcLType"] = rhs
        elif var == "momBal_bcB_qd": s["bcBType"] = rhs
    # checkInput runs before computeMinTimeStep, so minDeltaT is still the
    # parsed value here (strikeSlip_linearElastic_qd.cpp:218-220)
    if s["initDeltaT"] < s["minDeltaT"] or s["initDeltaT"] < 1e-14:
        s["initDeltaT"] = s["minDeltaT"]
    return s


def parse_bc(name):
    """parseBCs (strikeSlip_linearElastic_qd.cpp:326-373)."""
    if name in ("symmFault", "rigidFault", "remoteLoading"):
        return "Dirichlet"
    if name in ("freeSurface", "outGoingCharacteristics"):
        return "Neumann"
    raise ValueError(name)


def build_qd_problem(text, input_dir=None):
    """Everything the linear-elastic quasi-dynamic driver needs, as host arrays."""
    d = domain_settings(text)
    if input_dir is not None:
        d["inputDir"] = input_dir
    Ny, Nz = d["Ny"], d["Nz"]
    N = Ny * Nz
    dq = 1.0 / (Ny - 1.0) if Ny > 1 else 1.0
    dr = 1.0 / (Nz - 1.0) if Nz > 1 else 1.0
    Ii = np.arange(N)
    q = dq * (Ii // Nz)
    r = dr * (Ii - Nz * (Ii // Nz))
    y = _load_vec_file(d["inputDir"], "y", N)
    y_loaded = y is not None
    if y is None:
        y = q * d["Ly"] if d["bCoordTrans"] <= 0 else d["Ly"] * np.sinh(d["bCoordTrans"] * q) / np.sinh(d["bCoordTrans"])
    z = _load_vec_file(d["inputDir"], "z", N)
    z_loaded = z is not None
    if z is None:
        z = r * d["Lz"]
    m = material_settings(text)
    mu = set_vec(y, m["muVals"], m["muDepths"])      # mu against y (linearElastic.cpp:353)
    rho = set_vec(z, m["rhoVals"], m["rhoDepths"])   # rho against z (linearElastic.cpp:354)
    for nm, arr in (("momBal_mu", "mu"), ("momBal_rho", "rho")):
        v = _load_vec_file(d["inputDir"], nm, N)
        if v is not None:
            if arr == "mu": mu = v
            else: rho = v
    cs = np.sqrt(np.abs(mu / rho))
    v = _load_vec_file(d["inputDir"], "momBal_cs", N)
    if v is not None:
        cs = v
    f = fault_settings(text)
    zf = z[:Nz].copy()
    a = set_vec(zf, f["aVals"], f["aDepths"])
    b = set_vec(zf, f["bVals"], f["bDepths"])
    sN = set_vec(zf, f["sNVals"], f["sNDepths"])
    Dc = set_vec(zf, f["DcVals"], f["DcDepths"])
    locked = set_vec(zf, f["lockedVals"], f["lockedDepths"]) if f["lockedVals"] else np.zeros(Nz)
    rho_f = set_vec(z, f["rhoVals"], f["rhoDepths"])[:Nz]   # fault.cpp:263-271
    mu_f = set_vec(z, f["muVals"], f["muDepths"])[:Nz]
    psi = set_vec(zf, f["stateVals"], f["stateDepths"]) if f["stateVals"] else np.full(Nz, f["f0"])
    sN = np.maximum(np.minimum(sN, f["sN_cap"]), f["sN_floor"])
    sNEff = sN.copy()
    fin = {}
    for nm in ("sNEff", "psi", "slip", "tauQS", "tau", "prestress", "a", "b", "Dc"):
        fin[nm] = _load_vec_file(d["inputDir"], nm, Nz)
    if fin["sNEff"] is not None: sNEff = fin["sNEff"]
    if fin["psi"] is not None: psi = fin["psi"]
    if fin["a"] is not None: a = fin["a"]
    if fin["b"] is not None: b = fin["b"]
    if fin["Dc"] is not None:
        # per-node Dc is an extension: the reference does not read inputDir/Dc
        Dc = fin["Dc"]
    prestress = fin["prestress"] if fin["prestress"] is not None else np.zeros(Nz)
    s = driver_settings(text)
    if s["stateLaw"] is None:
        s["stateLaw"] = f["stateLaw"]
    bc = {k: parse_bc(s["bc%sType" % k]) for k in "RTLB"}
    fts = 1.0 if s["bcLType"] == "rigidFault" else 2.0
    bcL0 = _load_vec_file(d["inputDir"], "momBal_bcL", Nz)
    bcRShift = _load_vec_file(d["inputDir"], "momBal_bcR", Nz)
    return dict(domain=d, material=m, fault=f, driver=s, N=N, Ny=Ny, Nz=Nz, y=y, z=z, q=q, r=r,
                y_loaded=y_loaded, z_loaded=z_loaded, mu=mu, rho=rho, cs=cs,
                a=a, b=b, sN=sNEff, Dc=Dc, locked=locked, psi=psi, prestress=prestress,
                mu_f=mu_f, rho_f=rho_f, bc=bc, faultTypeScale=fts,
                bcL0=np.zeros(Nz) if bcL0 is None else bcL0,
                bcRShift=np.zeros(Nz) if bcRShift is None else bcRShift)
