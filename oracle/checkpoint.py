"""Checkpoint files of the linear-elastic quasi-dynamic driver (oracle; test
infrastructure only).

Reads the files a checkpointing run leaves in its outputDir and builds the
problem of the restarted run, as the reference does:

* StrikeSlip_LinearElastic_qd::writeCheckpoint
  (source/strikeSlip_linearElastic_qd.cpp:527-557) writes ckptNumber and the
  ASCII scalars chkpt_currT, chkpt_stepCount, chkpt_prevErr, chkpt_currErr,
  chkpt_deltaT; LinearElastic::writeCheckpoint (linearElastic.cpp:689-) the
  PETSc-binary chkpt_momBal_bc{R,RShift,T,L,B}; Fault::writeCheckpoint
  (fault.cpp:561-584) chkpt_{slip,slipVel,psi,sNEff,sN,tau,tauQS,prestress}.
* A restart (ctor :33-39, LinearElastic::loadCheckpoint :396-410,
  Fault::loadCheckpoint fault.cpp:144-166): initTime and initDeltaT from the
  checkpoint, no steady-state guess, the boundary data, state, normal stress
  and prestress from the files; initiateIntegrand then takes the slip as
  bcL times the fault-type scale (:377-413).  integrate (:727-738) calls
  timeMonitor(initTime, initDeltaT, 0) before reading the step count and the
  error history back, which sets the step count to 0 and rewrites the files
  with the fresh integrator's zero errors: the restarted run counts from 0
  with an empty error history, as a fresh AdaptiveRK does.
"""
import copy

from .infile import read_petsc_vecs

SCALARS = ("ckptNumber", "chkpt_currT", "chkpt_stepCount", "chkpt_prevErr", "chkpt_currErr", "chkpt_deltaT")
VECS = ("slip", "slipVel", "psi", "sNEff", "sN", "tau", "tauQS", "prestress", "momBal_bcR", "momBal_bcRShift",
        "momBal_bcT", "momBal_bcL", "momBal_bcB")


def read_checkpoint(out_prefix):
    """The checkpoint under outputDir ``out_prefix`` (a path prefix that
    file names are appended to, as the reference's outputDir is)."""
    ck = {}
    for nm in SCALARS:
        ck[nm] = float(open(out_prefix + nm).read().split()[0])
    for nm in VECS:
        ck[nm] = read_petsc_vecs(out_prefix + "chkpt_" + nm)[0]
    return ck


def restart_problem(P, ck):
    """The problem of the run restarted from checkpoint ``ck``."""
    P2 = copy.deepcopy(P)
    s = P2["driver"]
    s["initTime"] = ck["chkpt_currT"]
    s["initDeltaT"] = ck["chkpt_deltaT"]
    s["guessSteadyStateICs"] = 0
    P2["psi"] = ck["psi"].copy()
    P2["sN"] = ck["sNEff"].copy()
    P2["prestress"] = ck["prestress"].copy()
    P2["bcL0"] = ck["momBal_bcL"].copy()
    P2["bcRShift"] = ck["momBal_bcRShift"].copy()
    return P2
