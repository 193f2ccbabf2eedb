"""ctypes declarations of the fault / quasi-dynamic driver entry points."""
import ctypes as C

from . import _lib as S

dptr = C.POINTER(C.c_double)


class FaultDesc(C.Structure):
    _fields_ = [("Nz", C.c_int), ("a", dptr), ("b", dptr), ("sN", dptr), ("Dc", dptr), ("eta", dptr),
                ("locked", dptr), ("prestress", dptr), ("f0", C.c_double), ("v0", C.c_double), ("vL", C.c_double),
                ("root_tol", C.c_double), ("max_its", C.c_int), ("state_law", C.c_int), ("exact_jacobian", C.c_int)]


class QDDesc(C.Structure):
    _fields_ = [("grid", S.GridDesc), ("fault", FaultDesc), ("fault_type_scale", C.c_double),
                ("bcL_from_slip", C.c_int), ("bcR_remote", C.c_int), ("vL", C.c_double), ("bcL0", dptr),
                ("bcRShift", dptr), ("solve", S.SolveOpts)]


class OdeOpts(C.Structure):
    _fields_ = [("method", C.c_int), ("control", C.c_int), ("norm", C.c_int), ("tol", C.c_double),
                ("min_dt", C.c_double), ("max_dt", C.c_double), ("init_dt", C.c_double), ("t0", C.c_double),
                ("t1", C.c_double), ("max_steps", C.c_long), ("n_err", C.c_int), ("err_keys", C.c_int * 4),
                ("err_scale", C.c_double * 4)]


class OdeStats(C.Structure):
    _fields_ = [("t", C.c_double), ("dt", C.c_double), ("new_dt", C.c_double), ("step_count", C.c_long),
                ("rejected", C.c_long), ("d_dt_evals", C.c_long), ("solve_its", C.c_long), ("solves", C.c_long),
                ("errA", C.c_double * 2), ("done", C.c_int)]


FIELDS = {"psi": 0, "slip": 1, "slipVel": 2, "tauP": 3, "tauQSP": 4, "strength": 5, "u": 6, "surfDisp": 7,
          "sxy": 8, "dpsi": 9, "dslip": 10, "gVxy": 11, "gVxz": 12, "sxz": 13, "sdev": 14, "effVisc": 15,
          "T": 16, "Vw": 17, "dT": 18}
BODY_FIELDS = ("u", "sxy", "gVxy", "gVxz", "sxz", "sdev", "effVisc", "T", "dT")
LAWS = {"agingLaw": 0, "slipLaw": 1, "constantState": 2, "flashHeating": 3}


def declare(L):
    vp = C.c_void_p
    L.scy_qd_create.argtypes = [C.POINTER(QDDesc), C.POINTER(vp)]
    L.scy_qd_destroy.argtypes = [vp]
    L.scy_qd_set_stream.argtypes = [vp, vp]
    L.scy_qd_d_dt.argtypes = [vp, C.c_double, vp, vp]
    L.scy_qd_integrate_begin.argtypes = [vp, C.POINTER(OdeOpts), dptr]
    L.scy_qd_integrate_steps.argtypes = [vp, C.c_long, C.POINTER(OdeStats)]
    L.scy_qd_force_attempts.argtypes = [vp, dptr, C.POINTER(C.c_int), C.c_long]
    L.scy_qd_record_attempts.argtypes = [vp, C.c_int]
    L.scy_qd_get_attempts.argtypes = [vp, dptr, C.POINTER(C.c_int), C.c_long, C.POINTER(C.c_long)]
    L.scy_qd_get_step_sizes.argtypes = [vp, dptr, C.c_long, C.POINTER(C.c_long)]
    L.scy_qd_set_output.argtypes = [vp, C.c_char_p, C.c_int, C.c_int, C.c_int]
    L.scy_qd_flush_output.argtypes = [vp]
    L.scy_qd_get_field.argtypes = [vp, C.c_int, dptr]
    L.scy_qd_create_from_in.argtypes = [C.c_char_p, C.POINTER(S.SolveOpts), C.POINTER(vp)]
    L.scy_qd_get_problem.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(OdeOpts)]
    L.scy_qd_integrate_begin_from_in.argtypes = [vp]
    L.scy_qd_set_state.argtypes = [vp, dptr, C.c_int]
    L.scy_qd_set_jacobian.argtypes = [vp, C.c_int]
    L.scy_qd_fault_d_dt.argtypes = [vp, vp, vp, vp]
    L.scy_qd_steady_state_info.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_long)]
    L.scy_qd_steady_state_trace.argtypes = [vp, dptr, C.c_long, C.POINTER(C.c_long)]
    L.scy_qd_set_mode.argtypes = [vp, C.c_int]
    L.scy_pl_create.argtypes = [C.POINTER(QDDesc), vp, C.POINTER(vp)]
    L.scy_qd_state_size.argtypes = [vp, C.POINTER(C.c_long)]
    L.scy_in_problem_field.argtypes = [C.c_char_p, C.c_char_p, dptr, C.c_long, C.POINTER(C.c_long)]
    L.scy_in_problem_info.argtypes = [C.c_char_p, C.POINTER(S.GridDesc), C.POINTER(OdeOpts), C.POINTER(C.c_int),
                                      C.POINTER(C.c_int), C.POINTER(C.c_double)]
    return L


class CycleDesc(C.Structure):
    _fields_ = [("rho", dptr), ("cs", dptr), ("rho_fault", dptr), ("fd_bcR", C.c_int), ("fd_bcT", C.c_int),
                ("fd_bcB", C.c_int), ("deltaT_fd", C.c_double), ("CFL", C.c_double),
                ("trigger_qd2fd", C.c_double), ("trigger_fd2qd", C.c_double), ("limit_qd", C.c_double),
                ("limit_fd", C.c_double), ("max_num_cycles", C.c_int), ("ay_index_quirk", C.c_int)]


class CycleStats(C.Structure):
    _fields_ = [("t", C.c_double), ("dt", C.c_double), ("new_dt", C.c_double), ("dt_fd", C.c_double),
                ("step_count", C.c_long),
                ("phase", C.c_int), ("cycle_count", C.c_int), ("allowed", C.c_int), ("done", C.c_int),
                ("qd_steps", C.c_long), ("fd_steps", C.c_long), ("switches", C.c_long),
                ("last_ratio", C.c_double), ("d_dt_evals", C.c_long), ("solve_its", C.c_long),
                ("solves", C.c_long), ("qd_ms", C.c_double), ("fd_ms", C.c_double)]


PHASES = {0: "qd", 1: "fd", 2: "done"}


def declare_cycle(L):
    vp = C.c_void_p
    L.scy_cycle_create.argtypes = [C.POINTER(QDDesc), C.POINTER(CycleDesc), C.POINTER(vp)]
    L.scy_cycle_create_from_in.argtypes = [C.c_char_p, C.POINTER(S.SolveOpts), C.POINTER(vp)]
    L.scy_cycle_destroy.argtypes = [vp]
    L.scy_cycle_get_problem.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_double),
                                        C.POINTER(OdeOpts)]
    L.scy_cycle_begin.argtypes = [vp, C.POINTER(OdeOpts), dptr]
    L.scy_cycle_begin_from_in.argtypes = [vp]
    L.scy_cycle_run.argtypes = [vp, C.c_long, C.POINTER(CycleStats)]
    L.scy_cycle_get_field.argtypes = [vp, C.c_int, dptr]
    L.scy_cycle_get_switches.argtypes = [vp, C.POINTER(C.c_long), dptr, C.POINTER(C.c_int), C.c_long,
                                         C.POINTER(C.c_long)]
    L.scy_cycle_force_attempts.argtypes = [vp, dptr, C.POINTER(C.c_int), C.c_long]
    L.scy_cycle_record_attempts.argtypes = [vp, C.c_int]
    L.scy_cycle_get_attempts.argtypes = [vp, dptr, C.POINTER(C.c_int), C.c_long, C.POINTER(C.c_long)]
    L.scy_cycle_set_mode.argtypes = [vp, C.c_int]
    L.scy_cycle_set_jacobian.argtypes = [vp, C.c_int]
    L.scy_cycle_set_fd_batch.argtypes = [vp, C.c_int]
    L.scy_cycle_time_kernels.argtypes = [vp, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                         C.POINTER(C.c_double)]
    L.scy_cycle_set_fd_fused.argtypes = [vp, C.c_int]
    L.scy_cycle_set_fd_state.argtypes = [vp, C.c_double, C.c_long, C.c_int] + [dptr] * 10
    L.scy_in_cycle_info.argtypes = [C.c_char_p, C.POINTER(CycleDesc), C.POINTER(C.c_double), dptr, C.c_long,
                                    C.POINTER(C.c_long)]
    return L


class BatchOpts(C.Structure):
    _fields_ = [("precision", C.c_int), ("cg_its", C.c_int), ("graphs", C.c_int), ("concurrent", C.c_int),
                ("exact_jacobian", C.c_int), ("fd_dense", C.c_int), ("transform_planes", C.c_int)]


class BatchStats(C.Structure):
    _fields_ = [("rounds", C.c_long), ("redo_rounds", C.c_long), ("graph_launches", C.c_long),
                ("instance_steps", C.c_long), ("stage_solves", C.c_long), ("cg_its", C.c_int), ("groups", C.c_int),
                ("done", C.c_int)]


def declare_batch(L):
    L.scy_batch_tuning.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                                   C.POINTER(C.c_double)]
    L.scy_batch_operator_form.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    vp = C.c_void_p
    L.scy_batch_create_from_in.argtypes = [C.c_int, C.POINTER(C.c_char_p), C.POINTER(S.SolveOpts),
                                           C.POINTER(BatchOpts), C.POINTER(vp)]
    L.scy_batch_destroy.argtypes = [vp]
    L.scy_batch_info.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.scy_batch_instance.argtypes = [vp, C.c_int, C.POINTER(vp)]
    L.scy_batch_run.argtypes = [vp, C.c_long, C.POINTER(BatchStats)]
    L.scy_batch_state_size.argtypes = [vp, C.POINTER(C.c_long)]
    L.scy_batch_set_states.argtypes = [vp, dptr]
    L.scy_batch_get_fault_field.argtypes = [vp, C.c_int, dptr]
    L.scy_batch_set_graphs.argtypes = [vp, C.c_int]
    L.scy_batch_set_sweep_test.argtypes = [vp, C.c_int, C.c_int]
    L.scy_batch_profile.argtypes = [vp, C.c_int]
    L.scy_batch_profile_collect.argtypes = [vp, C.c_int, dptr, C.POINTER(C.c_longlong), dptr]
    L.scy_batch_profile_clear.argtypes = [vp]
