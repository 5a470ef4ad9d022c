"""ctypes declarations of include/avionic.h (kept in step with the header;
tests/test_abi.py checks that every declared function is exported and bound)."""

import ctypes as C

VP = C.c_void_p
U = C.c_uint
I = C.c_int
F = C.c_float
D = C.c_double


class PDParams(C.Structure):
    _fields_ = [
        ("maxIt", U), ("stopPDGap", F), ("sigma", F), ("tau", F), ("sigmaTauRatio", F),
        ("timeSpaceWeight", F), ("lambda_", F), ("dx", F), ("dy", F), ("dt", F),
        ("alpha0", F), ("alpha1", F), ("alpha", F), ("timeSpaceWeight2", F),
        ("dx2", F), ("dy2", F), ("dt2", F), ("adaptLambda", I), ("adaptK", F), ("adaptD", F),
    ]


class RunStats(C.Structure):
    _fields_ = [
        ("iterations", U), ("sigma", F), ("tau", F), ("gap_count", U), ("last_gap", D),
        ("stopped_by_gap", I), ("elapsed_ms", F), ("kernel_launches", U),
    ]


class CoilParams(C.Structure):
    _fields_ = [
        ("uH1mu", F), ("uReg", F), ("uNrIt", U), ("uTau", F), ("uSigma", F), ("uSigmaTauRatio", F),
        ("uAlpha0", F), ("uAlpha1", F), ("b1Reg", F), ("b1NrIt", U), ("b1Tau", F), ("b1Sigma", F),
        ("b1SigmaTauRatio", F), ("b1FinalReg", F), ("b1FinalNrIt", U),
    ]


class Request(C.Structure):
    """avx_request"""
    _fields_ = [
        ("method", I), ("op_kind", I), ("width", U), ("height", U), ("coils", U), ("frames", U),
        ("params", PDParams), ("dft_mode", I), ("d_mask", VP), ("centered", I),
        ("n_fe", U), ("spokes_per_frame", U), ("d_traj", VP), ("d_dens", VP),
        ("kernel_width", F), ("sector_width", F), ("osf", F),
        ("d_data", VP), ("d_x", VP), ("d_b1", VP), ("tag", C.c_ulonglong), ("stop_gap_rel", F),
    ]


class Completion(C.Structure):
    """avx_completion"""
    _fields_ = [
        ("tag", C.c_ulonglong), ("status", I), ("dft_mode", I), ("stats", RunStats),
        ("queue_ms", D), ("run_ms", D), ("workspace_bytes", C.c_size_t),
    ]


EXPORT_CB = C.CFUNCTYPE(None, C.c_char_p, C.c_char_p, VP, C.c_size_t, VP)

# name -> (restype, argtypes)
SIGNATURES = {
    "avx_version": (C.c_char_p, []),
    "avx_last_error": (C.c_char_p, []),
    "avx_cartesian_operator_create": (I, [U, U, U, U, VP, I, C.POINTER(VP)]),
    "avx_radial_operator_create": (I, [U, U, U, U, U, U, U, VP, VP, F, F, F, C.POINTER(VP)]),
    "avx_radial_sector_map": (I, [VP, VP, VP, VP]),
    "avx_operator_backward": (I, [VP, VP, VP, VP]),
    "avx_operator_forward": (I, [VP, VP, VP, VP]),
    "avx_operator_adapt_lambda": (I, [VP, F, F, C.POINTER(F)]),
    "avx_operator_opnorm": (I, [VP, VP, VP, U, C.POINTER(D), C.POINTER(D)]),
    "avx_operator_destroy": (None, [VP]),
    "avx_default_params": (I, [I, C.POINTER(PDParams)]),
    "avx_solver_create": (I, [I, U, U, U, U, C.POINTER(PDParams), VP, C.POINTER(VP)]),
    "avx_solver_get_params": (I, [VP, C.POINTER(PDParams)]),
    "avx_solver_set_params": (I, [VP, C.POINTER(PDParams)]),
    "avx_solver_set_verbose": (I, [VP, I]),
    "avx_solver_set_debug": (I, [VP, I, I]),
    "avx_solver_set_relative_stop": (I, [VP, D]),
    "avx_solver_set_stream": (I, [VP, VP]),
    "avx_solver_set_tuning": (I, [VP, I, I, I]),
    "avx_solver_get_tuning": (I, [VP, C.POINTER(I), C.POINTER(I), C.POINTER(C.c_char_p), C.POINTER(I)]),
    "avx_solver_set_kspace_schedule": (I, [VP, I, I]),
    "avx_solver_get_kspace_schedule": (I, [VP, C.POINTER(I), C.POINTER(I)]),
    "avx_solver_run": (I, [VP, VP, VP, VP]),
    "avx_solver_adapt_step_size": (I, [VP, C.POINTER(VP), VP]),
    "avx_solver_compute_gap": (I, [VP, C.POINTER(VP), C.POINTER(VP), VP, VP, VP, C.POINTER(D), C.POINTER(D)]),
    "avx_solver_opnorm": (I, [VP, VP, VP, U, I, C.POINTER(D), C.POINTER(D)]),
    "avx_solver_export": (I, [VP, C.c_char_p, EXPORT_CB, VP]),
    "avx_solver_get_stats": (I, [VP, C.POINTER(RunStats)]),
    "avx_solver_destroy": (None, [VP]),
    "avx_solver_set_timing": (I, [VP, I]),
    "avx_solver_kernel_times": (I, [VP, C.POINTER(F), C.POINTER(U)]),
    "avx_gradient": (I, [VP, C.POINTER(VP), U, U, U, F, F, F]),
    "avx_divergence": (I, [C.POINTER(VP), VP, U, U, U, F, F, F]),
    "avx_sym_gradient": (I, [C.POINTER(VP), C.POINTER(VP), U, U, U, F, F, F]),
    "avx_sym_divergence": (I, [C.POINTER(VP), C.POINTER(VP), U, U, U, F, F, F]),
    "avx_prox3": (I, [C.POINTER(VP), U, F]),
    "avx_prox6": (I, [C.POINTER(VP), U, F]),
    "avx_norm3": (I, [C.POINTER(VP), VP, U]),
    "avx_norm6": (I, [C.POINTER(VP), VP, U]),
    "avx_tv_norm": (I, [VP, U, U, U, F, F, F, C.POINTER(D)]),
    "avx_tgv2_norm": (I, [VP, C.POINTER(VP), F, F, U, U, U, F, F, F, C.POINTER(D)]),
    "avx_ictgv2_norm": (I, [VP, C.POINTER(VP), VP, C.POINTER(VP), F, F, F, U, U, U, C.POINTER(F), C.POINTER(F),
                            C.POINTER(D)]),
    "avx_tv_norm_noalloc": (I, [VP, U, U, U, F, F, F, C.POINTER(D)]),
    "avx_ellipke": (F, [F]),
    "avx_time_space_weights": (I, [F, C.POINTER(F), C.POINTER(F)]),
    "avx_coil_default_params": (I, [C.POINTER(CoilParams)]),
    "avx_coil_time_averaged": (I, [U, U, U, U, VP, VP, VP, VP, I]),
    "avx_coil_b1_from_u_h1": (I, [U, U, U, C.POINTER(CoilParams), VP, VP, VP]),
    "avx_coil_utgv2": (I, [U, U, C.POINTER(CoilParams), VP, VP, VP, U, VP]),
    "avx_coil_b1_recon": (I, [U, U, U, U, F, C.POINTER(CoilParams), VP, VP, VP]),
    "avx_coil_construction": (I, [U, U, U, U, C.POINTER(CoilParams), VP, VP, VP, VP]),
    "avx_coil_time_averaged_radial": (I, [U, U, U, U, U, VP, VP, VP, VP, VP, I]),
    "avx_coil_construction_radial": (I, [U, U, U, U, U, C.POINTER(CoilParams), VP, VP, VP, VP, VP]),
    "avx_normalize_data": (I, [U, U, U, U, U, VP, VP, VP, C.POINTER(F)]),
    "avx_reconstruct_host": (I, [I, U, U, U, U, C.POINTER(PDParams), I, VP, VP, VP, VP, VP, C.POINTER(RunStats)]),
    "avx_reconstruct_host_release": (None, []),
    "avx_operator_set_dft_mode": (I, [VP, I]),
    "avx_query_workspace": (I, [C.POINTER(Request), C.POINTER(C.c_size_t)]),
    "avx_batch_create": (I, [I, C.c_size_t, I, C.POINTER(VP)]),
    "avx_batch_submit": (I, [VP, C.POINTER(Request)]),
    "avx_serve_poll": (I, [VP, C.POINTER(Completion), I, C.POINTER(I), I]),
    "avx_batch_drain": (I, [VP]),
    "avx_batch_pending": (I, [VP]),
    "avx_batch_destroy": (None, [VP]),
    "avx_operator_get_dft_mode": (I, [VP, C.POINTER(I)]),
}


def declare(lib):
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
