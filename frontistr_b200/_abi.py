"""ctypes signatures of include/hecmw33_gpu.h (every argument by pointer)."""
import ctypes

_i = ctypes.POINTER(ctypes.c_int)
_d = ctypes.POINTER(ctypes.c_double)
_v = ctypes.c_void_p
# hecmw33_exchange_fn / hecmw33_allreduce_fn
EXCHANGE_FN = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                               ctypes.POINTER(ctypes.c_double))
ALLREDUCE_FN = ctypes.CFUNCTYPE(ctypes.c_double, ctypes.c_void_p, ctypes.c_double)

SIGNATURES = {
    "hecmw33_gpu_create": [_i, _i],
    "hecmw33_gpu_destroy": [_i, _i],
    "hecmw33_gpu_set_matrix": [_i, _i, _i, _i, _i, _i, _i, _i, _i, _d, _d, _d, _i, _i],
    "hecmw33_gpu_set_mpc": [_i, _i, _i, _i, _i, _d, _d, _i],
    "hecmw33_gpu_set_domain": [_i, _i, _i, _i, _i, _i, _i, EXCHANGE_FN, ALLREDUCE_FN, _v, _i],
    "hecmw33_gpu_solve_resident": [_i, _d, _d, _i, _d, _i, _d, _d, _i],
    "hecmw33_gpu_solve_resident_device": [_i, _v, _v, _i, _d, _i, _d, _d, _i],
    "hecmw33_gpu_solve": [_i, _i, _i, _i, _i, _i, _i, _i, _i, _d, _d, _d, _d, _d, _i, _d, _i, _d,
                          _d, _i],
    "hecmw33_gpu_solve_multi": [_i, _i, _d, _d, _i, _d, _i, _d, _i, _d, _d, _i],
    "hecmw33_gpu_solve_multi_device": [_i, _i, _v, _v, _i, _d, _i, _d, _i, _d, _d, _i],
    "hecmw33_gpu_matvec": [_i, _d, _d, _i],
    "hecmw33_gpu_precond_apply": [_i, _d, _d, _i, _d, _i],
    "hecmw33_gpu_get_colouring": [_i, _i, _i, _i, _i],
    "hecmw33_gpu_colour_schedule": [_i, _i, _i, _i, _i, _i, _i, _i, _i, _i],
    "hecmw33_gpu_smoother_schedule": [_i, _i, _i, _i, _i, _i, _i, _i, _i],
    "hecmw33_gpu_coarse_aggregates": [_i, _i, _i, _i, _i, _i, _i, _i, _i],
    "hecmw33_gpu_last_solve_info": [_i, _i, _d, _i],
    "hecmw33_gpu_condition_estimate": [_i, _i, _d, _d, _i],
    "hecmw33_gpu_time_spmv": [_i, _i, _d, _i],
    "hecmw33_gpu_time_precond": [_i, _i, _i, _d, _d, _i],
    "hecmw33_gpu_learn_record": [_i, _i, _i, _i, _i],
    "hecmw33_gpu_learn_train": [_i, _i, _d, _d, _i],
    "hecmw33_gpu_learn_weights": [_i, _i, ctypes.POINTER(ctypes.c_float), _i, _i],
    "hecmw33_gpu_learn_eval": [_i, ctypes.POINTER(ctypes.c_float), _d, _d, _d, _d, ctypes.POINTER(ctypes.c_float),
                               _i],
    "hecmw33_gpu_rel_resid_noalloc": [_i, _v, _v, _v, _v, _v, _v, _v, _v, _v, _d, _i],
    "hecmw33_gpu_batch_create": [_i, _i],
    "hecmw33_gpu_batch_destroy": [_i, _i],
    "hecmw33_gpu_batch_set_matrix": [_i, _i, _i, _i, _i, _i, _i, _i, _i, _i, _i, _d, _d, _d, _i, _d, _i],
    "hecmw33_gpu_batch_solve": [_i, _d, _d, _i, _d, _i, _d, _i, _d, _d, _i],
    "hecmw33_gpu_batch_solve_device": [_i, _v, _v, _i, _d, _i, _d, _i, _d, _d, _i],
    "hecmw33_gpu_batch_autotune": [_i, _d, _d, _i, _d, _i],
    "hecmw33_gpu_batch_info": [_i, _i, _d, _i],
    "hecmw33_gpu_assemble_hex8": [_i, _i, _d, _i, _i, _d, _d, _d, _i, _i, _i, _d, _i, _i, _i, _i],
    "hecmw33_gpu_assemble_hex8_neohooke": [_i, _i, _d, _i, _i, _d, _d, _d, _d, _i, _i, _i, _d, _i, _i, _i, _i,
                                           _i],
    "hecmw33_gpu_get_matrix": [_i, _i, _i, _i, _i, _d, _d, _d, _d, _i],
    "hecmw33_gpu_solve_assembled": [_i, _d, _i, _d, _i, _d, _d, _i],
    "hecmw33_gpu_last_error": [ctypes.c_char_p, ctypes.c_int],
}

RESTYPES = {"hecmw33_gpu_last_error": ctypes.c_int}


def declare(lib):
    for name, args in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = RESTYPES.get(name, None)


def exported_names():
    return sorted(SIGNATURES)
