"""ctypes loaders for the in-tree native libraries.

The solver has no CPU fallback: if libhecmw33_gpu.so is missing or cannot be
loaded, gpu_lib() raises.  Build the libraries with `python -m frontistr_b200.build`.
"""
import ctypes
import os

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(_PKG, "lib")

_gpu = None
_asm = None

_i32p = ctypes.POINTER(ctypes.c_int)
_f64p = ctypes.POINTER(ctypes.c_double)
_vp = ctypes.c_void_p


class NativeLibraryMissing(RuntimeError):
    pass


def _load(name):
    path = os.path.join(LIB_DIR, name)
    if not os.path.exists(path):
        raise NativeLibraryMissing(
            "%s not built (expected %s); run `python -m frontistr_b200.build`" % (name, path))
    return ctypes.CDLL(path)


def assemble_lib():
    global _asm
    if _asm is None:
        lib = _load("libfistr_assemble.so")
        lib.fistr_box_counts.restype = ctypes.c_int
        lib.fistr_box_assemble.restype = ctypes.c_int
        lib.fistr_box_assemble.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _f64p,
                                           ctypes.c_uint64, _i32p, _i32p, _i32p, _i32p,
                                           _f64p, _f64p, _f64p, _f64p, _f64p]
        lib.fistr_mesh_profile_counts.restype = ctypes.c_int
        lib.fistr_mesh_assemble.restype = ctypes.c_int
        lib.fistr_mat_ass_bc.restype = None
        lib.fistr_mat_ass_bc.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, _i32p, _i32p,
                                         _i32p, _i32p, _f64p, _f64p, _f64p, _f64p]
        lib.fistr_mat_ass_bc_list.restype = None
        lib.fistr_mat_ass_bc_list.argtypes = [ctypes.c_int, _i32p, _i32p, _f64p, _i32p, _i32p, _i32p, _i32p,
                                              _f64p, _f64p, _f64p, _f64p]
        lib.fistr_box_neohooke.restype = ctypes.c_int
        lib.fistr_box_neohooke.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                           ctypes.c_double, ctypes.c_double, _f64p, _i32p, _i32p, _i32p, _i32p,
                                           _f64p, _f64p, _f64p, _f64p]
        _asm = lib
    return _asm


def gpu_lib():
    """The CUDA solver library (include/hecmw33_gpu.h)."""
    global _gpu
    if _gpu is None:
        from . import _abi
        lib = _load("libhecmw33_gpu.so")
        _abi.declare(lib)
        _gpu = lib
    return _gpu
