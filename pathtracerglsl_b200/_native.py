"""Loader of the CUDA library (``libptx_rt.so``) with the C signatures of include/ptx_rt.h.

There is no fallback: if the library is missing or cannot be loaded, importing the
engine raises.  The transport loop runs only on the GPU.
"""
import ctypes as C
import os

from . import abi

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libptx_rt.so")

# name -> (restype, argtypes); the exact set of entry points include/ptx_rt.h declares
SIGNATURES = {
    "ptr_abi_version": (C.c_int, []),
    "ptr_create": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "ptr_destroy": (C.c_int, [C.c_void_p]),
    "ptr_last_error": (C.c_char_p, [C.c_void_p]),
    "ptr_upload_scene": (C.c_int, [C.c_void_p, C.POINTER(abi.SceneDesc), C.POINTER(C.c_void_p)]),
    "ptr_free_scene": (C.c_int, [C.c_void_p]),
    "ptr_upload_scene_rails": (C.c_int, [C.c_void_p, C.POINTER(abi.SceneDesc), C.POINTER(abi.Rails), C.POINTER(C.c_void_p)]),
    "ptr_compile": (C.c_int, [C.c_void_p, C.POINTER(abi.ProgramDesc), C.POINTER(C.c_void_p)]),
    "ptr_free_program": (C.c_int, [C.c_void_p]),
    "ptr_render": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(abi.Frame)]),
    "ptr_render_samples": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(abi.Frame), C.POINTER(C.c_float), C.c_size_t]),
    "ptr_get_stream": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "ptr_trace_closest": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int,
                                    C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "ptr_build_bvh": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p,
                                C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "ptr_build_cwbvh": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_void_p, C.c_int, C.c_void_p,
                                  C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "ptr_build_light_tree": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]),
    "ptr_render_noalloc": (C.c_int, [C.POINTER(abi.SceneDesc), C.POINTER(abi.ProgramDesc), C.POINTER(abi.Frame),
                                     C.c_void_p, C.c_void_p, C.c_void_p]),
    "ptr_render_batch": (C.c_int, [C.c_void_p, C.POINTER(abi.BatchJob), C.c_int]),
    "ptr_get_batch_counters": (C.c_int, [C.c_void_p, C.POINTER(abi.Counters)]),
    "ptr_profile_batch_next": (C.c_int, [C.c_void_p, C.c_int]),
    "ptr_get_batch_profile": (C.c_int, [C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_int), C.c_int]),
    "ptr_backward": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(abi.Frame), C.POINTER(C.c_float),
                               C.POINTER(C.c_double), C.c_size_t]),
    "ptr_update_params": (C.c_int, [C.c_void_p, C.POINTER(abi.Material), C.c_int, C.POINTER(abi.Region), C.c_int]),
    "ptr_set_tuning": (C.c_int, [C.c_void_p, C.POINTER(abi.Tuning)]),
    "ptr_specialize": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_double)]),
    "ptr_specialize_batch": (C.c_int, [C.c_void_p, C.POINTER(abi.BatchJob), C.c_int, C.POINTER(C.c_double)]),
    "ptr_set_accel_build": (C.c_int, [C.c_void_p, C.c_int]),
    "ptr_get_tuning": (C.c_int, [C.c_void_p, C.POINTER(abi.Tuning)]),
    "ptr_sync": (C.c_int, [C.c_void_p, C.c_int]),
    "ptr_read_export": (C.c_int, [C.c_void_p, C.c_char_p, C.POINTER(C.c_float), C.c_size_t]),
    "ptr_read_export_device": (C.c_int, [C.c_void_p, C.c_char_p, C.c_void_p, C.c_size_t]),
    "ptr_get_counters": (C.c_int, [C.c_void_p, C.POINTER(abi.Counters)]),
    "ptr_profile_next": (C.c_int, [C.c_void_p, C.c_int]),
    "ptr_get_profile": (C.c_int, [C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_int), C.c_int]),
}

_lib = None


def load(path=None):
    """Load the library and bind every entry point; raises if anything is missing.
    PTX_RT_LIB names another build of the same library (e.g. one compiled with different
    launch bounds, for an A/B measurement)."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or os.environ.get("PTX_RT_LIB") or LIB_PATH
    if not os.path.exists(path):
        raise RuntimeError(f"CUDA library not built: {path} (run pathtracerglsl_b200.build.build())")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)   # AttributeError if the export is missing
        fn.restype = res
        fn.argtypes = args
    if lib.ptr_abi_version() != abi.ABI_VERSION:
        raise RuntimeError("libptx_rt.so ABI version does not match pathtracerglsl_b200.abi")
    _lib = lib
    return lib
