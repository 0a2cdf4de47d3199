"""ctypes binding of the C ABI in include/cubvh_b200.h (libcubvh_b200.so).

The shared library is built in-tree (``make -C cubvh_b200/csrc`` or
``__graft_entry__.build()``).  There is no fallback: if the library is
missing or fails to load, importing the query API raises.
"""

from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcubvh_b200.so")

_lib = None

c_i64 = ctypes.c_int64
c_i32 = ctypes.c_int32
c_u32 = ctypes.c_uint32
c_vp = ctypes.c_void_p
c_sz = ctypes.c_size_t
c_int = ctypes.c_int

# name -> argtypes (every entry point returns int status unless noted)
_SIGS = {
    "cubvh_bvh_create": [c_vp, c_i64, c_vp, c_i64, ctypes.POINTER(c_vp)],
    "cubvh_bvh_create_from_records": [c_vp, c_i64, ctypes.POINTER(c_vp)],
    "cubvh_bvh_create_from_state_dict": [c_vp, c_i64, c_vp, c_i64, ctypes.POINTER(c_vp)],
    "cubvh_bvh_create_device": [c_vp, c_i64, c_vp, c_i64, c_i32, c_vp, ctypes.POINTER(c_vp)],
    "cubvh_bvh_destroy": [c_vp],
    "cubvh_bvh_info": [c_vp, ctypes.POINTER(c_i64), ctypes.POINTER(c_i64), ctypes.POINTER(c_i32)],
    "cubvh_bvh_state_dict_sizes": [c_vp, ctypes.POINTER(c_i64), ctypes.POINTER(c_i64)],
    "cubvh_bvh_state_dict": [c_vp, c_vp, c_vp],
    "cubvh_bvh_layout": [c_vp, c_vp, c_vp],
    "cubvh_bvh_upload": [c_vp],
    "cubvh_unsigned_distance": [c_vp, c_vp, c_i64, c_vp, c_vp, c_vp, c_vp],
    "cubvh_signed_distance": [c_vp, c_vp, c_i64, c_u32, c_vp, c_vp, c_vp, c_vp],
    "cubvh_ray_trace": [c_vp, c_vp, c_vp, c_i64, c_vp, c_vp, c_vp, c_vp],
    "cubvh_ray_trace_host": [c_vp, c_vp, c_vp, c_i64, c_vp, c_vp, c_vp, c_vp],
    "cubvh_signed_distance_host": [c_vp, c_vp, c_i64, c_u32, c_vp, c_vp, c_vp, c_vp],
    "cubvh_stab_directions": [c_i64, c_i64, c_vp, c_vp],
    "cubvh_floodfill_workspace_size": [c_int, c_int, c_int, c_int, ctypes.POINTER(c_sz)],
    "cubvh_floodfill": [c_vp, c_int, c_int, c_int, c_int, c_vp, c_vp, c_sz, c_vp],
    "cubvh_floodfill_check": [c_vp, c_int, c_int, c_int, c_int, c_vp],
    "cubvh_udf_to_sdf": [c_vp, c_int, c_int, c_int, c_int, ctypes.c_float, c_vp, c_vp, c_sz, c_vp],
    "cubvh_bvh_refit": [c_vp, c_vp, c_i64, c_vp],
    "cubvh_sparse_marching_cubes": [c_vp, c_vp, c_i64, ctypes.c_float, c_int, c_vp, ctypes.POINTER(c_vp),
                                    ctypes.POINTER(c_i64), ctypes.POINTER(c_i64)],
    "cubvh_sparse_mc_fetch": [c_vp, c_vp, c_vp, c_vp],
    "cubvh_sparse_mc_free": [c_vp],
    "cubvh_arena_create": [ctypes.c_int32, c_vp, c_vp, c_vp, c_vp, c_vp, ctypes.POINTER(c_vp)],
    "cubvh_arena_create_device": [ctypes.c_int32, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, ctypes.POINTER(c_vp)],
    "cubvh_arena_destroy": [c_vp],
    "cubvh_arena_info": [c_vp, ctypes.POINTER(c_i32), ctypes.POINTER(c_i64), ctypes.POINTER(c_i64)],
    "cubvh_arena_set_queries": [c_vp, c_vp, c_vp],
    "cubvh_arena_distance": [c_vp, c_vp, c_vp, c_vp, c_vp, c_vp],
    "cubvh_arena_backward": [c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp],
    "cubvh_distance_backward": [c_vp, c_vp, c_i64, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp],
}
_STR_FUNCS = ("cubvh_version", "cubvh_last_error")
_U64_FUNCS = ("cubvh_kernel_launches",)


def lib():
    """Load libcubvh_b200.so once and declare its signatures."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"cubvh_b200: native library not found at {LIB_PATH}; build it with "
                "`make -C cubvh_b200/csrc` (nvcc, sm_100a)")
        L = ctypes.CDLL(LIB_PATH)
        for name, args in _SIGS.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = c_int
        for name in _STR_FUNCS:
            fn = getattr(L, name)
            fn.argtypes = []
            fn.restype = ctypes.c_char_p
        for name in _U64_FUNCS:
            fn = getattr(L, name)
            fn.argtypes = []
            fn.restype = ctypes.c_uint64
        _lib = L
    return _lib


def exported_symbols():
    return list(_SIGS) + list(_STR_FUNCS) + list(_U64_FUNCS)


def check(rc: int, what: str):
    if rc != 0:
        msg = lib().cubvh_last_error().decode(errors="replace")
        raise RuntimeError(f"cubvh_b200.{what}: {msg} (status {rc})")


def version() -> str:
    return lib().cubvh_version().decode()


def kernel_launches() -> int:
    """Kernels launched by the library in this process so far."""
    return int(lib().cubvh_kernel_launches())
