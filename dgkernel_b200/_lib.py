"""ctypes binding of libdgk.so (the C ABI declared in include/dgk.h)."""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdgk.so")

# status codes (include/dgk.h)
OK, ERR_INVALID, ERR_STATE, ERR_NOT_FOUND, ERR_CUDA, ERR_TIMEOUT, ERR_UNSUPPORTED, ERR_NO_DEVICE = range(8)

# Every symbol include/dgk.h declares, with its ctypes signature.
_P = C.c_void_p
_S = C.c_char_p
_I32, _I64, _U64, _D = C.c_int32, C.c_int64, C.c_uint64, C.c_double
_PI64, _PD, _PI32 = C.POINTER(C.c_int64), C.POINTER(C.c_double), C.POINTER(C.c_int32)
SIGNATURES = {
    "dgk_runner_create": [_PI64, _I32, _I32, C.POINTER(_P)],
    "dgk_runner_create_host_only": [_PI64, _I32, _I32, C.POINTER(_P)],
    "dgk_runner_free": [_P],
    "dgk_last_error": [_P],
    "dgk_global_error": [],
    "dgk_set_stream": [_P, _P],
    "dgk_sync": [_P],
    "dgk_bind_array": [_P, _S, _I32, _I32, _I32, _I64, _I32, _PI64, _I32, _I32, _I64, _I64],
    "dgk_bind_matrix": [_P, _S, _I64, _I64, _PD, _I32, _I32],
    "dgk_bind_scalar": [_P, _S, _I32, _PD],
    "dgk_allocate": [_P],
    "dgk_copy_to_device": [_P, _S, _P, _I64],
    "dgk_copy_from_device": [_P, _S, _P, _I64],
    "dgk_copy_partition_to_device": [_P, _S, _I32, _P, _I64],
    "dgk_copy_partition_from_device": [_P, _S, _I32, _P, _I64],
    "dgk_copy_raw_from_device": [_P, _S, _I64, _P, _I64],
    "dgk_get_offsets": [_P, _S, _PI64],
    "dgk_device_ptr": [_P, _S, C.POINTER(_P)],
    "dgk_configure_kernel": [_P, _S, _I32, C.POINTER(_S), C.POINTER(C.c_uint32)],
    "dgk_build_kernel": [_P, _S, _S],
    "dgk_execute_kernel": [_P, _S, _I32, _PD, C.POINTER(_P)],
    "dgk_kernel_signature": [_P, _S, C.c_char_p, _I64],
    "dgk_generate_preamble": [_P, C.c_char_p, _I64],
    "dgk_element_create": [_I32, C.POINTER(_P)],
    "dgk_element_free": [_P],
    "dgk_element_dims": [_P, _PI32, _PI32],
    "dgk_element_get": [_P, _S, _PD, _I64],
    "dgk_element_fmask": [_P, _PI32],
    "dgk_kuhn_mesh": [_I32, _I32, _D, _D, _PD, _PD, _PD, _PI64, _PI64, _PI64],
    "dgk_ti_connect3d": [_I64, _PI64, _PI64, _PI64],
    "dgk_face_connector": [_I64, _I32, _I32, _I32, _PI64, _PI64, _I32, _PI64, _PI64, _PI64],
    "dgk_read_gambit": [C.c_char_p, _PI64, _PD, _PD, _PD, _PI64, _PI64, _PI64],
    "dgk_halo_plan": [_I64, _I32, _I32, _I32, _PI64, _PI64, _I32, _PI32, _I32, _I32, _PI64, _PI64, _PI32, _PI64,
                      _PI64, _PI64, _PI64],
    "dgk_gather_values": [_P, _I32, _I64, _P, _I64, _P, _P],
    "dgk_tile_halo": [_I32, _PI64, _PI64, _I32, _I32, _PI32, _I32, _I32, _I32, _I32, _I32, _PI64, _PI32, _PI64,
                      _PI32, _PI32, _PI32, C.POINTER(C.c_uint32)],
    "dgk_face_gather_map": [_I64, _I32, _I32, _I32, _PI64, _PI64, _I32, _PI64, _PI32],
    "dgk_init_field_parts": [_P, _S, _S, _S, _S, _D, _I32, _PD],
    "dgk_mlp_param_count": [_I32, _PI64],
    "dgk_mlp_forward": [_P, _P, _I64, _I32, _I32, _P, _P, _P],
    "dgk_mlp_loss_grad": [_P, _P, _P, _I64, _I32, _P, _P, _P],
    "dgk_mlp_adam": [_P, _P, _P, _P, _I64, C.c_float, C.c_float, C.c_float, C.c_float, _I32, _P],
    "dgk_capture_graph": [_P, _S, _I32, _I32, _PD, C.POINTER(_P)],
    "dgk_graph_launch": [_P, _I32],
    "dgk_graph_free": [_P],
    "dgk_compact_faces": [_I32, _PI64, _PI64, _PI64, _I32, _I32, _PI32, _PI32, C.POINTER(C.c_uint8), _I32, _PI32],
    "dgk_setup_geometry": [_P, _P, _I64, _PD, _PD, _PD, _PI64, _PI64, _PI64, _D, C.POINTER(_S), _PD],
    "dgk_init_field": [_P, _S, _S, _S, _S, _I32, _D, _D, _I32, _PD],
    "dgk_splitmix_uniform": [_U64, _I64, _PD],
    "dgk_convert_upload_noalloc": [_P, _I32, _P, _I32, _I64, _P],
}
_STRING_RESULT = {"dgk_last_error", "dgk_global_error"}

_lib = None


class DGKError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[dgk status {code}] {msg}")
        self.code = code


def lib():
    """Load libdgk.so; raises if it has not been built (there is no CPU fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python dgkernel_b200/build.py`")
        L = C.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = C.c_char_p if name in _STRING_RESULT else C.c_int
        _lib = L
    return _lib


def check(rc: int, runner_handle=None):
    if rc != OK:
        L = lib()
        msg = (L.dgk_last_error(runner_handle) if runner_handle else L.dgk_global_error()) or b""
        raise DGKError(rc, msg.decode(errors="replace"))
