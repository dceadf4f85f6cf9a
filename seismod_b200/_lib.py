"""ctypes binding of libseismod_gpu.so (C ABI declared in include/seismod_gpu.h).

The library is built in-tree (``make -C seismod_b200`` or
``__graft_entry__.build()``).  There is no fallback: if the library is
missing or fails to load, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libseismod_gpu.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "seismod_gpu.h")

SM_OK, SM_EINVAL, SM_ENOMEM, SM_ECUDA, SM_ECFL, SM_EIO, SM_ETIMEOUT, SM_EBUSY, SM_ESTATE, \
    SM_ENOTFOUND = range(10)
SM_FP32, SM_FP64, SM_FP16, SM_BF16, SM_BFP16 = 0, 1, 2, 3, 4
PRECISIONS = {"fp32": SM_FP32, "fp64": SM_FP64, "fp16": SM_FP16, "bf16": SM_BF16,
              "bfp16": SM_BFP16}
SM_SRC = {"sx": 0, "sz": 2, "sxz": 4, "bulk": 6}
SM_COMP = {"vx": 0, "vy": 1, "vz": 2, "txx": 5, "tzz": 6, "txz": 7, "p": 8}
SM_PART = {"total": 0, "x": 1, "z": 2}
# e_cyl_iso components (enum component, structs.h:45)
SM_VZ, SM_TZZ, SM_DIV, SM_CURL = 2, 6, 11, 12
SM_VR, SM_VT, SM_TRR, SM_TRT, SM_TRZ, SM_TTT, SM_TTZ = 13, 14, 15, 16, 17, 18, 19
SM_ALL_SHOTS = C.c_size_t(-1).value


class SeismodError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


_dp = C.POINTER(C.c_double)
_szp = C.POINTER(C.c_size_t)
_ip = C.POINTER(C.c_int)
_sz = C.c_size_t
_vp = C.c_void_p

_SIGS = {
    "sm_last_error": (C.c_char_p, []),
    "sm_abi_version": (C.c_int, []),
    "sm_device_info": (C.c_int, [C.c_int, _ip, _szp, _szp]),
    "sm_ricker_length": (_sz, [C.c_double, C.c_double, C.c_double]),
    "sm_ricker": (C.c_int, [_sz, _dp, _dp, C.c_double, C.c_double, _sz, _dp, _szp]),
    "sm_nsteps": (_sz, [C.c_double, C.c_double]),
    "sm_sample_predicate": (C.c_int, [_sz, C.c_double, C.c_double, C.c_double]),
    "sm_eiso_materials": (C.c_int, [_sz, _sz] + [_dp] * 8 + [_dp]),
    "sm_eiso_profiles": (C.c_int, [_sz, C.c_double, _sz, _dp, _dp, _dp, _dp]),
    "sm_a3d_pad_model": (C.c_int, [_sz, _sz, _sz, _sz, _dp, _dp, _dp, _dp]),
    "sm_a3d_cfl_vpmax": (C.c_double, [_sz, _sz, _dp]),
    "sm_a3d_cfl_vpmax_unpadded": (C.c_double, [_sz, _sz, _sz, _sz, _dp]),
    "sm_a3d_cpml": (C.c_int, [_sz, _sz, _sz, _sz] + [C.c_double] * 8 +
                    [C.c_int, C.c_double, C.POINTER(_dp)]),
    "sm_ecyl_pad_model": (C.c_int, [_sz, _sz, _sz] + [_dp] * 6),
    "sm_ecyl_materials": (C.c_int, [_sz, _sz, _dp, _dp, _dp, C.POINTER(_dp), _dp]),
    "sm_ecyl_cpml": (C.c_int, [_sz] + [C.c_double] * 8 + [C.c_int, C.POINTER(_dp)]),
    "sm_ecyl_kurkjian": (_sz, [C.c_double] * 7 + [C.c_int, _sz, _dp]),
    "sm_ecyl_create": (C.c_int, [C.c_int, _sz, _sz, _sz, C.c_int, C.c_double, C.c_double,
                                 C.c_double, C.POINTER(_dp), C.POINTER(_dp), C.c_int,
                                 C.POINTER(_vp)]),
    "sm_ecyl_set_sources": (C.c_int, [_vp, _sz, _szp, _ip, _dp, _szp, _sz]),
    "sm_ecyl_set_receivers": (C.c_int, [_vp, _sz, _szp, _ip, _dp, _dp, _sz]),
    "sm_ecyl_run": (C.c_int, [_vp, _sz]),
    "sm_ecyl_sync": (C.c_int, [_vp]),
    "sm_ecyl_reset": (C.c_int, [_vp]),
    "sm_ecyl_read_traces": (C.c_int, [_vp, _sz, _sz, _dp, _sz, _szp]),
    "sm_ecyl_get_field": (C.c_int, [_vp, C.c_int, _dp]),
    "sm_ecyl_set_field": (C.c_int, [_vp, C.c_int, _dp]),
    "sm_ecyl_stream": (C.c_int, [_vp, C.POINTER(_vp)]),
    "sm_ecyl_set_timing": (C.c_int, [_vp, C.c_int]),
    "sm_ecyl_kernel_stats": (C.c_int, [_vp, C.c_int, _dp, _szp, _szp]),
    "sm_ecyl_destroy": (C.c_int, [_vp]),
    "sm_ecyl_device_bytes": (_sz, [_sz, _sz, _sz, C.c_int]),
    "sm_eiso_create": (C.c_int, [C.c_int, _sz, _sz, _sz, C.c_double, C.c_double] + [_dp] * 8 +
                       [C.c_int, _sz, C.POINTER(_vp)]),
    "sm_eiso_set_sources": (C.c_int, [_vp, _sz, _sz, _szp, _ip, _dp, _szp, _sz, C.c_double]),
    "sm_eiso_set_receivers": (C.c_int, [_vp, _sz, _sz, _szp, _ip, _dp, _dp, _sz]),
    "sm_eiso_run": (C.c_int, [_vp, _sz]),
    "sm_eiso_group_run": (C.c_int, [C.POINTER(_vp), C.c_int, _sz]),
    "sm_a3d_group_run": (C.c_int, [C.POINTER(_vp), C.c_int, _sz]),
    "sm_eiso_sync": (C.c_int, [_vp]),
    "sm_eiso_step_count": (C.c_int, [_vp, _szp]),
    "sm_eiso_read_traces": (C.c_int, [_vp, _sz, _sz, _sz, _dp, _sz, _szp]),
    "sm_eiso_get_field": (C.c_int, [_vp, _sz, C.c_int, C.c_int, _dp]),
    "sm_eiso_set_field": (C.c_int, [_vp, _sz, C.c_int, C.c_int, _dp]),
    "sm_eiso_reset": (C.c_int, [_vp]),
    "sm_eiso_destroy": (C.c_int, [_vp]),
    "sm_a3d_create": (C.c_int, [C.c_int, _sz, _sz, _sz, _sz] + [C.c_double] * 4 +
                      [_dp, _dp, C.POINTER(_dp), C.c_int, C.POINTER(_vp)]),
    "sm_a3d_create_unpadded": (C.c_int, [C.c_int, _sz, _sz, _sz, _sz] + [C.c_double] * 4 +
                               [_dp, _dp, C.POINTER(_dp), C.c_int, C.POINTER(_vp)]),
    "sm_a3d_set_sources": (C.c_int, [_vp, _sz, _szp, _dp, _szp, _sz, C.c_double]),
    "sm_a3d_set_receivers": (C.c_int, [_vp, _sz, _szp, _ip, _dp, _dp, _sz]),
    "sm_a3d_run": (C.c_int, [_vp, _sz]),
    "sm_a3d_sync": (C.c_int, [_vp]),
    "sm_a3d_step_count": (C.c_int, [_vp, _szp]),
    "sm_a3d_read_traces": (C.c_int, [_vp, _sz, _sz, _dp, _sz, _szp]),
    "sm_a3d_get_field": (C.c_int, [_vp, C.c_int, _dp]),
    "sm_a3d_set_field": (C.c_int, [_vp, C.c_int, _dp]),
    "sm_a3d_reset": (C.c_int, [_vp]),
    "sm_a3d_destroy": (C.c_int, [_vp]),
    "sm_eiso_stream": (C.c_int, [_vp, C.POINTER(_vp)]),
    "sm_eiso_set_timing": (C.c_int, [_vp, C.c_int]),
    "sm_eiso_set_config": (C.c_int, [_vp, C.c_int]),
    "sm_eiso_get_config": (C.c_int, [_vp, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "sm_eiso_autotune": (C.c_int, [_vp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double)]),
    "sm_eiso_set_graph": (C.c_int, [_vp, C.c_int]),
    "sm_eiso_kernel_stats": (C.c_int, [_vp, C.c_int, _dp, _szp, _szp]),
    "sm_a3d_stream": (C.c_int, [_vp, C.POINTER(_vp)]),
    "sm_a3d_set_timing": (C.c_int, [_vp, C.c_int]),
    "sm_a3d_set_config": (C.c_int, [_vp, C.c_int]),
    "sm_a3d_set_chunk": (C.c_int, [_vp, C.c_int]),
    "sm_a3d_autotune": (C.c_int, [_vp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                  C.POINTER(C.c_double)]),
    "sm_a3d_set_graph": (C.c_int, [_vp, C.c_int]),
    "sm_a3d_get_config": (C.c_int, [_vp, _ip, _ip]),
    "sm_a3d_kernel_stats": (C.c_int, [_vp, C.c_int, _dp, _szp, _szp]),
    "sm_e_iso_main": (C.c_int, [C.c_int, C.POINTER(C.c_char_p)]),
    "sm_a_iso_3d_main": (C.c_int, [C.c_int, C.POINTER(C.c_char_p)]),
}

_LIB = None


def header_symbols():
    """Every function the public header declares."""
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(sm_[a-z0-9_]+)\s*\(", txt)))


def load():
    """Load the library (raises if it is missing: there is no fallback)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise SeismodError(-1, f"{LIB_PATH} not built; run make -C seismod_b200")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


def check(rc):
    if rc != SM_OK:
        msg = load().sm_last_error()
        raise SeismodError(rc, msg.decode() if msg else "")
    return rc


def dptr(a):
    return a.ctypes.data_as(_dp)


def szptr(a):
    return a.ctypes.data_as(_szp)


def iptr(a):
    return a.ctypes.data_as(_ip)
