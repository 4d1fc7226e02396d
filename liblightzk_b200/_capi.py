"""ctypes binding of liblzk_b200.so (the C ABI declared in include/lzk.h).

The shared library is built in-tree by ``python -m liblightzk_b200.build``.
There is no fallback: if the library is missing every entry point raises.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liblzk_b200.so")

c_p = ctypes.c_void_p
c_sz = ctypes.c_size_t
c_u32 = ctypes.c_uint32
c_i = ctypes.c_int

# name -> (restype, argtypes); every function of include/lzk.h
SIGNATURES = {
    "lzk_status_string": (ctypes.c_char_p, [c_i]),
    "lzk_version": (ctypes.c_char_p, []),
    "lzk_msm_g1": (c_i, [c_p, c_p, c_sz, c_p, c_p, c_p]),
    "lzk_msm_g2": (c_i, [c_p, c_p, c_sz, c_p, c_p, c_p]),
    "lzk_msm_workspace_bytes": (c_sz, [c_i, c_sz, c_p]),
    "lzk_msm_autotune_window": (c_u32, [c_i, c_sz, c_u32]),
    "lzk_g1_precompute": (c_i, [c_p, c_sz, c_u32, c_u32, c_p, c_sz, c_p]),
    "lzk_g2_precompute": (c_i, [c_p, c_sz, c_u32, c_u32, c_p, c_sz, c_p]),
    "lzk_msm_precomp_windows": (c_u32, [c_u32]),
    "lzk_g1_to_affine": (c_i, [c_p, c_p, c_sz, c_p]),
    "lzk_g2_to_affine": (c_i, [c_p, c_p, c_sz, c_p]),
    "lzk_ntt": (c_i, [c_p, c_u32, c_i, c_p]),
    "lzk_ntt_batch": (c_i, [c_p, c_u32, c_u32, c_sz, c_i, c_p]),
    "lzk_ntt_prepare": (c_i, [c_u32]),
    "lzk_number_theory_transformation": (c_i, [c_sz, c_sz, c_p, c_p, c_p, c_p]),
    "lzk_spmv3": (c_i, [c_p, c_p, c_p, c_p, c_p, c_p, c_p, c_p]),
    "lzk_spmv": (c_i, [c_p, c_p, c_p, c_p]),
}


class MsmCfg(ctypes.Structure):
    """struct lzk_msm_cfg"""

    _fields_ = [
        ("window_bits", ctypes.c_uint32),
        ("flags", ctypes.c_uint32),
        ("precomp_windows", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32),
        ("level_stride", ctypes.c_size_t),
        ("workspace", ctypes.c_void_p),
        ("workspace_bytes", ctypes.c_size_t),
    ]


LZK_MSM_PRECOMPUTED = 0x1
NTT_FORWARD, NTT_INVERSE, NTT_COSET_FORWARD, NTT_COSET_INVERSE = 0, 1, 2, 3


class Csr(ctypes.Structure):
    """struct lzk_csr"""

    _fields_ = [
        ("val", ctypes.c_void_p),
        ("col_idx", ctypes.c_void_p),
        ("row_ptr", ctypes.c_void_p),
        ("rows", ctypes.c_uint64),
        ("cols", ctypes.c_uint64),
        ("nnz", ctypes.c_uint64),
        ("index_bytes", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32),
    ]


class LzkError(RuntimeError):
    def __init__(self, status, where=""):
        self.status = status
        msg = lib().lzk_status_string(status).decode()
        super().__init__(f"{where}: liblzk_b200 status {status} ({msg})")


_lib = None


def lib():
    """The loaded library, with argument/return types declared."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is not built: run `python -m liblightzk_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(status, where=""):
    if status != 0:
        raise LzkError(status, where)
    return status


def call(name, *args):
    """Call an int-status entry point and raise LzkError on failure."""
    return check(getattr(lib(), name)(*args), name)
