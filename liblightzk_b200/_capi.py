"""ctypes binding of liblzk_b200.so (the C ABI declared in include/lzk.h).

The shared library is built in-tree by ``python -m liblightzk_b200.build``.
There is no fallback: if the library is missing every entry point raises.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
# LZK_LIBRARY selects another build of the library (e.g. a tuning variant)
LIB_PATH = os.environ.get("LZK_LIBRARY") or os.path.join(_HERE, "liblzk_b200.so")

c_p = ctypes.c_void_p
c_sz = ctypes.c_size_t
c_u32 = ctypes.c_uint32
c_i = ctypes.c_int

# name -> (restype, argtypes); every function of include/lzk.h
SIGNATURES = {
    "lzk_status_string": (ctypes.c_char_p, [c_i]),
    "lzk_version": (ctypes.c_char_p, []),
    "lzk_field_op": (c_i, [c_i, c_i, c_p, c_p, c_p, c_sz, c_p]),
    "lzk_msm_g1": (c_i, [c_p, c_p, c_sz, c_p, c_p, c_p]),
    "lzk_msm_g2": (c_i, [c_p, c_p, c_sz, c_p, c_p, c_p]),
    "lzk_msm_g1_noalloc": (c_i, [c_p, c_p, c_sz, c_p, c_u32, c_p]),
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
    "lzk_poly_a_times_b_minus_c": (c_i, [c_p, c_p, c_p, c_sz, c_p]),
    "lzk_random_fr": (c_i, [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, c_sz, c_p, c_p]),
    "lzk_g1_fixed_base": (c_i, [c_p, c_sz, c_p, c_p]),
    "lzk_g2_fixed_base": (c_i, [c_p, c_sz, c_p, c_p]),
    "lzk_r1cs_solve": (c_i, [c_p, c_p, c_p, c_p, ctypes.c_uint64, ctypes.c_uint64, c_p]),
    "lzk_r1cs_check": (c_i, [c_p, c_p, c_p, c_p, c_p, c_p]),
    "lzk_prover_create": (c_i, [c_p, c_p, c_i, c_u32, c_p]),
    "lzk_prover_destroy": (c_i, [c_p]),
    "lzk_prover_device_bytes": (c_sz, [c_p]),
    "lzk_groth16_prove": (c_i, [c_p, c_p, c_p, c_p, c_p, c_p]),
    "lzk_groth16_proof_to_wire": (c_i, [c_p, c_p, c_p]),
    "lzk_pk_save": (c_i, [ctypes.c_char_p, c_p, c_p]),
    "lzk_pk_load": (c_i, [ctypes.c_char_p, c_p, c_p, c_p]),
    "lzk_pk_free": (c_i, [c_p]),
    "lzk_groth16_proof_from_wire": (c_i, [c_p, c_p, c_p, c_p]),
    "lzk_server_create": (c_i, [c_p, c_p]),
    "lzk_server_add_circuit": (c_i, [c_p, c_p, c_p]),
    "lzk_server_submit": (c_i, [c_p, c_u32, c_p, c_p, c_p, c_u32, c_p]),
    "lzk_server_poll": (c_i, [c_p, ctypes.c_uint64, c_p, c_p]),
    "lzk_server_cancel": (c_i, [c_p, ctypes.c_uint64]),
    "lzk_server_wait_idle": (c_i, [c_p, c_i]),
    "lzk_server_get_stats": (c_i, [c_p, c_p]),
    "lzk_server_reset_stats": (c_i, [c_p]),
    "lzk_server_destroy": (c_i, [c_p]),
    "lzk_batch_plan_create": (c_i, [c_i, c_p, c_sz, c_p, c_sz, c_p]),
    "lzk_batch_plan_create_ex": (c_i, [c_i, c_p, c_sz, c_p, c_sz, c_u32, c_p]),
    "lzk_batch_plan_run": (c_i, [c_p, c_i, c_p]),
    "lzk_batch_plan_device_bytes": (c_sz, [c_p]),
    "lzk_batch_plan_destroy": (c_i, [c_p]),
    "lzk_msm_set_window": (c_i, [c_i, c_u32, c_u32]),
    "lzk_tune_set": (c_i, [c_i, c_i, c_u32, c_u32]),
    "lzk_tune_get": (c_u32, [c_i, c_i, c_u32]),
    "lzk_trace_enable": (None, [c_i]),
    "lzk_trace_nvtx": (None, [c_i]),
    "lzk_trace_reset": (None, []),
    "lzk_trace_only": (c_i, [ctypes.c_char_p]),
    "lzk_trace_get": (c_i, [ctypes.c_char_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_uint64)]),
    "lzk_trace_timeline": (c_i, [c_p, c_sz, ctypes.POINTER(c_sz)]),
    "lzk_probe_imad_rate": (c_i, [ctypes.POINTER(ctypes.c_double)]),
    "lzk_probe_mont_rate": (c_i, [ctypes.POINTER(ctypes.c_double)]),
    "lzk_probe_mont_rate_int": (c_i, [ctypes.POINTER(ctypes.c_double)]),
    "lzk_launch_count": (ctypes.c_uint64, []),
    "lzk_debug_fail_allocations": (c_i, [ctypes.c_longlong]),
    "lzk_debug_persistent_barrier": (c_i, [ctypes.c_uint32, ctypes.c_uint32]),
    "lzk_debug_check_word": (c_u32, [c_i]),
    "lzk_debug_checks_enabled": (c_i, []),
}


class MsmCfg(ctypes.Structure):
    """struct lzk_msm_cfg"""

    _fields_ = [
        ("window_bits", ctypes.c_uint32),
        ("flags", ctypes.c_uint32),
        ("precomp_windows", ctypes.c_uint32),
        ("base_layout", ctypes.c_uint32),
        ("level_stride", ctypes.c_size_t),
        ("workspace", ctypes.c_void_p),
        ("workspace_bytes", ctypes.c_size_t),
        ("acc_chunk", ctypes.c_uint32),
        ("reduce_run", ctypes.c_uint32),
    ]


LZK_MSM_PRECOMPUTED = 0x1
BASES_AFFINE, BASES_REF_G1_JAC, BASES_REF_G2_LANES = 0, 1, 2
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


class MsmDesc(ctypes.Structure):
    """struct lzk_msm_desc"""

    _fields_ = [("scalars", ctypes.c_void_p), ("bases", ctypes.c_void_p), ("n", ctypes.c_size_t),
                ("out", ctypes.c_void_p), ("window_bits", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


class NttDesc(ctypes.Structure):
    """struct lzk_ntt_desc"""

    _fields_ = [("data", ctypes.c_void_p), ("log_n", ctypes.c_uint32), ("direction", ctypes.c_int)]


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


def trace_enable(on=True):
    lib().lzk_trace_enable(1 if on else 0)


def trace_only(names=None):
    """trace only these region names (an iterable of str; None = all)"""
    call("lzk_trace_only", ",".join(names).encode() if names else None)


def trace_reset():
    lib().lzk_trace_reset()


def trace_get(name):
    """(total device ms, count) of completed regions named `name`"""
    ms, cnt = ctypes.c_double(), ctypes.c_uint64()
    call("lzk_trace_get", name.encode(), ctypes.byref(ms), ctypes.byref(cnt))
    return ms.value, cnt.value


class TraceSpan(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 40), ("start_ms", ctypes.c_double), ("end_ms", ctypes.c_double)]


def trace_timeline():
    """[(name, start ms, end ms)] of the regions completed since the last
    reset, on one device clock whose zero is the first region's start"""
    n = ctypes.c_size_t()
    call("lzk_trace_timeline", None, 0, ctypes.byref(n))
    buf = (TraceSpan * max(n.value, 1))()
    call("lzk_trace_timeline", buf, n.value, ctypes.byref(n))
    return [(t.name.decode(), t.start_ms, t.end_ms) for t in buf[:n.value]]


def probe_imad_rate():
    r = ctypes.c_double()
    call("lzk_probe_imad_rate", ctypes.byref(r))
    return r.value


def probe_mont_rate():
    r = ctypes.c_double()
    call("lzk_probe_mont_rate", ctypes.byref(r))
    return r.value


def probe_mont_rate_int():
    r = ctypes.c_double()
    call("lzk_probe_mont_rate_int", ctypes.byref(r))
    return r.value


def launch_count():
    return int(lib().lzk_launch_count())
