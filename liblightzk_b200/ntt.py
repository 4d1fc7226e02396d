"""NTT over Fr and R1CS evaluation (SpMV) on the device.

Wrappers over lzk_ntt / lzk_ntt_batch / lzk_number_theory_transformation
and lzk_spmv3 (include/lzk.h).  Data are device tensors (n, 4) of
Montgomery limbs (int64 storage).
"""
import ctypes

from . import _capi
from .device import ptr, stream_ptr

FORWARD, INVERSE, COSET_FORWARD, COSET_INVERSE = 0, 1, 2, 3


def ntt(data, log_n, direction=FORWARD, stream=None):
    """in-place transform of data[:2^log_n]"""
    assert data.shape[0] >= (1 << log_n)
    _capi.call("lzk_ntt", ptr(data), log_n, direction, stream_ptr(stream))
    return data


def ntt_batch(data, log_n, count, stride, direction=FORWARD, stream=None):
    _capi.call("lzk_ntt_batch", ptr(data), log_n, count, stride, direction, stream_ptr(stream))
    return data


def prepare(log_n):
    _capi.call("lzk_ntt_prepare", log_n)


def number_theory_transformation(deg, log_deg, coeffs, omega_powers, factor=None, stream=None):
    """the reference's operator (poly.cuh:65-73) with the caller's table"""
    _capi.call("lzk_number_theory_transformation", deg, log_deg, ptr(coeffs), ptr(omega_powers), ptr(factor),
               stream_ptr(stream))
    return coeffs


def csr(val, col_idx, row_ptr, rows, cols, nnz):
    """lzk_csr over device tensors; index width from col_idx's dtype"""
    c = _capi.Csr()
    c.val, c.col_idx, c.row_ptr = ptr(val), ptr(col_idx), ptr(row_ptr)
    c.rows, c.cols, c.nnz = rows, cols, nnz
    c.index_bytes = col_idx.element_size()
    return c


def spmv3(A, B, C, z, Az, Bz, Cz, stream=None):
    """Az = A*z, Bz = B*z, Cz = C*z (A, B, C: lzk_csr or None)"""
    ref = lambda m: ctypes.byref(m) if m is not None else None  # noqa: E731
    _capi.call("lzk_spmv3", ref(A), ref(B), ref(C), ptr(z), ptr(Az), ptr(Bz), ptr(Cz), stream_ptr(stream))
