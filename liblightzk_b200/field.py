"""Element-wise field arithmetic on device arrays (lzk_field_op).

Arrays are device tensors holding Montgomery limbs: Fr / Fq (n, 4), Fq2
(n, 2, 4).  The operation codes follow include/lzk.h (LZK_FOP_*).
"""
import torch

from . import _capi
from .device import ptr, stream_ptr

FR, FQ, FQ2 = 0, 1, 2
ADD, SUB, MUL, SQR, NEG, INV, FROM_MONT, TO_MONT = range(8)


def field_op(field, op, a, b=None, out=None, stream=None):
    """out[i] = a[i] op b[i] (unary ops ignore b); returns out"""
    n = a.shape[0]
    if out is None:
        out = torch.empty_like(a)
    _capi.call("lzk_field_op", field, op, ptr(a), ptr(b), ptr(out), n, stream_ptr(stream))
    return out
