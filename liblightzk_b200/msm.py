"""Multi-scalar multiplication over BN254 G1/G2 on the device.

Thin wrappers over lzk_msm_g1/_g2, lzk_g*_precompute and lzk_g*_to_affine
(include/lzk.h).  All tensors are device tensors holding the limb layout of
include/lzk.h (int64 storage of uint64 limbs):
  scalars (n, 4)  bases G1 (n, 2, 4) / G2 (n, 2, 2, 4)
  result  G1 (3, 4) / G2 (3, 2, 4) Jacobian.
"""
import ctypes

import torch

from . import _capi
from .device import ptr, stream_ptr

_AFF_SHAPE = {1: (2, 4), 2: (2, 2, 4)}
_JAC_SHAPE = {1: (3, 4), 2: (3, 2, 4)}


def _cfg(window_bits=0, flags=0, windows=0, level_stride=0, workspace=None):
    c = _capi.MsmCfg()
    c.window_bits = window_bits
    c.flags = flags
    c.precomp_windows = windows
    c.level_stride = level_stride
    if workspace is not None:
        c.workspace = workspace.data_ptr()
        c.workspace_bytes = workspace.numel() * workspace.element_size()
    return c


def msm(group, scalars, bases, window_bits=0, out=None, stream=None, workspace=None):
    """sum_i scalars[i] * bases[i] for plain affine bases; returns Jacobian."""
    n = scalars.shape[0]
    assert bases.shape[0] >= n
    if out is None:
        out = torch.empty(_JAC_SHAPE[group], dtype=torch.int64, device=scalars.device)
    cfg = _cfg(window_bits, workspace=workspace)
    name = "lzk_msm_g1" if group == 1 else "lzk_msm_g2"
    _capi.call(name, ptr(scalars), ptr(bases), n, ptr(out), ctypes.byref(cfg), stream_ptr(stream))
    return out


def windows_for(window_bits):
    return int(_capi.lib().lzk_msm_precomp_windows(window_bits))


def autotune_window(group, n, precomputed=False):
    return int(_capi.lib().lzk_msm_autotune_window(group, n, _capi.LZK_MSM_PRECOMPUTED if precomputed else 0))


def precompute(group, bases, window_bits, windows=None, level_stride=None, stream=None):
    """Table of shifted copies 2^(j*c) * P_i (affine), j < windows."""
    n = bases.shape[0]
    windows = windows or windows_for(window_bits)
    level_stride = level_stride or n
    table = torch.empty((windows * level_stride,) + _AFF_SHAPE[group], dtype=torch.int64, device=bases.device)
    name = "lzk_g1_precompute" if group == 1 else "lzk_g2_precompute"
    _capi.call(name, ptr(bases), n, window_bits, windows, ptr(table), level_stride, stream_ptr(stream))
    return table


def msm_precomputed(group, scalars, table, window_bits, windows, level_stride, out=None, stream=None,
                    workspace=None):
    """MSM over a shifted-copy table (every window shares one bucket set)."""
    n = scalars.shape[0]
    if out is None:
        out = torch.empty(_JAC_SHAPE[group], dtype=torch.int64, device=scalars.device)
    cfg = _cfg(window_bits, _capi.LZK_MSM_PRECOMPUTED, windows, level_stride, workspace)
    name = "lzk_msm_g1" if group == 1 else "lzk_msm_g2"
    _capi.call(name, ptr(scalars), ptr(table), n, ptr(out), ctypes.byref(cfg), stream_ptr(stream))
    return out


def workspace_bytes(group, n, window_bits=0, precomputed=False, level_stride=0):
    cfg = _cfg(window_bits, _capi.LZK_MSM_PRECOMPUTED if precomputed else 0, 0, level_stride)
    return int(_capi.lib().lzk_msm_workspace_bytes(group, n, ctypes.byref(cfg)))


def to_affine(group, jac, stream=None):
    """Jacobian (n, 3, ...) -> affine (n, 2, ...); infinity -> (0, 0)."""
    n = jac.shape[0]
    out = torch.empty((n,) + _AFF_SHAPE[group], dtype=torch.int64, device=jac.device)
    name = "lzk_g1_to_affine" if group == 1 else "lzk_g2_to_affine"
    _capi.call(name, ptr(jac), ptr(out), n, stream_ptr(stream))
    return out
