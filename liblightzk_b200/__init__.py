"""liblightzk_b200 -- a B200 (sm_100a) Groth16 prover hot path for BN254.

The compute lives in liblzk_b200.so (hand-written CUDA, C ABI in
include/lzk.h).  This package is the host side above that ABI:
  _capi    ctypes binding of every entry point
  device   torch tensors as raw HBM buffers
  msm      multi-scalar multiplication (G1, G2, shifted-base tables)
"""
from . import _capi, device, msm  # noqa: F401
from ._capi import LzkError, lib  # noqa: F401

__all__ = ["lib", "LzkError", "msm", "device"]
