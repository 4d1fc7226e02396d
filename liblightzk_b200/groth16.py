"""Groth16 prover over the C ABI (lzk_prover_create / lzk_groth16_prove).

    prover = Prover(circuit, pk, mode=STANDARD)
    proof = prover.prove(z, r, s)     # device tensor (48,) int64:
                                      # A (3,4) | B (3,2,4) | C (3,4) Jacobian
"""
import ctypes

import numpy as np
import torch

from . import _capi
from .device import ptr, stream_ptr, to_host

STANDARD, REFERENCE = 0, 1


class _Fq(ctypes.Structure):
    _fields_ = [("limb", ctypes.c_uint64 * 4)]


class _G1Aff(ctypes.Structure):
    _fields_ = [("x", _Fq), ("y", _Fq)]


class _G2Aff(ctypes.Structure):
    _fields_ = [("x", _Fq * 2), ("y", _Fq * 2)]


class Circuit(ctypes.Structure):
    """struct lzk_groth16_circuit"""

    _fields_ = [("A", _capi.Csr), ("B", _capi.Csr), ("C", _capi.Csr), ("n_vars", ctypes.c_uint64),
                ("n_public", ctypes.c_uint64), ("log_domain", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


class Pk(ctypes.Structure):
    """struct lzk_groth16_pk"""

    _fields_ = [("a_query", ctypes.c_void_p), ("b1_query", ctypes.c_void_p), ("b2_query", ctypes.c_void_p),
                ("l_query", ctypes.c_void_p), ("h_query", ctypes.c_void_p), ("alpha1", _G1Aff), ("beta1", _G1Aff),
                ("delta1", _G1Aff), ("beta2", _G2Aff), ("delta2", _G2Aff)]


class PkInfo(ctypes.Structure):
    """struct lzk_pk_info"""

    _fields_ = [("n_vars", ctypes.c_uint64), ("n_public", ctypes.c_uint64), ("log_domain", ctypes.c_uint32),
                ("version", ctypes.c_uint32)]


def _fill(struct, t):
    """copy a device point tensor's limbs into a ctypes affine struct"""
    a = to_host(t).reshape(-1)
    ctypes.memmove(ctypes.addressof(struct), a.ctypes.data, ctypes.sizeof(struct))


def fr_struct(v):
    """host Fr value (4 uint64 Montgomery limbs) as a ctypes object"""
    f = _Fq()
    a = np.ascontiguousarray(v, dtype=np.uint64).reshape(4)
    for i in range(4):
        f.limb[i] = int(a[i])
    return f


PROOF_WORDS = 12 + 24 + 12


def split_proof(proof):
    """device/host proof (48,) -> (A (3,4), B (3,2,4), C (3,4)) numpy"""
    p = to_host(proof) if isinstance(proof, torch.Tensor) else np.asarray(proof, np.uint64)
    return p[:12].reshape(3, 4), p[12:36].reshape(3, 2, 4), p[36:48].reshape(3, 4)


WIRE_BYTES = 256


def to_wire(proof, stream=None):
    """device proof (48 int64 words) -> its 256-byte wire form (device, 32
    int64 words): affine A, B, C as canonical little-endian integers"""
    wire = torch.empty(WIRE_BYTES // 8, dtype=torch.int64, device=proof.device)
    _capi.call("lzk_groth16_proof_to_wire", ptr(proof), ptr(wire), stream_ptr(stream))
    return wire


def from_wire(wire, stream=None):
    """wire form (device) -> (proof with Z = 1, flag tensor: 1 if a
    coordinate was not canonical)"""
    proof = torch.empty(PROOF_WORDS, dtype=torch.int64, device=wire.device)
    bad = torch.zeros(1, dtype=torch.int32, device=wire.device)
    _capi.call("lzk_groth16_proof_from_wire", ptr(wire), ptr(proof), ptr(bad), stream_ptr(stream))
    return proof, bad


def pk_struct(pk):
    """struct lzk_groth16_pk of a key: a LoadedKey's view, or one built from
    the device tensors of a synth.ProvingKey"""
    if isinstance(pk, LoadedKey):
        return pk.view
    k = Pk()
    k.a_query, k.b1_query, k.b2_query = ptr(pk.a), ptr(pk.b1), ptr(pk.b2)
    k.l_query, k.h_query = ptr(pk.l), ptr(pk.h)
    _fill(k.alpha1, pk.alpha1)
    _fill(k.beta1, pk.beta1)
    _fill(k.delta1, pk.delta1)
    _fill(k.beta2, pk.beta2)
    _fill(k.delta2, pk.delta2)
    return k


def save_key(path, pk, circuit):
    """write the proving key of `circuit` to a key file (lzk_pk_save)"""
    info = PkInfo(circuit.n_vars, circuit.n_public, circuit.log_m, 0)
    torch.cuda.synchronize()
    _capi.call("lzk_pk_save", str(path).encode(), ctypes.byref(pk_struct(pk)), ctypes.byref(info))


class LoadedKey:
    """a key file loaded into device memory (lzk_pk_load); `view` is the
    lzk_groth16_pk for lzk_prover_create, `info` the circuit shape"""

    def __init__(self, path):
        self.view, self.info = Pk(), PkInfo()
        h = ctypes.c_void_p()
        _capi.call("lzk_pk_load", str(path).encode(), ctypes.byref(h), ctypes.byref(self.view),
                   ctypes.byref(self.info))
        self.handle = h

    def close(self):
        if self.handle:
            _capi.call("lzk_pk_free", self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Prover:
    def __init__(self, circuit, pk, mode=STANDARD, window_bits=0):
        """pk: a synth.ProvingKey (device tensors) or a LoadedKey"""
        self.circuit = circuit   # keeps the CSR tensors alive
        c = Circuit()
        c.A, c.B, c.C = circuit.A.desc(), circuit.B.desc(), circuit.C.desc()
        c.n_vars, c.n_public, c.log_domain = circuit.n_vars, circuit.n_public, circuit.log_m
        if isinstance(pk, LoadedKey):
            i = pk.info
            if (i.n_vars, i.n_public, i.log_domain) != (circuit.n_vars, circuit.n_public, circuit.log_m):
                raise ValueError("key file was saved for another circuit shape")
        k = pk_struct(pk)
        self._c, self._k = c, k
        h = ctypes.c_void_p()
        _capi.call("lzk_prover_create", ctypes.byref(c), ctypes.byref(k), mode, window_bits, ctypes.byref(h))
        self.handle = h
        self.mode = mode

    def device_bytes(self):
        return int(_capi.lib().lzk_prover_device_bytes(self.handle))

    def prove(self, z, r, s, proof=None, stream=None):
        if proof is None:
            proof = torch.empty(PROOF_WORDS, dtype=torch.int64, device=z.device)
        rr, ss = fr_struct(r), fr_struct(s)
        _capi.call("lzk_groth16_prove", self.handle, ptr(z), ctypes.byref(rr), ctypes.byref(ss), ptr(proof),
                   stream_ptr(stream))
        return proof

    def close(self):
        if self.handle:
            _capi.call("lzk_prover_destroy", self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
