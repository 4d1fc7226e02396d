"""Proving keys on disk (lzk_pk_save / lzk_pk_load / lzk_pk_free).

On the CPU: files that are missing, short, of another format or another
shape are refused with LZK_EIO while the header is read, before any device
call.  On the GPU: a key saved and loaded back gives the same proofs as the
key it was saved from (both modes), a flipped byte in the body fails the
checksum, and a server adds a resident circuit straight from its key file
and serves the same proof."""
import ctypes
import os
import struct

import numpy as np
import pytest

from helpers import same_point
from oracle import FR

LZK_EIO = -9
HEADER = 128


def _load_status(path):
    from liblightzk_b200 import _capi, groth16
    view, info, h = groth16.Pk(), groth16.PkInfo(), ctypes.c_void_p()
    st = _capi.lib().lzk_pk_load(str(path).encode(), ctypes.byref(h), ctypes.byref(view), ctypes.byref(info))
    if st == 0:
        _capi.call("lzk_pk_free", h)
    return st


def _header(n_vars=10, n_public=1, log_domain=3, counts=None, magic=b"LZKG16PK", version=1):
    counts = counts or [n_vars, n_vars, n_vars, n_vars - n_public - 1, (1 << log_domain) - 1]
    h = magic + struct.pack("<IIQQII", version, HEADER, n_vars, n_public, log_domain, 0)
    h += struct.pack("<5Q", *counts) + struct.pack("<Q", 0)
    return h + b"\0" * (HEADER - len(h))


def test_bad_key_files_are_refused_before_device_work(tmp_path):
    import liblightzk_b200
    liblightzk_b200.lib()
    assert _load_status(tmp_path / "missing.pk") == LZK_EIO
    cases = {
        "short": _header()[:100],
        "magic": _header(magic=b"NOTAKEY!"),
        "version": _header(version=2),
        "counts": _header(counts=[10, 10, 10, 8, 6]),
        "shape": _header(n_vars=1, n_public=1, counts=[1, 1, 1, 0, 7]),
        "truncated_body": _header() + b"\0" * 64,
    }
    for name, data in cases.items():
        p = tmp_path / f"{name}.pk"
        p.write_bytes(data)
        assert _load_status(p) == LZK_EIO, name


def _prove(orc, prover, z, seed):
    from liblightzk_b200 import groth16
    r, s = orc.rand_field(FR, 2, np.array([seed], np.uint64))
    return groth16.split_proof(prover.prove(z, r, s)), (r, s)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [0, 1])
def test_saved_key_proves_the_same(cuda, orc, tmp_path, mode):
    from liblightzk_b200 import groth16, synth
    circ = synth.Circuit(10, seed=4, n_public=2, n_free=64, block=64)
    z = circ.witness(5)
    pk = synth.ProvingKey(circ, seed=6)
    path = tmp_path / "circuit.pk"
    groth16.save_key(path, pk, circ)
    size = 128 + 3 * 64 + 2 * 128 + (3 * circ.n_vars - circ.n_public - 1 + circ.M - 1) * 64 + circ.n_vars * 128
    assert os.path.getsize(path) == size
    key = groth16.LoadedKey(path)
    assert (key.info.n_vars, key.info.n_public, key.info.log_domain, key.info.version) == \
        (circ.n_vars, circ.n_public, circ.log_m, 1)
    p0 = groth16.Prover(circ, pk, mode=mode, window_bits=9)
    p1 = groth16.Prover(circ, key, mode=mode, window_bits=9)
    key.close()                      # the prover keeps its own tables
    for seed in (7, 8):
        (A0, B0, C0), rs = _prove(orc, p0, z, seed)
        A1, B1, C1 = groth16.split_proof(p1.prove(z, *rs))
        assert same_point(orc, 1, A0, A1) and same_point(orc, 2, B0, B1) and same_point(orc, 1, C0, C1)
    p0.close()
    p1.close()
    # a key saved for one shape is not accepted for another
    other = synth.Circuit(10, seed=4, n_public=3, n_free=64, block=64)
    k2 = groth16.LoadedKey(path)
    with pytest.raises(ValueError):
        groth16.Prover(other, k2, mode=mode, window_bits=9)
    k2.close()


@pytest.mark.gpu
def test_corrupted_key_fails_the_checksum(cuda, tmp_path):
    from liblightzk_b200 import groth16, synth
    circ = synth.Circuit(6, seed=4, n_public=1, n_free=8, block=8)
    pk = synth.ProvingKey(circ, seed=6)
    path = tmp_path / "k.pk"
    groth16.save_key(path, pk, circ)
    data = bytearray(path.read_bytes())
    assert _load_status(path) == 0
    data[HEADER + 1000] ^= 0x40
    path.write_bytes(bytes(data))
    assert _load_status(path) == LZK_EIO


@pytest.mark.gpu
def test_server_adds_a_circuit_from_its_key_file(cuda, orc, tmp_path):
    from liblightzk_b200 import device, groth16, serve, synth
    circ = synth.Circuit(9, seed=21, n_public=1, n_free=32, block=32)
    z = circ.witness(22)
    pk = synth.ProvingKey(circ, seed=23)
    path = tmp_path / "served.pk"
    groth16.save_key(path, pk, circ)
    alone = groth16.Prover(circ, pk, mode=groth16.STANDARD, window_bits=8)
    (A0, B0, C0), (r, s) = _prove(orc, alone, z, 24)
    alone.close()
    srv = serve.Server(8 << 30, max_inflight=2)
    cid = srv.add_key_file(circ, path, mode=groth16.STANDARD, window_bits=8)
    rid = srv.submit(cid, device.to_host(z), r, s)
    A1, B1, C1 = groth16.split_proof(srv.wait(rid))
    srv.close()
    assert same_point(orc, 1, A0, A1) and same_point(orc, 2, B0, B1) and same_point(orc, 1, C0, C1)
