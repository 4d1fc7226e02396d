"""Drop-in check: a C++ program written against the reference's operator
names (tests/compat/msm_check.cpp, the shape of the reference's
test/msm-check.cu) links liblzk_b200.so through include/lzk_compat.hpp and
runs multi_scalar_multiplication_g1/_g2 on tables in the reference's own
record layouts (Jacobian Z = 1 G1 records; G2 lane-pair halves),
number_theory_transformation with an ntt_setup table, the SpMV over size_t
descriptors and polynomial_A_times_B_minus_C.  Outputs are compared with the
oracle."""
import os
import subprocess

import numpy as np
import pytest

from oracle import FR, MUL, SUB

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _build(tmp):
    exe = os.path.join(tmp, "msm_check")
    libdir = os.path.join(ROOT, "liblightzk_b200")
    cmd = ["/usr/bin/g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include",
           os.path.join(ROOT, "tests", "compat", "msm_check.cpp"), "-o", exe, "-L", libdir, "-llzk_b200",
           "-L", "/usr/local/cuda/lib64", "-lcudart", f"-Wl,-rpath,{libdir}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_reference_call_sites(cuda, orc, rng_state, tmp_path):
    from liblightzk_b200 import device, msm
    tmp = str(tmp_path)
    n, c = 300, 12
    W = msm.windows_for(c)     # 22, as the reference's Setup(12) (groth16.cuh:52)
    s = orc.rand_field(FR, n, rng_state)
    b1 = orc.fixed_base(1, orc.rand_field(FR, n, rng_state))
    b2 = orc.fixed_base(2, orc.rand_field(FR, n, rng_state))
    t1 = device.to_host(msm.precompute(1, device.to_device(b1), c, W, n))   # (W*n, 2, 4) affine
    t2 = device.to_host(msm.precompute(2, device.to_device(b2), c, W, n))   # (W*n, 2, 2, 4)
    one = orc.to_mont(1, np.array([[1, 0, 0, 0]], np.uint64))[0]
    inf1 = (t1 == 0).all(axis=(1, 2))
    jac = np.zeros((W * n, 3, 4), np.uint64)
    jac[:, :2] = t1
    jac[:, 2] = one
    jac[inf1, 2] = 0
    lanes = np.zeros((W * n, 2, 3, 4), np.uint64)       # [X.c0 Y.c0 Z.c0][X.c1 Y.c1 Z.c1]
    lanes[:, 0, 0], lanes[:, 1, 0] = t2[:, 0, 0], t2[:, 0, 1]
    lanes[:, 0, 1], lanes[:, 1, 1] = t2[:, 1, 0], t2[:, 1, 1]
    lanes[:, 0, 2] = one
    log_deg = 9
    M = 1 << log_deg
    params = orc.ntt_setup(M)
    nin = orc.rand_field(FR, M, rng_state)
    rows, cols = 400, 100
    rng = np.random.default_rng(5)
    z = orc.rand_field(FR, cols, rng_state)
    mats = []
    for name, mx in (("a", 3), ("b", 1), ("c", 2)):
        per = rng.integers(0, mx + 1, rows)
        rp = np.concatenate([[0], np.cumsum(per)[:-1]]).astype(np.uint64)
        col = rng.integers(0, cols, int(per.sum())).astype(np.uint64)
        val = orc.rand_field(FR, int(per.sum()), rng_state)
        mats.append((val, col, rp))
        val.tofile(os.path.join(tmp, f"{name}_val.bin"))
        col.tofile(os.path.join(tmp, f"{name}_col.bin"))
        rp.tofile(os.path.join(tmp, f"{name}_rp.bin"))
    np.array([n, c, W, log_deg, rows, 0, cols], np.uint64).tofile(os.path.join(tmp, "meta.bin"))
    s.tofile(os.path.join(tmp, "scalars.bin"))
    jac.tofile(os.path.join(tmp, "table_g1.bin"))
    lanes.tofile(os.path.join(tmp, "table_g2.bin"))
    params.tofile(os.path.join(tmp, "ntt_params.bin"))
    nin.tofile(os.path.join(tmp, "ntt_in.bin"))
    z.tofile(os.path.join(tmp, "z.bin"))

    exe = _build(tmp)
    r = subprocess.run([exe, tmp], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "compat ok" in r.stdout, r.stdout + r.stderr

    g1 = np.fromfile(os.path.join(tmp, "out_g1.bin"), np.uint64).reshape(3, 4)
    g2 = np.fromfile(os.path.join(tmp, "out_g2.bin"), np.uint64).reshape(3, 2, 4)
    assert (orc.jac_to_aff(1, g1[None]) == orc.jac_to_aff(1, orc.msm(1, s, b1)[None])).all()
    assert (orc.jac_to_aff(2, g2[None]) == orc.jac_to_aff(2, orc.msm(2, s, b2)[None])).all()
    got = np.fromfile(os.path.join(tmp, "out_ntt.bin"), np.uint64).reshape(M, 4)
    assert (got == orc.ntt_ref(nin, params[M:2 * M], params[2 * M])).all()
    sp = [orc.spmv(v, cl, rp, z) for v, cl, rp in mats]
    expect = orc.field_op(FR, SUB, orc.field_op(FR, MUL, sp[0], sp[1]), sp[2])
    got = np.fromfile(os.path.join(tmp, "out_abc.bin"), np.uint64).reshape(rows, 4)
    assert (got == expect).all()


@pytest.mark.parametrize("g", [1, 2])
def test_reference_layout_plain_bases(cuda, orc, rng_state, g):
    """reference-layout records without shifted copies (flags = 0)"""
    import ctypes

    from liblightzk_b200 import _capi, device
    n = 257
    s = orc.rand_field(FR, n, rng_state)
    b = orc.fixed_base(g, orc.rand_field(FR, n, rng_state))
    b[5] = 0   # infinity
    one = orc.to_mont(1, np.array([[1, 0, 0, 0]], np.uint64))[0]
    if g == 1:
        rec = np.zeros((n, 3, 4), np.uint64)
        rec[:, :2] = b
        rec[:, 2] = one
        rec[5, 2] = 0
    else:
        rec = np.zeros((n, 2, 3, 4), np.uint64)
        rec[:, 0, 0], rec[:, 1, 0], rec[:, 0, 1], rec[:, 1, 1] = b[:, 0, 0], b[:, 0, 1], b[:, 1, 0], b[:, 1, 1]
        rec[:, 0, 2] = one
        rec[5, :, 2] = 0
    cfg = _capi.MsmCfg()
    cfg.base_layout = _capi.BASES_REF_G1_JAC if g == 1 else _capi.BASES_REF_G2_LANES
    out = device.empty((3, 4) if g == 1 else (3, 2, 4))
    ds, dr = device.to_device(s), device.to_device(rec)
    _capi.call(f"lzk_msm_g{g}", ds.data_ptr(), dr.data_ptr(), n, out.data_ptr(), ctypes.byref(cfg), None)
    got = device.to_host(out)
    assert (orc.jac_to_aff(g, got[None]) == orc.jac_to_aff(g, orc.msm(g, s, b)[None])).all()
    cfg.base_layout = 2 if g == 1 else 1   # the other group's layout is refused
    st = getattr(_capi.lib(), f"lzk_msm_g{g}")(ds.data_ptr(), dr.data_ptr(), n, out.data_ptr(), ctypes.byref(cfg), None)
    assert st == -1


def test_groth16_class(cuda, orc, tmp_path):
    """Groth16_BN254(input_scale::MatMul_p_39).Setup(12).Prove() from a C++
    program (tests/compat/groth16_check.cpp, the shape of test/groth16.cu)
    gives the proof the Python prover gives on the same seeded instance,
    in the reference's chain mode; its printed affine coordinates are the
    wire form's numbers."""
    from liblightzk_b200 import device, groth16, synth
    libdir = os.path.join(ROOT, "liblightzk_b200")
    exe = os.path.join(str(tmp_path), "groth16_check")
    cmd = ["/usr/bin/g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include",
           os.path.join(ROOT, "tests", "compat", "groth16_check.cpp"), "-o", exe, "-L", libdir, "-llzk_b200",
           "-L", "/usr/local/cuda/lib64", "-lcudart", f"-Wl,-rpath,{libdir}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    seed = 7
    r = subprocess.run([exe, str(seed)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    lines = r.stdout.splitlines()
    wire = np.array([int(x, 16) for x in next(l for l in lines if l.startswith("WIRE")).split()[1:]], np.uint32)
    # the printed proof: A (x, y), C (x, y), B (x.c0, x.c1, y.c0, y.c1), most significant digit first
    hexes = [l for l in lines if len(l) == 64]
    order = [0, 1, 6, 7, 2, 3, 4, 5]          # wire coordinates in print order
    assert [int(h, 16) for h in hexes] == [int("".join(f"{w:08x}" for w in wire[8 * k:8 * k + 8][::-1]), 16)
                                           for k in order]
    circ = synth.MatMulCircuit(39)
    z = circ.witness(seed + 100)
    pk = synth.ProvingKey(circ, seed=seed)
    rs = device.to_host(synth.random_fr(2, seed + 200, 99))
    prover = groth16.Prover(circ, pk, mode=groth16.REFERENCE, window_bits=12)
    want = device.to_host(groth16.to_wire(prover.prove(z, rs[0], rs[1]))).view(np.uint32)
    prover.close()
    assert (wire == want).all()
