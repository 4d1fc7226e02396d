"""NTT and SpMV parity: CUDA path through the C ABI against the oracle's
restatement of the reference's number_theory_transformation (poly.cuh:32-73,
pinned to the reference by the golden fixtures) and of
batch_sparse_matrix_vector_multiplication (poly.cuh:5-30).  Bit-exact."""
import numpy as np
import pytest

from oracle import FR

pytestmark = pytest.mark.gpu


def _dev(a):
    from liblightzk_b200 import device
    return device.to_device(a)


def _host(t):
    from liblightzk_b200 import device
    return device.to_host(t)


@pytest.mark.parametrize("logn", [0, 1, 2, 3, 5, 8, 11, 12, 13, 16, 20])
@pytest.mark.parametrize("direction", [0, 1, 2, 3])
def test_ntt_directions(cuda, orc, rng_state, logn, direction):
    from liblightzk_b200 import ntt
    if logn >= 16 and direction in (1, 2):
        pytest.skip("large sizes: forward and coset-inverse cover both table kinds")
    n = 1 << logn
    a = orc.rand_field(FR, n, rng_state)
    d = _dev(a)
    ntt.ntt(d, logn, direction)
    assert (_host(d) == orc.ntt(a, logn, direction)).all()


@pytest.mark.parametrize("logn", [4, 10, 15])
def test_ntt_roundtrip_and_batch(cuda, orc, rng_state, logn):
    from liblightzk_b200 import ntt
    n, count = 1 << logn, 3
    stride = n + 8
    a = orc.rand_field(FR, stride * count, rng_state)
    d = _dev(a)
    ntt.ntt_batch(d, logn, count, stride, ntt.COSET_FORWARD)
    got = _host(d)
    for t in range(count):
        seg = a[t * stride: t * stride + n]
        assert (got[t * stride: t * stride + n] == orc.ntt(seg, logn, 2)).all()
        assert (got[t * stride + n: (t + 1) * stride] == a[t * stride + n: (t + 1) * stride]).all()
    ntt.ntt_batch(d, logn, count, stride, ntt.COSET_INVERSE)
    assert (_host(d) == a).all()


@pytest.mark.parametrize("logn", [3, 9, 14])
def test_number_theory_transformation_reference_table(cuda, orc, rng_state, logn):
    """the reference's operator signature with an ntt_setup table
    (groth16-operator.cuh:6-31): iNTT_M with factor M^-1, then NTT_2M"""
    from liblightzk_b200 import ntt
    M = 1 << logn
    tab = orc.ntt_setup(M)
    a = orc.rand_field(FR, M, rng_state)
    dt = _dev(tab)
    d = _dev(a)
    ntt.number_theory_transformation(M, logn, d, dt[M:2 * M], dt[2 * M:2 * M + 1])
    assert (_host(d) == orc.ntt_ref(a, tab[M:2 * M], tab[2 * M])).all()
    b = np.concatenate([a, np.zeros_like(a)])
    d2 = _dev(b)
    ntt.number_theory_transformation(2 * M, logn + 1, d2, dt[2 * M + 1:4 * M + 1], None)
    assert (_host(d2) == orc.ntt_ref(b, tab[2 * M + 1:4 * M + 1])).all()


def _rand_csr(rng, orc, st, rows, cols, maxnnz, ones_frac=0.5):
    per = rng.integers(0, maxnnz + 1, rows)
    row_ptr = np.concatenate([[0], np.cumsum(per)[:-1]]).astype(np.uint64)
    nnz = int(per.sum())
    col = rng.integers(0, cols, nnz).astype(np.uint64)
    val = orc.rand_field(FR, nnz, st)
    one = orc.to_mont(FR, np.array([[1, 0, 0, 0]], np.uint64))[0]
    val[rng.random(nnz) < ones_frac] = one
    return val, col, row_ptr, nnz


@pytest.mark.parametrize("index_bytes", [4, 8])
def test_spmv3(cuda, orc, rng_state, index_bytes):
    from liblightzk_b200 import ntt
    rng = np.random.default_rng(3)
    rows, cols = 5000, 3000
    z = orc.rand_field(FR, cols, rng_state)
    dz = _dev(z)
    mats, outs, expect = [], [], []
    for mx in (3, 1, 6):
        val, col, rp, nnz = _rand_csr(rng, orc, rng_state, rows, cols, mx)
        it = np.uint32 if index_bytes == 4 else np.uint64
        t = (_dev(val), _dev(col.astype(it)), _dev(rp.astype(it)))
        mats.append((t, ntt.csr(t[0], t[1], t[2], rows, cols, nnz)))
        outs.append(_dev(np.zeros((rows, 4), np.uint64)))
        expect.append(orc.spmv(val, col, rp, z))
    ntt.spmv3(mats[0][1], mats[1][1], mats[2][1], dz, *outs)
    for o, e in zip(outs, expect):
        assert (_host(o) == e).all()


def test_spmv_empty_rows_and_last_row(cuda, orc, rng_state):
    """reference descriptor: row_ptr has `rows` entries, the last row runs to nnz"""
    from liblightzk_b200 import ntt
    rows, cols = 9, 4
    rp = np.array([0, 0, 2, 2, 2, 5, 5, 6, 6], np.uint64)   # last row: [6, nnz)
    nnz = 9
    col = np.array([0, 3, 1, 1, 2, 3, 0, 1, 2], np.uint64)
    val = orc.rand_field(FR, nnz, rng_state)
    z = orc.rand_field(FR, cols, rng_state)
    t = (_dev(val), _dev(col), _dev(rp))
    out = _dev(np.zeros((rows, 4), np.uint64))
    ntt.spmv3(ntt.csr(t[0], t[1], t[2], rows, cols, nnz), None, None, _dev(z), out, None, None)
    assert (_host(out) == orc.spmv(val, col, rp, z)).all()
