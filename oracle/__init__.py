"""Python bindings of the CPU checkers (test infrastructure only).

* ``Oracle`` wraps ``oracle/liblzk_oracle.so``, the C restatement of the
  reference's Groth16 hot path (``oracle/lzk_oracle.c``).
* ``Ref`` wraps ``oracle/_ref/libref.so``, the reference's own host
  arithmetic (include/host-arith, src/host-arith) built from the reference
  tree by ``oracle/Makefile``, plus the bridge in ``oracle/ref_bridge.cpp``.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg import this package; the product (``liblightzk_b200``) never does.

Arrays are numpy ``uint64`` with the limb layout of the reference's host
types: field element (..., 4) Montgomery limbs; Fq2 (..., 2, 4);
G1 Jacobian (..., 3, 4); G1 affine (..., 2, 4); G2 Jacobian (..., 3, 2, 4);
G2 affine (..., 2, 2, 4).
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liblzk_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libref.so")

FR, FQ = 0, 1
ADD, SUB, MUL, SQR, NEG, INV, FROM_MONT, TO_MONT = range(8)
G_ADD, G_MADD, G_DBL, G_NEG, G_AFF, G_EQ, G_WF = range(7)

_P = ctypes.POINTER(ctypes.c_uint64)


def _p(a):
    if a is None:
        return None
    assert a.dtype == np.uint64 and a.flags["C_CONTIGUOUS"], "need C-contiguous uint64"
    return a.ctypes.data_as(_P)


def _u64(a):
    return np.ascontiguousarray(a, dtype=np.uint64)


class _Lib:
    prefix = ""

    def __init__(self, path):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built (run make -C oracle)")
        self.lib = ctypes.CDLL(path)

    def _f(self, name):
        return getattr(self.lib, self.prefix + name)

    # --- fields ---
    def field_op(self, kind, op, a, b=None):
        a = _u64(a)
        b = None if b is None else _u64(b)
        n = a.size // 4
        out = np.zeros_like(a)
        self._f("field_op")(ctypes.c_int(kind), ctypes.c_int(op), _p(a), _p(b), _p(out), ctypes.c_size_t(n))
        return out

    def fq2_op(self, op, a, b=None):
        a = _u64(a)
        b = None if b is None else _u64(b)
        out = np.zeros_like(a)
        self._f("fq2_op")(ctypes.c_int(op), _p(a), _p(b), _p(out), ctypes.c_size_t(a.size // 8))
        return out

    def to_mont(self, kind, canon):
        return self.field_op(kind, TO_MONT, canon)

    def from_mont(self, kind, mont):
        return self.field_op(kind, FROM_MONT, mont)

    # --- groups ---
    def g1_op(self, op, a, b=None):
        a = _u64(a)
        b = None if b is None else _u64(b)
        n = a.size // 12
        out = np.zeros(n, np.uint64) if op in (G_EQ, G_WF) else np.zeros_like(a)
        self._f("g1_op")(ctypes.c_int(op), _p(a), _p(b), _p(out), ctypes.c_size_t(n))
        return out

    def g2_op(self, op, a, b=None):
        a = _u64(a)
        b = None if b is None else _u64(b)
        n = a.size // 24
        out = np.zeros(n, np.uint64) if op in (G_EQ, G_WF) else np.zeros_like(a)
        self._f("g2_op")(ctypes.c_int(op), _p(a), _p(b), _p(out), ctypes.c_size_t(n))
        return out

    def g1_one(self):
        out = np.zeros((3, 4), np.uint64)
        self._f("g1_one")(_p(out))
        return out

    def g2_one(self):
        out = np.zeros((3, 2, 4), np.uint64)
        self._f("g2_one")(_p(out))
        return out

    def g1_mul(self, s, pts):
        s, pts = _u64(s), _u64(pts)
        out = np.zeros_like(pts)
        self._f("g1_mul")(_p(s), _p(pts), _p(out), ctypes.c_size_t(s.size // 4))
        return out

    def g2_mul(self, s, pts):
        s, pts = _u64(s), _u64(pts)
        out = np.zeros_like(pts)
        self._f("g2_mul")(_p(s), _p(pts), _p(out), ctypes.c_size_t(s.size // 4))
        return out


class Ref(_Lib):
    """The reference's own host arithmetic (oracle/_ref/libref.so)."""

    prefix = "ref_"

    def __init__(self, path=REF_SO):
        super().__init__(path)
        self.lib.ref_init()

    def g1_msm_naive_jac(self, s, jac):
        s, jac = _u64(s), _u64(jac)
        out = np.zeros((3, 4), np.uint64)
        self.lib.ref_g1_msm_naive(_p(s), _p(jac), ctypes.c_size_t(s.size // 4), _p(out))
        return out

    def g2_msm_naive_jac(self, s, jac):
        s, jac = _u64(s), _u64(jac)
        out = np.zeros((3, 2, 4), np.uint64)
        self.lib.ref_g2_msm_naive(_p(s), _p(jac), ctypes.c_size_t(s.size // 4), _p(out))
        return out

    def ntt_table(self, which, k):
        out = np.zeros(4, np.uint64)
        assert self.lib.ref_ntt_table(ctypes.c_int(which), ctypes.c_size_t(k), _p(out)) == 0
        return out

    def ntt_setup(self, M):
        out = np.zeros((6 * M + 2, 4), np.uint64)
        assert self.lib.ref_ntt_setup(ctypes.c_size_t(M), _p(out)) == 0
        return out

    def ntt_ref(self, coeffs, omega_powers, factor=None):
        c = _u64(coeffs).copy()
        self.lib.ref_ntt(_p(c), ctypes.c_size_t(c.size // 4), _p(_u64(omega_powers)),
                         None if factor is None else _p(_u64(factor)))
        return c

    def spmv(self, val, col_idx, row_ptr, z):
        val, col_idx, row_ptr, z = _u64(val), _u64(col_idx), _u64(row_ptr), _u64(z)
        rows = row_ptr.size
        out = np.zeros((rows, 4), np.uint64)
        self.lib.ref_spmv(_p(val), _p(col_idx), _p(row_ptr), ctypes.c_size_t(rows),
                          ctypes.c_size_t(val.size // 4), _p(z), _p(out))
        return out

    def groth16_assemble(self, alpha1, beta1, delta1, beta2, delta2, g1res, g2res, r, s):
        og1 = np.zeros((2, 3, 4), np.uint64)
        og2 = np.zeros((3, 2, 4), np.uint64)
        args = [_u64(x) for x in (alpha1, beta1, delta1, beta2, delta2, g1res, g2res, r, s)]
        self.lib.ref_groth16_assemble(*[_p(a) for a in args], _p(og1), _p(og2))
        return og1, og2


class Oracle(_Lib):
    """The C restatement (oracle/liblzk_oracle.so)."""

    prefix = "orc_"

    def __init__(self, path=ORACLE_SO):
        super().__init__(path)
        self.lib.orc_rand_u64.restype = ctypes.c_uint64

    def rand_field(self, kind, n, state):
        """n uniform elements (Montgomery limbs); state: np.uint64 array of 1."""
        out = np.zeros((n, 4), np.uint64)
        self.lib.orc_rand_field(ctypes.c_int(kind), _p(state), _p(out), ctypes.c_size_t(n))
        return out

    def jac_to_aff(self, g, jac):
        jac = _u64(jac)
        n = jac.size // (12 if g == 1 else 24)
        out = np.zeros((n, 2, 4) if g == 1 else (n, 2, 2, 4), np.uint64)
        getattr(self.lib, f"orc_g{g}_jac_to_aff")(_p(jac), _p(out), ctypes.c_size_t(n))
        return out

    def aff_to_jac(self, g, aff):
        aff = _u64(aff)
        n = aff.size // (8 if g == 1 else 16)
        out = np.zeros((n, 3, 4) if g == 1 else (n, 3, 2, 4), np.uint64)
        getattr(self.lib, f"orc_g{g}_aff_to_jac")(_p(aff), _p(out), ctypes.c_size_t(n))
        return out

    def fixed_base(self, g, k):
        k = _u64(k)
        n = k.size // 4
        out = np.zeros((n, 2, 4) if g == 1 else (n, 2, 2, 4), np.uint64)
        getattr(self.lib, f"orc_g{g}_fixed_base")(_p(k), _p(out), ctypes.c_size_t(n))
        return out

    def msm(self, g, s, aff, naive=False):
        s, aff = _u64(s), _u64(aff)
        out = np.zeros((3, 4) if g == 1 else (3, 2, 4), np.uint64)
        name = f"orc_g{g}_msm" + ("_naive" if naive else "")
        getattr(self.lib, name)(_p(s), _p(aff), ctypes.c_size_t(s.size // 4), _p(out))
        return out

    def ntt_table(self, which, k):
        out = np.zeros(4, np.uint64)
        assert self.lib.orc_ntt_table(ctypes.c_int(which), ctypes.c_uint32(k), _p(out)) == 0
        return out

    def ntt_setup(self, M):
        out = np.zeros((6 * M + 2, 4), np.uint64)
        assert self.lib.orc_ntt_setup(ctypes.c_size_t(M), _p(out)) == 0
        return out

    def ntt_ref(self, coeffs, omega_powers, factor=None):
        c = _u64(coeffs).copy()
        self.lib.orc_ntt_ref(_p(c), ctypes.c_size_t(c.size // 4), _p(_u64(omega_powers)),
                             None if factor is None else _p(_u64(factor)))
        return c

    def ntt(self, data, log_n, direction):
        d = _u64(data).copy()
        assert self.lib.orc_ntt(_p(d), ctypes.c_uint32(log_n), ctypes.c_int(direction)) == 0
        return d

    def spmv(self, val, col_idx, row_ptr, z):
        val, col_idx, row_ptr, z = _u64(val), _u64(col_idx), _u64(row_ptr), _u64(z)
        rows = row_ptr.size
        out = np.zeros((rows, 4), np.uint64)
        self.lib.orc_spmv(_p(val), _p(col_idx), _p(row_ptr), ctypes.c_size_t(rows),
                          ctypes.c_size_t(val.size // 4), _p(z), _p(out))
        return out


def have_ref():
    return os.path.exists(REF_SO)


class _OrcCsr(ctypes.Structure):
    _fields_ = [("val", _P), ("col", _P), ("row_ptr", _P), ("rows", ctypes.c_size_t), ("nnz", ctypes.c_size_t)]


class _OrcG16(ctypes.Structure):
    _fields_ = [("A", _OrcCsr), ("B", _OrcCsr), ("C", _OrcCsr), ("n_vars", ctypes.c_size_t),
                ("n_public", ctypes.c_size_t), ("log_m", ctypes.c_uint32),
                ("a_query", _P), ("b1_query", _P), ("b2_query", _P), ("l_query", _P), ("h_query", _P),
                ("alpha1", _P), ("beta1", _P), ("delta1", _P), ("beta2", _P), ("delta2", _P)]


def _groth16_struct(mats, rows, n_vars, n_public, log_m, keys):
    """mats: 3 tuples (val, col, row_ptr) of numpy arrays, row_ptr with
    `rows` or rows+1 entries; keys: dict of affine numpy arrays."""
    keep = []
    g = _OrcG16()
    for name, (val, col, rp) in zip("ABC", mats):
        val, col, rp = _u64(val), _u64(col), _u64(rp)
        keep += [val, col, rp]
        setattr(g, name, _OrcCsr(_p(val), _p(col), _p(rp), rows, val.size // 4))
    g.n_vars, g.n_public, g.log_m = n_vars, n_public, log_m
    for k in ("a_query", "b1_query", "b2_query", "l_query", "h_query", "alpha1", "beta1", "delta1", "beta2",
              "delta2"):
        arr = _u64(keys[k])
        keep.append(arr)
        setattr(g, k, _p(arr))
    return g, keep


def _oracle_groth16(self, mats, rows, n_vars, n_public, log_m, keys, z, r, s, mode):
    g, keep = _groth16_struct(mats, rows, n_vars, n_public, log_m, keys)
    z, r, s = _u64(z), _u64(r), _u64(s)
    pa = np.zeros((3, 4), np.uint64)
    pb = np.zeros((3, 2, 4), np.uint64)
    pc = np.zeros((3, 4), np.uint64)
    rc = self.lib.orc_groth16_prove(ctypes.byref(g), ctypes.c_int(mode), _p(z), _p(r), _p(s), _p(pa), _p(pb), _p(pc))
    assert rc == 0
    return pa, pb, pc


def _oracle_groth16_h(self, mats, rows, n_vars, n_public, log_m, z, mode):
    dummy = {k: np.zeros(8, np.uint64) for k in ("a_query", "b1_query", "b2_query", "l_query", "h_query", "alpha1",
                                                  "beta1", "delta1", "beta2", "delta2")}
    g, keep = _groth16_struct(mats, rows, n_vars, n_public, log_m, dummy)
    h = np.zeros(((1 << log_m) - 1, 4), np.uint64)
    assert self.lib.orc_groth16_h(ctypes.byref(g), ctypes.c_int(mode), _p(_u64(z)), _p(h)) == 0
    return h


def _oracle_assemble(self, alpha1, beta1, delta1, beta2, delta2, g1res, g2res, r, s):
    og1 = np.zeros((2, 3, 4), np.uint64)
    og2 = np.zeros((3, 2, 4), np.uint64)
    args = [_u64(x) for x in (alpha1, beta1, delta1, beta2, delta2, g1res, g2res, r, s)]
    self.lib.orc_groth16_assemble(*[_p(a) for a in args], _p(og1), _p(og2))
    return og1, og2


Oracle.groth16_prove = _oracle_groth16
Oracle.groth16_h = _oracle_groth16_h
Oracle.groth16_assemble = _oracle_assemble
