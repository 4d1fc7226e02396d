"""Synthetic Groth16 instances: R1CS, satisfying witness and proving key.

The workload of the benchmark: M = 2^log_m multiplication gates
w_i = x_a * x_b, with a and b uniform over variables defined before the
gate's block; rows of A and B are unit vectors (x_a, x_b) plus 0-2 extra
random (column, Fr) terms, and row i of C is the unit vector of w_i plus 0-2
extra terms, with w_i solved so that every constraint holds.  Variables:
z_0 = 1, n_public public inputs, n_free free witnesses (uniform Fr), then
the M gate outputs.  The structure (indices) comes from numpy's seeded PCG64;
every field value comes from lzk_random_fr (seeded, on the device); the
witness is solved on the device block by block (lzk_r1cs_solve).

The proving key follows the reference's Setup (groth16.cuh:88-126): every
key element is an independent seeded Fr multiple of the generator, here
computed with the fixed-base kernels (lzk_g1/g2_fixed_base).  Its shape is
the reference's: a, b1, b2 over all n_vars variables, the L query over the
n_vars - n_public - 1 private ones, M - 1 H-query points.
"""
import numpy as np
import torch

from . import _capi
from .device import ptr, stream_ptr
from .ntt import csr as make_csr

FR_ONE = np.array([0xAC96341C4FFFFFFB, 0x36FC76959F60CD29, 0x666EA36F7879462E, 0x0E0A77C19A07DF2F], np.uint64)

# lzk_random_fr stream ids
SID_A, SID_B, SID_C, SID_WIT, SID_KEY = 1, 2, 3, 4, 16


def random_fr(n, seed, sid, offset=0, device="cuda", stream=None):
    out = torch.empty((n, 4), dtype=torch.int64, device=device)
    _capi.call("lzk_random_fr", seed, sid, offset, n, ptr(out), stream_ptr(stream))
    return out


def fixed_base(group, k, stream=None):
    n = k.shape[0]
    shape = (n, 2, 4) if group == 1 else (n, 2, 2, 4)
    out = torch.empty(shape, dtype=torch.int64, device=k.device)
    _capi.call("lzk_g1_fixed_base" if group == 1 else "lzk_g2_fixed_base", ptr(k), n, ptr(out), stream_ptr(stream))
    return out


class Matrix:
    """CSR matrix in device memory: 4- or 8-byte indices (from col's dtype);
    row_ptr with rows + 1 offsets, or the reference's rows offsets with the
    last row ending at nnz."""

    def __init__(self, val, col, row_ptr, rows, cols):
        self.val, self.col, self.row_ptr = val, col, row_ptr
        self.rows, self.cols = rows, cols
        self.nnz = int(val.shape[0])

    def desc(self):
        return make_csr(self.val, self.col, self.row_ptr, self.rows, self.cols, self.nnz)

    def host(self):
        """(val, col, row_ptr) as numpy uint64 arrays (row_ptr with rows+1 entries)"""
        from .device import to_host
        rp = to_host(self.row_ptr).astype(np.uint64)
        if rp.shape[0] == self.rows:       # the reference's layout: the last row ends at nnz
            rp = np.append(rp, np.uint64(self.nnz))
        return (to_host(self.val), to_host(self.col).astype(np.uint64), rp)


def _rows(rng, unit, avail, maxextra):
    m = unit.shape[0]
    k = rng.integers(0, maxextra + 1, m)
    per = 1 + k
    row_ptr = np.zeros(m + 1, np.int64)
    np.cumsum(per, out=row_ptr[1:])
    nnz = int(row_ptr[-1])
    rep = np.repeat(np.arange(m), per)
    pos = np.arange(nnz) - row_ptr[rep]
    extra = (rng.random(nnz) * avail[rep]).astype(np.int64)
    col = np.where(pos == 0, unit[rep], extra)
    return col, row_ptr, pos == 0


class Circuit:
    """A synthetic instance resident on the device."""

    def __init__(self, log_m, seed=1, n_public=1, n_free=4096, block=4096, max_extra=2, device="cuda"):
        self.log_m = log_m
        self.M = M = 1 << log_m
        self.seed = seed
        self.n_public = n_public
        self.n_free = n_free
        self.block = block
        first_def = 1 + n_public + n_free
        self.n_vars = first_def + M
        rng = np.random.default_rng(seed)
        i = np.arange(M)
        avail = first_def + (i // block) * block
        a_unit = (rng.random(M) * avail).astype(np.int64)
        b_unit = (rng.random(M) * avail).astype(np.int64)
        c_unit = first_def + i
        self.mats = []
        for sid, unit in ((SID_A, a_unit), (SID_B, b_unit), (SID_C, c_unit)):
            col, row_ptr, is_unit = _rows(rng, unit, avail, max_extra)
            val = random_fr(col.shape[0], seed, sid, device=device)
            unit_idx = torch.from_numpy(np.nonzero(is_unit)[0]).to(device)
            val[unit_idx] = torch.from_numpy(FR_ONE.view(np.int64)).to(device)
            self.mats.append(Matrix(val, torch.from_numpy(col.astype(np.int32)).to(device),
                                    torch.from_numpy(row_ptr.astype(np.int32)).to(device), M, self.n_vars))
        self.A, self.B, self.C = self.mats
        self.device = device

    def witness(self, wseed):
        """satisfying witness for a fresh seed: z_0 = 1, public and free
        inputs uniform, gate outputs solved block by block"""
        first_def = 1 + self.n_public + self.n_free
        z = torch.empty((self.n_vars, 4), dtype=torch.int64, device=self.device)
        z[0] = torch.from_numpy(FR_ONE.view(np.int64)).to(self.device)
        z[1:first_def] = random_fr(first_def - 1, wseed, SID_WIT, device=self.device)
        a, b, c = (m.desc() for m in self.mats)
        import ctypes
        s = stream_ptr(None)
        for r0 in range(0, self.M, self.block):
            _capi.call("lzk_r1cs_solve", ctypes.byref(a), ctypes.byref(b), ctypes.byref(c), ptr(z), r0,
                       min(r0 + self.block, self.M), s)
        return z

    def unsatisfied_rows(self, z):
        import ctypes
        bad = torch.zeros(1, dtype=torch.int64, device=self.device)
        a, b, c = (m.desc() for m in self.mats)
        _capi.call("lzk_r1cs_check", ctypes.byref(a), ctypes.byref(b), ctypes.byref(c), ptr(z), ptr(bad),
                   stream_ptr(None))
        return int(bad.item())


class ProvingKey:
    """Seeded proving key in device memory (affine points)."""

    def __init__(self, circuit, seed=7):
        n, M, nl = circuit.n_vars, circuit.M, circuit.n_vars - circuit.n_public - 1
        dev = circuit.device
        sid = SID_KEY
        self.a = fixed_base(1, random_fr(n, seed, sid + 0, device=dev))
        self.b1 = fixed_base(1, random_fr(n, seed, sid + 1, device=dev))
        self.b2 = fixed_base(2, random_fr(n, seed, sid + 2, device=dev))
        self.l = fixed_base(1, random_fr(max(nl, 1), seed, sid + 3, device=dev))[:nl]
        self.h = fixed_base(1, random_fr(M - 1, seed, sid + 4, device=dev))
        g1 = fixed_base(1, random_fr(3, seed, sid + 5, device=dev))
        g2 = fixed_base(2, random_fr(2, seed, sid + 6, device=dev))
        self.alpha1, self.beta1, self.delta1 = g1[0], g1[1], g1[2]
        self.beta2, self.delta2 = g2[0], g2[1]


def _next_pow2(x):
    return 1 << max(0, int(x - 1).bit_length())


class MatMulCircuit:
    """The reference's benchmark circuit: the product Z = X Y of two p x p
    matrices (xpu-spmat.cuh:33-65, Groth16 input scales MatMul_p_39 / 63 /
    100 of groth16.cuh:11-46, i.e. 2^16, 2^18 and 2^20 constraints).

    Variables: z_0 = 1, X (p^2), Y (p^2), Z (p^2), then the p^3 products
    t_(i1 p^2 + i2 p + i3); the k = 3p^2 entries of X, Y and Z are the public
    inputs.  Rows 0 .. p^3 - 1 are the products (A selects X, B selects Y,
    C selects t), rows p^3 .. p^3 + p^2 - 1 the sums (A adds p products, B
    is the constant 1, C selects Z), the remaining rows up to
    M = next_pow2(p^3 + p^2) are empty; every coefficient is one.  The
    matrices are built with the reference's layout: 8-byte column indices and
    row offsets, `rows` = M offsets with the last row ending at nnz.  Unlike
    the reference's random witness (groth16.cuh:128-132), witness() solves the
    gates, so the instance is satisfied."""

    def __init__(self, p, device="cuda"):
        self.p = p
        p2, p3 = p * p, p * p * p
        self.M = M = _next_pow2(p3 + p2)
        self.log_m = M.bit_length() - 1
        self.n_public = 3 * p2
        self.n_vars = 1 + 3 * p2 + p3
        self.device = device
        i = np.arange(p3, dtype=np.int64)
        i1, i2, i3 = i // p2, (i % p2) // p, i % p
        r = np.arange(p2, dtype=np.int64)
        a_col = np.concatenate([1 + i2 * p + i1, (1 + 3 * p2 + np.arange(p)[None, :] * p2 + r[:, None]).reshape(-1)])
        a_ptr = np.concatenate([np.arange(p3), p3 + p * r, np.full(M - p3 - p2, 2 * p3)])
        b_col = np.concatenate([1 + p2 + i1 * p + i3, np.zeros(p2, np.int64)])
        c_col = np.concatenate([1 + 3 * p2 + i, 1 + 2 * p2 + r])
        bc_ptr = np.concatenate([np.arange(p3 + p2), np.full(M - p3 - p2, p3 + p2)])
        one = torch.from_numpy(FR_ONE.view(np.int64)).to(device)
        self.mats = []
        for col, rp in ((a_col, a_ptr), (b_col, bc_ptr), (c_col, bc_ptr)):
            val = one.repeat(col.shape[0], 1)
            self.mats.append(Matrix(val, torch.from_numpy(col).to(device), torch.from_numpy(rp.astype(np.int64)).to(device),
                                    M, self.n_vars))
        self.A, self.B, self.C = self.mats

    def witness(self, wseed):
        """z_0 = 1, X and Y uniform (seeded), then the products and the sums
        solved on the device (lzk_r1cs_solve)"""
        import ctypes
        p2, p3 = self.p * self.p, self.p ** 3
        z = torch.zeros((self.n_vars, 4), dtype=torch.int64, device=self.device)
        z[0] = torch.from_numpy(FR_ONE.view(np.int64)).to(self.device)
        z[1:1 + 2 * p2] = random_fr(2 * p2, wseed, SID_WIT, device=self.device)
        a, b, c = (m.desc() for m in self.mats)
        s = stream_ptr(None)
        for r0, r1 in ((0, p3), (p3, p3 + p2)):
            _capi.call("lzk_r1cs_solve", ctypes.byref(a), ctypes.byref(b), ctypes.byref(c), ptr(z), r0, r1, s)
        return z

    unsatisfied_rows = Circuit.unsatisfied_rows

