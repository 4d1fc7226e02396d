"""The multi-GPU MSM path (liblightzk_b200/shard.py) with 2 and 3 ranks over
gloo on the CPU: the range split, the all-gather of the partial points and
the final sum, with the per-rank device operations replaced by the oracle,
against the oracle's MSM over all points.  Covers ranges that do not divide
evenly, ranks with empty ranges, G2, and ranks that hold only their own range
of bases."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _oracle_ops():
    from oracle import G_ADD, Oracle
    orc = Oracle()

    def local_msm(group, s, b, window_bits):
        s, b = s.numpy().view(np.uint64), b.numpy().view(np.uint64)
        shape = (3, 4) if group == 1 else (3, 2, 4)
        r = orc.msm(group, s, b) if s.shape[0] else _inf(orc, group, shape)
        return torch.from_numpy(np.ascontiguousarray(r).view(np.int64))

    def local_sum(group, parts):
        p = parts.numpy().view(np.uint64)
        op = orc.g1_op if group == 1 else orc.g2_op
        acc = p[0]
        for q in p[1:]:
            acc = op(G_ADD, acc, q)
        return torch.from_numpy(np.ascontiguousarray(acc).view(np.int64))
    return orc, local_msm, local_sum


def _inf(orc, group, shape):
    from oracle import FQ
    r = np.zeros(shape, np.uint64)
    one = orc.to_mont(FQ, np.array([[1, 0, 0, 0]], np.uint64))[0]
    r[1] = one if group == 1 else np.stack([one, np.zeros(4, np.uint64)])
    return r


def _worker(rank, world, port, cases, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import FR
        from liblightzk_b200 import shard
        orc, local_msm, local_sum = _oracle_ops()
        out = []
        for group, n, seed, own_range in cases:
            st = np.array([seed], np.uint64)
            s = orc.rand_field(FR, n, st)
            b = orc.fixed_base(group, orc.rand_field(FR, n, st))
            if own_range:
                lo, hi = shard.shard_range(n, rank, world)
                b = b[lo:hi]
            t = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.int64))  # noqa: E731
            r = shard.sharded_msm(group, t(s), t(b), local_msm=local_msm, local_sum=local_sum)
            out.append(r.numpy().view(np.uint64).copy())
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_msm_gloo(world, orc):
    from oracle import FR
    cases = [(1, 101, 3, False), (1, 2, 4, False), (2, 17, 5, False), (1, 64, 6, True)]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, cases, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = dict(q.get(timeout=300) for _ in range(world))
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    for k, (group, n, seed, _) in enumerate(cases):
        st = np.array([seed], np.uint64)
        s = orc.rand_field(FR, n, st)
        b = orc.fixed_base(group, orc.rand_field(FR, n, st))
        expect = orc.jac_to_aff(group, orc.msm(group, s, b)[None])
        for r in range(world):
            assert (orc.jac_to_aff(group, results[r][k][None]) == expect).all(), (world, k, r)


def test_shard_ranges_cover_exactly():
    from liblightzk_b200.shard import shard_range
    for n in (0, 1, 2, 7, 100, 1 << 20):
        for world in (1, 2, 3, 8):
            rs = [shard_range(n, r, world) for r in range(world)]
            assert rs[0][0] == 0 and rs[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(rs, rs[1:]))
            assert max(h - lo for lo, h in rs) - min(h - lo for lo, h in rs) <= 1
