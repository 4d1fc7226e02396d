"""Device side of the range-sharded MSM (liblightzk_b200/shard.py): the sum
of the gathered partial points (an MSM with unit scalars over their affine
forms) against the oracle, including a partial at infinity, and the whole
path on one rank over NCCL against the plain MSM."""
import socket

import numpy as np
import pytest

from helpers import same_point
from oracle import FR, G_ADD

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("group", [1, 2])
def test_sum_of_partials(cuda, orc, rng_state, group):
    from liblightzk_b200 import device, msm, shard
    parts = []
    for n in (5, 9, 0, 13):      # n = 0: a partial at infinity
        s = orc.rand_field(FR, max(n, 1), rng_state)[:n]
        b = orc.fixed_base(group, orc.rand_field(FR, max(n, 1), rng_state))[:n]
        parts.append(device.to_host(msm.msm(group, device.to_device(s), device.to_device(b))) if n else None)
    inf = device.to_host(msm.msm(group, device.to_device(np.zeros((0, 4), np.uint64)),
                                 device.to_device(np.zeros((0, 2, 4) if group == 1 else (0, 2, 2, 4), np.uint64))))
    parts = [p if p is not None else inf for p in parts]
    got = device.to_host(shard._gpu_sum(group, device.to_device(np.stack(parts))))
    op = orc.g1_op if group == 1 else orc.g2_op
    acc = parts[0]
    for q in parts[1:]:
        acc = op(G_ADD, acc, q)
    assert same_point(orc, group, got, acc)


def test_sharded_msm_one_rank_nccl(cuda, orc, rng_state):
    import torch.distributed as dist

    from liblightzk_b200 import device, msm, shard
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1)
    try:
        n = 3000
        s = device.to_device(orc.rand_field(FR, n, rng_state))
        b = device.to_device(orc.fixed_base(1, orc.rand_field(FR, n, rng_state)))
        got = device.to_host(shard.sharded_msm(1, s, b, window_bits=10))
        want = device.to_host(msm.msm(1, s, b))
        assert same_point(orc, 1, got, want)
    finally:
        dist.destroy_process_group()
