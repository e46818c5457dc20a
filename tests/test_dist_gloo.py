"""Multi-rank host logic on CPU with the gloo backend (world size 2):
replica sharding covers every solve exactly once and the timing reductions
return the max / sum over ranks."""
from __future__ import annotations

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, size, port, q):
    os.environ.update(WORLD_SIZE=str(size), RANK=str(rank), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    from gpe_b200 import dist

    d = dist.init(backend="gloo", timeout_s=30)
    assert d is not None
    owned = dist.shard(range(11))
    mx = dist.max_over_ranks(1.5 + rank)
    sm = dist.sum_over_ranks(len(owned))
    dist.barrier()
    q.put((rank, owned, mx, sm))
    dist.finalize()


def test_gloo_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, o0, m0, s0), (r1, o1, m1, s1) = out
    assert sorted(o0 + o1) == list(range(11)) and not set(o0) & set(o1)
    assert m0 == m1 == 2.5
    assert s0 == s1 == 11


def test_single_process_defaults():
    from gpe_b200 import dist

    if "WORLD_SIZE" in os.environ and os.environ["WORLD_SIZE"] != "1":
        pytest.skip("running under a launcher")
    assert dist.init() is None
    assert dist.max_over_ranks(3.0) == 3.0
    assert dist.shard([1, 2, 3]) == [1, 2, 3]


def _slab_worker(rank, size, port, q):
    os.environ.update(WORLD_SIZE=str(size), RANK=str(rank), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    from gpe_b200 import dist

    dist.init(backend="gloo", timeout_s=30)
    r, n, nid, k0, nzl = dist.slab_plan(37)
    q.put((rank, r, n, nid, k0, nzl))
    dist.finalize()


def test_gloo_slab_plan_two_ranks():
    """z-slab set-up of one solve over 2 ranks: both ranks hold rank 0's
    NCCL id and their slabs tile the 37 planes in rank order."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_slab_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(60)
        assert p.exitcode == 0
    (_, r0, n0, id0, a0, b0), (_, r1, n1, id1, a1, b1) = res
    assert (r0, r1, n0, n1) == (0, 1, 2, 2)
    assert id0 == id1 and len(id0) == 128
    assert (a0, b0, a1, b1) == (0, 19, 19, 18)


def test_slab_partition_tiles_the_axis():
    from gpe_b200 import slab

    for nz in (6, 7, 64, 257):
        for n in range(1, 9):
            spans = [slab.partition(nz, n, r) for r in range(n)]
            assert spans[0][0] == 0
            assert all(a + b == c for (a, b), (c, _) in zip(spans, spans[1:]))
            assert spans[-1][0] + spans[-1][1] == nz
            sizes = [b for _, b in spans]
            assert max(sizes) - min(sizes) <= 1 and sizes == sorted(sizes, reverse=True)
