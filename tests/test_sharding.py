"""The multi-rank path on CPU: two and three gloo ranks shard source positions
(5 of them: uneven shares) and gather Pi_mu_nu; the result must equal the
single-process run bit for bit.
The per-source computation here is the oracle's contraction on a small
lattice (the CUDA library is not needed to test the host orchestration)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from golden import inputs

DIMS, V = (4, 2, 2, 2), 32
SOURCES = [0, 3, 5, 17, 30]


def pi_for_source(src):
    import oracle_bind as ob
    o = ob.Oracle(*DIMS, 0.15, 0.03)
    o.set_gauge(inputs.gauge(9, V))
    fields = [inputs.field(1000 * (src + 1) + i, 24 * V) for i in range(120)]
    conn, _ = o.cvc_contract(fields, src)
    return conn


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, q):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, here)
    sys.path.insert(0, os.path.dirname(here))
    import torch.distributed as dist
    from cvc_b200 import sharding
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        res = sharding.run_sharded(SOURCES, pi_for_source)
        mine = sharding.my_items(range(len(SOURCES)), world, rank)
        local = [torch.from_numpy(pi_for_source(SOURCES[i])) for i in mine]
        stacked = sharding.gather_tensors(local, len(SOURCES))
        tmax = sharding.max_over_ranks(1.0 + rank)
        q.put((rank, {k: v for k, v in res.items()}, stacked.numpy(), tmax, mine))
    finally:
        dist.destroy_process_group()


def test_partition_covers_each_item_once():
    from cvc_b200 import sharding
    for world in (1, 2, 3, 8):
        seen = []
        for r in range(world):
            seen += sharding.my_items(range(13), world, r)
        assert sorted(seen) == list(range(13))


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_match_single_process(oracle_mod, world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=240) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    serial = {s: pi_for_source(s) for s in SOURCES}
    for rank, res, stacked, tmax, mine in out:
        assert tmax == float(world)
        assert set(res) == set(SOURCES)
        for s in SOURCES:
            assert np.array_equal(res[s], serial[s])
        for i, s in enumerate(SOURCES):
            assert np.array_equal(stacked[i], serial[s])
    assert sorted(sum((o[4] for o in out), [])) == list(range(len(SOURCES)))


# ---- the P -> gamma gamma driver's orchestration (cvc_b200.p2gg.run_sources):
# gauge made on rank 0 and broadcast, sources dealt round-robin, Pi gathered.
# The per-source work is the oracle's contraction (the GPU solve and
# contraction are replaced, the orchestration code is the product's).
P2_SOURCES = [1, 4, 9, 22, 31]


def _make_gauge():
    return inputs.gauge(11, V)


def _compute(gauge, src):
    import oracle_bind as ob
    o = ob.Oracle(*DIMS, 0.15, 0.03)
    o.set_gauge(gauge)
    fields = [inputs.field(7000 + 131 * src + i, 24 * V) for i in range(120)]
    conn, contact = o.cvc_contract(fields, src)
    return torch.from_numpy(conn), torch.from_numpy(contact)


def _p2gg_rank_main(rank, world, port, q):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, here)
    sys.path.insert(0, os.path.dirname(here))
    import torch.distributed as dist
    from cvc_b200 import p2gg
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    made = []

    def make():
        made.append(rank)
        return _make_gauge()

    try:
        conn, contact = p2gg.run_sources(P2_SOURCES, make, _compute, 72 * V)
        q.put((rank, conn.numpy(), contact.numpy(), made))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_p2gg_driver_sharded_matches_single_process(oracle_mod, world):
    from cvc_b200 import p2gg
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_p2gg_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=240) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    conn1, contact1 = p2gg.run_sources(P2_SOURCES, _make_gauge, _compute, 72 * V)
    for rank, conn, contact, made in out:
        assert made == ([0] if rank == 0 else [])  # the gauge is made once, on rank 0
        assert np.array_equal(conn, conn1.numpy())
        assert np.array_equal(contact, contact1.numpy())
