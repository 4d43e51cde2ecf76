"""Host side of the batched workload: the seeded generator (pinned by a committed digest), the
heat map, the greedy shard and the gather of results on rank 0 (world size 2, gloo)."""
import json
import os
import sys

import numpy as np

from h2_b200 import batch as B

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

from make_batch_spec import digest  # noqa: E402


def test_generator_matches_digest():
    want = json.load(open(os.path.join(HERE, "golden", "batch64_digest.json")))
    got = digest(B.draw_batch(64, 1000))
    assert got == want


def test_draws_follow_the_spec():
    ms = B.draw_batch(64, 1000)
    assert {m.nx for m in ms} <= set(B.SIZES) and len({m.nx for m in ms}) == 3
    for m in ms:
        for d in range(3):
            assert 4 <= sum(1 for h in m.hotspots if h.die == d) <= 16
        for h in m.hotspots:
            assert B.FOOTPRINT[0] <= h.x0 < h.x1 <= B.FOOTPRINT[1]
            assert B.FOOTPRINT[0] <= h.y0 < h.y1 <= B.FOOTPRINT[1]
            assert h.x1 - h.x0 <= 0.25e-3 + 1e-18 and h.q > 0
    qs = np.log([h.q for m in ms for h in m.hotspots])
    assert abs(np.median(qs) - np.log(1e8)) < 0.15 and abs(qs.std() - 1.0) < 0.1
    assert B.from_json(B.to_json(ms[:3])) == ms[:3]


def test_heat_map(oracle):
    m = B.draw_member(5, 1000, sizes=(24,))
    NX = m.nx
    Z, ZC, dZ = oracle.genz(B.NZ)
    ID = oracle.fill_id(NX, NX, B.NZ)
    dx = oracle.pitch(NX)
    hs = B.heat_map(m, ID, ZC, dx, dx)
    assert hs.flags.f_contiguous and hs.shape == ID.shape
    sil = np.isin(ID, B.SILICON_IDS)
    assert (hs[~sil] == 0).all()
    assert (hs[sil] > 0).all()
    assert hs[0].max() == hs[-1].max() == hs[:, 0].max() == hs[:, :, 0].max() == 0
    # a cell covered by no hotspot has the background; a covered one the sum of densities
    xc = (np.arange(NX + 2) - 0.5) * dx
    for (i, j, k) in zip(*np.nonzero(sil)):
        die = [d for d, (z0, z1) in enumerate(B.DIE_Z) if z0 <= ZC[k] <= z1]
        assert len(die) == 1
        q = sum(h.q for h in m.hotspots if h.die == die[0] and h.x0 <= xc[i] < h.x1 and h.y0 <= xc[j] < h.y1)
        assert hs[i, j, k] == (q if q > 0 else B.BACKGROUND)


def test_shard_balance():
    ms = B.draw_batch(64, 1000)
    for world in (1, 2, 4, 8):
        parts = B.shard(ms, world)
        assert sorted(i for p in parts for i in p) == list(range(64))
        loads = [sum(ms[i].cells for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(m.cells for m in ms)
    assert B.shard(ms, 1) == [list(range(64))]


def _rank_main(rank, world, port, q):
    import torch.distributed as td
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    td.init_process_group("gloo", rank=rank, world_size=world)
    ms = B.draw_batch(10, 1000, sizes=(12, 16))
    mine = B.shard(ms, world)[rank]
    local = {i: {"rank": rank, "cells": ms[i].cells} for i in mine}
    merged = B.gather_results(local)
    q.put((rank, merged))
    td.destroy_process_group()


def test_shard_and_gather_two_ranks():
    import multiprocessing as mp
    import socket
    ctx = mp.get_context("spawn")
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    q = ctx.Queue()
    ps = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    got = dict(q.get(timeout=120) for _ in range(2))
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got[1] is None
    merged = got[0]
    ms = B.draw_batch(10, 1000, sizes=(12, 16))
    assert sorted(merged) == list(range(10))
    parts = B.shard(ms, 2)
    for r in range(2):
        assert all(merged[i]["rank"] == r for i in parts[r])
