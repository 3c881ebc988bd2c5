"""Multi-rank host logic on CPU (gloo, world size 2): stripes are sharded
across ranks with no data-path exchange, each rank codes its own shard, and
the union equals the single-process result.  The CPU oracle stands in for the
per-rank engine here; the GPU path uses the same partition."""
import datetime
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

from scrs_b200.shard import shard_by_bytes, shard_range


def test_shard_range_covers_once():
    for n in (0, 1, 7, 64, 1001):
        for world in (1, 2, 3, 8):
            seen = []
            for r in range(world):
                lo, hi = shard_range(n, r, world)
                seen += list(range(lo, hi))
                assert hi - lo in (n // world, n // world + 1)
            assert seen == list(range(n))


def test_shard_by_bytes_balanced():
    rng = np.random.default_rng(1)
    sizes = rng.choice([1024, 4096, 65536], 500).tolist()
    for world in (1, 2, 4, 8):
        parts = shard_by_bytes(sizes, world)
        assert parts[0][0] == 0 and parts[-1][1] == len(sizes)
        assert all(a[1] == b[0] for a, b in zip(parts, parts[1:]))
        per = [sum(sizes[lo:hi]) for lo, hi in parts]
        assert max(per) - min(per) <= 2 * max(sizes)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, specs, q):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import sys
        from pathlib import Path

        root = Path(__file__).resolve().parents[1]
        sys.path.insert(0, str(root))
        from scrs_b200.api import Api, Library
        from scrs_b200.shard import all_ranks_ok, max_over_ranks, shard_by_bytes

        oracle = Api(Library(root / "oracle" / "_build" / "liboracle.so", prefix="oracle_", device=False))
        lo, hi = shard_by_bytes([k * L for _, k, m, L, _ in specs], world)[rank]
        mine = {}
        for s in range(lo, hi):
            engine, k, m, L, seed = specs[s]
            p = oracle.resolve(engine, k, m, L)
            data = np.random.default_rng(seed).integers(0, 256, k * L, dtype=np.uint8)
            rep = np.zeros(m * L, np.uint8)
            oracle.batch_encoder(p).encode_into(data, rep)
            mine[s] = rep.tobytes()
        t = max_over_ranks(float(rank + 1))
        ok = all_ranks_ok(True)
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        q.put((rank, t, ok, gathered if rank == 0 else None))
    finally:
        dist.destroy_process_group()


def test_two_rank_sharded_encode_matches_single_process(oracle):
    from scrs_b200.api import Engine

    rng = np.random.default_rng(7)
    specs = [(Engine.GOOD_CAUCHY if i % 2 else Engine.STANDARD_CAUCHY, int(rng.integers(2, 20)),
              int(rng.integers(1, 6)), int(rng.choice([64, 256, 1000])), 1000 + i) for i in range(24)]
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, specs, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(world):
        rank, t, ok, gathered = q.get(timeout=120)
        res[rank] = (t, ok, gathered)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(res[r][0] == float(world) for r in res)  # max over ranks
    assert all(res[r][1] for r in res)
    merged = {}
    for part in res[0][2]:
        assert not (set(part) & set(merged))  # each stripe coded by exactly one rank
        merged.update(part)
    assert sorted(merged) == list(range(len(specs)))
    for s, (engine, k, m, L, seed) in enumerate(specs):
        p = oracle.resolve(engine, k, m, L)
        data = np.random.default_rng(seed).integers(0, 256, k * L, dtype=np.uint8)
        rep = np.zeros(m * L, np.uint8)
        oracle.batch_encoder(p).encode_into(data, rep)
        assert merged[s] == rep.tobytes()
