"""The N > 1 path of the benchmark without a GPU: two `gloo` ranks on 127.0.0.1 take the benchmark's own steps.

The path shards by whole solves (replicas, no collective on the data path): every rank draws the same seeded
stream, keeps its share, and after the timed steps the ranks agree on the max of their seconds and the sum of their
unconverged solves. These tests run those functions of `bench.py` on two processes."""
import datetime
import importlib.util
import os
import socket

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, secs, nfail, out):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        bench = _bench()
        reqs, _ = bench.stream(2026, 24, lambda r: True)
        share = [r["k"] for r in bench.rank_share(reqs, rank, world)]
        dist.barrier()
        t, f = bench.over_ranks(secs[rank], nfail[rank], dist, "cpu")
        out.put((rank, t, f, share))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_the_ranks_share_the_stream_and_agree_on_the_timing(world):
    secs = [1.25, 3.5, 2.0][:world]
    nfail = [1, 0, 4][:world]
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, secs, nfail, out)) for r in range(world)]
    for p in procs:
        p.start()
    got = {}
    try:
        for _ in range(world):
            rank, t, f, share = out.get(timeout=120)
            got[rank] = (t, f, share)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs)
    for rank in range(world):
        t, f, _ = got[rank]
        assert t == max(secs) and f == sum(nfail)
    shares = [set(got[r][2]) for r in range(world)]
    assert set().union(*shares) == set(range(24)) and sum(map(len, shares)) == 24
    assert max(map(len, shares)) - min(map(len, shares)) <= 1


def test_every_rank_draws_the_same_stream():
    bench = _bench()
    a, _ = bench.stream(7, 40, lambda r: r["d"] == 2)
    b, _ = bench.stream(7, 40, lambda r: r["d"] == 2)
    assert [r["k"] for r in a] == [r["k"] for r in b] and all(r["d"] == 2 for r in a)
    assert all((bench.positions(7, x) == bench.positions(7, y)).all() for x, y in zip(a[:3], b[:3]))
