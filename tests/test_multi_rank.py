"""The N > 1 host path with two `gloo` ranks on CPU: disjoint per-rank s
values, max over ranks of the timed region, the sharded deep scan gathering
every result line in input order (the scan itself is a stand-in here; the
GPU scan is covered by the GPU tests), and the degree-sharded sieve whose
ranks merge best[] by an all-reduce minimum (the oracle's sieve stands in
for the device sieve)."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from mersenne_trinomial_b200 import multi


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _fake_scan(r, s_values, k0, maxd, **kw):
    return [f"{s} {k0 + (s % 7) + 1} p{(s * 2654435761) % (1 << 40):x}" for s in s_values]


SIEVE_R, SIEVE_D = 44687, 20


def _oracle_sieve_degrees(r, degrees, smax):
    from oracle import oracle as O
    best = None
    for d in sorted(degrees):
        best = O.sieve(r, d, smax, dmin=d, best=best)
    return best


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        s = multi.rank_s_values(136279841, 16, rank)
        parts = [None] * world
        dist.all_gather_object(parts, s.tolist())
        t = multi.max_over_ranks(1.5 + rank, dist, device="cpu")
        surv = list(range(3, 40, 2))
        lines = multi.scan_sharded(4423, surv, 5, 200, rank, world, dist, scan_fn=_fake_scan)
        best = multi.sieve_sharded(SIEVE_R, 2, SIEVE_D, SIEVE_R // 2, rank, world, dist,
                                   sieve_fn=_oracle_sieve_degrees)
        out[rank] = {"s_sets": parts, "tmax": t, "lines": lines, "best": best.tobytes(),
                     "degrees": multi.sieve_degrees(2, SIEVE_D, rank, world)}
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_two_gloo_ranks():
    world = 2
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_worker, args=(world, _free_port(), out), nprocs=world,
                           start_method="spawn", join=True)
        res = dict(out)
    assert set(res) == {0, 1}
    a, b = res[0]["s_sets"]
    assert len(a) == len(b) == 16 and not set(a) & set(b)      # disjoint per-rank s values
    assert res[0]["tmax"] == res[1]["tmax"] == 2.5             # max over ranks
    want = _fake_scan(4423, list(range(3, 40, 2)), 5, 200)
    assert res[0]["lines"] == res[1]["lines"] == want          # every s once, input order
    # degree-sharded sieve: disjoint degrees, merged keys equal one sieve of all
    d0, d1 = res[0]["degrees"], res[1]["degrees"]
    assert sorted(d0 + d1) == list(range(2, SIEVE_D + 1)) and not set(d0) & set(d1)
    from oracle import oracle as O
    direct = O.sieve(SIEVE_R, SIEVE_D, SIEVE_R // 2).tobytes()
    assert res[0]["best"] == res[1]["best"] == direct


def test_shard_covers_each_item_once():
    items = list(range(23))
    for world in (1, 2, 3, 8):
        got = sorted(x for rk in range(world) for x in multi.shard(items, rk, world))
        assert got == items
    with pytest.raises(ValueError):
        multi.shard(items, 2, 2)


def test_sieve_degree_split_balances_cost():
    for world in (1, 2, 3, 8):
        parts = [multi.sieve_degrees(2, 31, rk, world) for rk in range(world)]
        assert sorted(d for p in parts for d in p) == list(range(2, 32))
        loads = [sum(1 << d for d in p) for p in parts]
        assert max(loads) - min(loads) <= 1 << 31       # at most one top degree apart
    with pytest.raises(ValueError):
        multi.sieve_degrees(2, 31, 3, 3)


def test_single_process_paths():
    assert multi.max_over_ranks(3.0) == 3.0
    lines = multi.scan_sharded(4423, [3, 5, 7], 5, 200, 0, 1, scan_fn=_fake_scan)
    assert lines == _fake_scan(4423, [3, 5, 7], 5, 200)
