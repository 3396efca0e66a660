"""Serving front end: a Poisson stream of (r, s-set, d-range) search jobs fed
to the engine's continuous-batching server (gf2e_server_*, csrc/server.cu).

    python -m mersenne_trinomial_b200.serve [--seconds 20] [--rate 2.0] [--seed 1]

Prints one JSON line: job p50/p99 latency, aggregate sieved and scanned
(s, d) pairs per second, and the same jobs run one at a time (plain path)
for comparison.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import sys
import time

import numpy as np

from ._lib import call, lib
from .engine import _sp
from . import workloads as W


class Server:
    """Owner of one gf2e_server (device memory budget, scanner slots per r)."""

    def __init__(self, budget_bytes: int = 64 << 30, slots_per_r: int = 64, block: int = 1):
        h = C.c_void_p()
        call("gf2e_server_create_blocked", budget_bytes, slots_per_r, block, C.byref(h))
        self.h = h.value

    def submit(self, job_id: int, r: int, s_values, dmax: int, L0: int = 64, Lmax: int = 4096):
        s = np.ascontiguousarray(np.asarray(s_values, dtype=np.uint64))
        call("gf2e_server_submit", self.h, job_id, r, s.ctypes.data, s.size, dmax, L0, Lmax)

    def step(self, degrees: int = 16, stream=None):
        call("gf2e_server_step", self.h, degrees, _sp(stream))

    def status(self):
        w, a, f = C.c_int(), C.c_int(), C.c_int()
        used = C.c_size_t()
        call("gf2e_server_status", self.h, C.byref(w), C.byref(a), C.byref(f), C.byref(used))
        return {"waiting": w.value, "active": a.value, "finished": f.value, "used": used.value}

    def pairs(self):
        """(sieved, scanned) (s, d) pairs actually worked through so far."""
        a, b = C.c_uint64(), C.c_uint64()
        call("gf2e_server_pairs", self.h, C.byref(a), C.byref(b))
        return a.value, b.value

    def poll(self, cap: int = 1024):
        ids = np.zeros(cap, dtype=np.uint64)
        lat = np.zeros(cap, dtype=np.float64)
        n = C.c_int()
        call("gf2e_server_poll", self.h, ids.ctypes.data, lat.ctypes.data, cap, C.byref(n))
        return list(zip(ids[: n.value].tolist(), lat[: n.value].tolist()))

    def lines(self, job_id: int) -> list:
        need = C.c_size_t()
        call("gf2e_server_job_lines", self.h, job_id, None, 0, C.byref(need))
        buf = C.create_string_buffer(need.value)
        call("gf2e_server_job_lines", self.h, job_id, buf, need.value, C.byref(need))
        return buf.value.decode().splitlines()

    def release(self, job_id: int):
        call("gf2e_server_release", self.h, job_id)

    def close(self):
        if self.h:
            lib().gf2e_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


R_CLASSES = {"1e5": 100_000, "1e6": 1_000_000, "1e7": 10_000_000}
BAD_R = {127, 151, 241, 257, 337, 8191, 131071, 178481, 524287}


# largest s-set of a deep (squaring + gcd) job per r class: every deep s costs
# at least one interval gcd of r-bit operands (about 0.1 s at r ~ 1e6, 1 s at
# r ~ 1e7 and 4 s at r = 136279841 with 8-16 of them running at once)
DEEP_S_CAP = {"1e5": 256, "1e6": 256, "1e7": 32, "deep": 4}


def job_stream(seed: int, n_jobs: int, rate: float, deep_max: int = 2000,
               s_lo: int = 16, s_hi: int = 4096, deep_frac: float = 0.6,
               deep_s_cap=None, deep_classes=("1e5", "1e6", "1e7", "deep")):
    """Seeded Poisson arrivals.  r from the set {~1e5, ~1e6, ~1e7, 136279841}
    (one seeded prime = +-1 mod 8 that the sieve supports near each of the
    first three); s-sets of s_lo..s_hi values (log-uniform); d-range 2..24
    (sieve only) or, for a fraction deep_frac of the jobs of every r, up to
    2..deep_max (squaring + gcd), their s-sets capped per r class
    (DEEP_S_CAP); deep_classes limits which r classes get deep jobs.  Jobs
    with the same r share that r's resident scanner."""
    caps = dict(DEEP_S_CAP, **(deep_s_cap or {}))
    rng = np.random.default_rng(seed)
    rset = {}
    for name, near in R_CLASSES.items():
        cands = [p for p in W.primes_pm1_mod8(near - 3000, near + 3000)
                 if p not in BAD_R and W.sieve_compatible(p, 24)]
        rset[name] = int(cands[int(rng.integers(len(cands)))])
    t = 0.0
    jobs = []
    for i in range(n_jobs):
        t += rng.exponential(1.0 / rate)
        cls = str(rng.choice(["1e5", "1e6", "1e7", "deep"]))
        r = W.R_DEEP if cls == "deep" else rset[cls]
        deep = rng.random() < deep_frac and cls in deep_classes
        hi = min(s_hi, caps[cls]) if deep else s_hi
        lo = min(s_lo, hi)
        ns = int(round(np.exp(rng.uniform(np.log(lo), np.log(hi)))))
        s = np.unique(rng.integers(3, r // 2, size=ns)).astype(np.uint64)
        dmax = int(rng.integers(25, deep_max + 1)) if deep else int(rng.integers(2, 25))
        jobs.append({"id": i + 1, "t": t, "r": r, "s": s, "dmax": dmax})
    return jobs


def run_stream(jobs, slots: int = 64, budget: int = 64 << 30, degrees: int = 16,
               realtime: bool = True, block: int = 1):
    """Serve `jobs` (arrival times in seconds); returns (latencies, wall,
    lines, pairs) with pairs the (sieved, scanned) (s, d) pairs worked."""
    srv = Server(budget, slots, block)
    t0 = time.perf_counter()
    pending = sorted(jobs, key=lambda j: j["t"])
    i = 0
    lat = {}
    lines = {}
    while len(lat) < len(jobs):
        now = time.perf_counter() - t0
        while i < len(pending) and (not realtime or pending[i]["t"] <= now):
            j = pending[i]
            srv.submit(j["id"], j["r"], j["s"], j["dmax"])
            i += 1
        srv.step(degrees)
        for jid, _ in srv.poll():
            j = next(x for x in jobs if x["id"] == jid)
            lat[jid] = time.perf_counter() - t0 - j["t"]
            lines[jid] = srv.lines(jid)
            srv.release(jid)
        if realtime and i < len(pending) and not srv.status()["active"] and \
                not srv.status()["waiting"]:
            time.sleep(max(0.0, min(0.01, pending[i]["t"] - (time.perf_counter() - t0))))
    wall = time.perf_counter() - t0
    pairs = srv.pairs()
    srv.close()
    return lat, wall, lines, pairs


def run_one_at_a_time(jobs, slots: int = 64, degrees: int = 16, block: int = 1,
                      budget: int = 64 << 30):
    """The plain path: the jobs one after another on one server (each alone
    on the GPU, nothing overlapping), same step size as the stream; returns
    (wall, lines, pairs)."""
    srv = Server(budget, slots, block)
    t0 = time.perf_counter()
    lines = {}
    for j in jobs:
        srv.submit(j["id"], j["r"], j["s"], j["dmax"])
        done = []
        while not done:
            srv.step(degrees)
            done = srv.poll()
        lines[j["id"]] = srv.lines(j["id"])
        srv.release(j["id"])
    wall = time.perf_counter() - t0
    pairs = srv.pairs()
    srv.close()
    return wall, lines, pairs


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=24)
    ap.add_argument("--rate", type=float, default=4.0)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--deep-max", type=int, default=1000)
    ap.add_argument("--block", type=int, default=1, help="blocked-DDF degrees per step")
    a = ap.parse_args(argv)
    jobs = job_stream(a.seed, a.jobs, a.rate, a.deep_max)
    lat, wall, lines, pairs = run_stream(jobs, block=a.block)
    plain_wall, plain_lines, plain_pairs = run_one_at_a_time(jobs, block=a.block)
    v = sorted(lat.values())
    same = all(lines[k] == plain_lines[k] for k in lines)
    out = {"jobs": len(jobs), "p50_s": float(np.percentile(v, 50)),
           "p99_s": float(np.percentile(v, 99)), "wall_s": wall,
           "sd_pairs_per_s": sum(pairs) / wall, "sieved_scanned_pairs": pairs,
           "plain_wall_s": plain_wall, "plain_sd_pairs_per_s": sum(plain_pairs) / plain_wall,
           "results_identical": same}
    print(json.dumps(out))
    return 0 if same else 1


if __name__ == "__main__":
    sys.exit(main())
