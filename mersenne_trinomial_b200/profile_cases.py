"""Small, self-contained launches of each hot kernel, sized for a profiler
capture (inputs larger than L2, a few GB at most, a handful of launches).

    python -m mersenne_trinomial_b200.profile_cases square [--r R] [--n N] [--k K]
    python -m mersenne_trinomial_b200.profile_cases fft [--m M]
    python -m mersenne_trinomial_b200.profile_cases sieve [--r R] [--depth D]
    python -m mersenne_trinomial_b200.profile_cases sieve_wide --depth D --dmin D --wide-from W
    python -m mersenne_trinomial_b200.profile_cases mul [--m M]
    python -m mersenne_trinomial_b200.profile_cases gcd|hgcd [--r R]
    python -m mersenne_trinomial_b200.profile_cases hgcd_many [--r R] [--n N]
    python -m mersenne_trinomial_b200.profile_cases scan [--r R --n N --k K]
    python -m mersenne_trinomial_b200.profile_cases scan_step [--r R --n N --block B]
    python -m mersenne_trinomial_b200.profile_cases config4 [--n 128 --maxd 20000 --block B
                                                             --l0 L0 --lmax LMAX --out PREFIX]
"""
from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np

import mersenne_trinomial_b200 as M
from mersenne_trinomial_b200 import workloads as W


def case_square(a):
    r, n, k = a.r, a.n, a.k
    nw = (r + 63) // 64
    stride = nw + (nw & 1)
    st = M.DeviceBuffer(8 * stride * n)
    sc = M.DeviceBuffer(st.nbytes)
    rng = np.random.default_rng(3)
    s = rng.integers(3, r // 2, size=n).astype(np.uint64)
    M.trin_set_x(st, stride, n, r)
    M.trin_square_batch(st, sc, stride, n, r, M.DeviceBuffer.from_array(s), k)
    M.stream_sync()


def case_fft(a):
    m = a.m
    F = M.CudaFFT()
    F.init(m)
    d = M.DeviceBuffer.from_array(W.splitmix64(5, 1 << m))
    F.fwd(d)
    F.inv(d)
    M.stream_sync()


def case_mul(a):
    bits = 1 << (a.m + 4)
    x = W.random_bits(bits, 1)
    y = W.random_bits(bits, 2)
    M.gf2x_fft_mul(x, bits, y, bits)


def case_gcd(a):
    """n gcds of an r-bit accumulator-like operand against x^r + x^s + 1."""
    r, n = a.r, a.n
    nw = (r + 1 + 63) // 64
    pairs, keep = [], []
    for i in range(n):
        T = np.zeros(nw, dtype=np.uint64)
        s = 1000 + 37 * i
        for e in (0, s, r):
            T[e >> 6] |= np.uint64(1 << (e & 63))
        A = W.random_bits(r, 50 + i)
        da, db = M.DeviceBuffer.from_array(A), M.DeviceBuffer.from_array(T)
        keep += [da, db]
        pairs.append((da, r, db, r + 1))
    t0 = time.perf_counter()
    degs, _ = M.gcd_batch(pairs)
    print(f"gcd: {n} x {r} bits in {time.perf_counter() - t0:.3f} s, degrees {degs[:4]}")


def case_scan(a):
    """A small deep scan: n seeded s at r, degrees k0 = 24 .. a.k."""
    rng = np.random.default_rng(9)
    s = rng.integers(3, a.r // 2, size=a.n).astype(np.uint64)
    t0 = time.perf_counter()
    lines = M.scan(a.r, s, 24, max(25, a.k), L0=64, Lmax=4096, batch=a.n)
    print(f"scan: {a.n} s x degrees 25..{a.k} at r={a.r} in {time.perf_counter() - t0:.3f} s:",
          lines[:3])


def case_scan_step(a):
    """The deep scan's per-degree work at r: n d <= 24 survivors on a
    scanner with the blocked DDF (block a.block; 1 = per degree), a ramp
    and one block, then 4 blocks of degrees; no interval end (no gcd)."""
    import ctypes as C
    from mersenne_trinomial_b200._lib import call
    smax = 200000
    best = M.run_sieve(a.r, 24, smax)
    surv = [s for s in range(3, smax + 1) if int(best[s]) == 0xFFFFFFFFFFFFFFFF][:a.n]
    h = C.c_void_p()
    call("gf2e_scanner_create_blocked", a.r, len(surv), a.block, C.byref(h))
    s_arr = np.asarray(surv, dtype=np.uint64)
    call("gf2e_scanner_submit", h.value, s_arr.ctypes.data, len(surv), 24, 24 + 1000000,
         1 << 30, 1 << 30, 0)
    call("gf2e_scanner_step", h.value, a.block, None)
    M.stream_sync()
    t0 = time.perf_counter()
    call("gf2e_scanner_step", h.value, 4 * a.block, None)
    M.stream_sync()
    dt = time.perf_counter() - t0
    M.lib().gf2e_scanner_destroy(h.value)
    print(f"scan_step: {len(surv)} s x {4 * a.block} degrees (block {a.block}) in {dt:.3f} s, "
          f"{dt * 1e3 / (4 * a.block * len(surv)):.3f} ms per (s, degree)")


def case_hgcd(a):
    """One half-gcd of a scan-like accumulator against x^r + x^s + 1."""
    r, s = a.r, 1001
    T = M.TrinGPU()
    T.init(r)
    T.set_s(s)
    T.set_x()
    T.reset_acc()
    for k in range(1, 40):
        T.square_A()
        if k > 24:
            T.accumulate()
    acc = T.read("ACC")
    T.fini()
    tri = np.zeros((r + 1 + 63) // 64, dtype=np.uint64)
    for e in (0, s, r):
        tri[e >> 6] |= np.uint64(1 << (e & 63))
    da, db = M.DeviceBuffer.from_array(acc), M.DeviceBuffer.from_array(tri)
    t0 = time.perf_counter()
    degs, _, st = M.gcd_large([(da, r, db, r + 1)])
    print(f"hgcd: {r} bits in {time.perf_counter() - t0:.3f} s, degree {degs[0]}, {st}")


def case_hgcd_many(a):
    """n half-gcds at once (one host thread and stream each): random r-bit
    operands against x^r + x^s + 1, s = 1000 + 7919 i; aggregate wall time."""
    r, n = a.r, a.n
    pairs, keep = [], []
    for i in range(n):
        s = 1000 + 7919 * i
        T = np.zeros((r + 1 + 63) // 64, dtype=np.uint64)
        for e in (0, s, r):
            T[e >> 6] |= np.uint64(1 << (e & 63))
        da = M.DeviceBuffer.from_array(W.random_bits(r, 100 + i))
        db = M.DeviceBuffer.from_array(T)
        keep += [da, db]
        pairs.append((da, r, db, r + 1))
    M.stream_sync()
    import resource
    import torch
    free0 = torch.cuda.mem_get_info()[0]
    ru0 = resource.getrusage(resource.RUSAGE_SELF)
    t0 = time.perf_counter()
    degs, _, _ = M.gcd_large(pairs, max_parallel=n)
    dt = time.perf_counter() - t0
    ru1 = resource.getrusage(resource.RUSAGE_SELF)
    cpu = (ru1.ru_utime - ru0.ru_utime) + (ru1.ru_stime - ru0.ru_stime)
    # the gcd memory pool keeps what it reserved: its high-water mark
    pool = free0 - torch.cuda.mem_get_info()[0]
    print(f"hgcd_many: {n} x {r} bits in {dt:.1f} s, {dt / n:.2f} s per gcd, "
          f"host cpu {cpu:.1f} s ({cpu / dt:.1f} cores of {os.cpu_count()}), "
          f"pool {pool / 2**30:.1f} GiB ({pool / n / 2**20:.0f} MiB a gcd), "
          f"degrees {sorted(set(degs.tolist()))[:4]}")


def case_sieve(a):
    smax = a.r // 2
    M.run_sieve(a.r, a.depth, smax)


def case_sieve_wide(a):
    """Degrees dmin..depth on the wide path (64-bit elements, sliced log
    table), from degree `wide_from` on."""
    os.environ["GF2E_SIEVE_WIDE_FROM"] = str(a.wide_from)
    smax = a.r // 2
    M.run_sieve(a.r, a.depth, smax, dmin=a.dmin)


def case_config4(a):
    """The batched deep scan at its stated shape: n seeded survivors of the
    d <= 24 sieve at r (every s <= (r-1)/2), each scanned to its least
    factor or maxd with the blocked DDF under the doubling interval schedule
    (L0, Lmax); writes <out>.results.txt ("s d p<hex>" / "s u" lines) and
    prints wall time, gcd count and gcd wall share (JSON)."""
    import json
    r, n = a.r, a.n
    smax = (r - 1) // 2
    t0 = time.perf_counter()
    best = M.run_sieve(r, 24, smax)
    t_sieve = time.perf_counter() - t0
    surv = np.nonzero(best == np.uint64(0xFFFFFFFFFFFFFFFF))[0]
    surv = surv[surv >= 3]
    rng = np.random.default_rng(a.seed)
    pick = np.sort(rng.choice(surv, size=min(n, surv.size), replace=False)).astype(np.uint64)
    S = M.engine.Scanner(r, slots=min(64, pick.size), block=a.block)
    S.submit(pick, k0=24, maxd=a.maxd, L0=a.l0, Lmax=a.lmax)
    lines = {}
    t1 = time.perf_counter()
    while len(lines) < pick.size:
        S.step(256)
        for s_, line in S.poll():
            lines[s_] = line
    t_scan = time.perf_counter() - t1
    gcds, t_gcd = S.gcd_time()
    pairs = S.pairs()
    S.close()
    with open(a.out + ".results.txt", "w") as f:
        f.write("".join(lines[s_] + "\n" for s_ in sorted(lines)))
    found = sum(1 for l in lines.values() if " p" in l)
    print(json.dumps({"r": r, "survivors": int(pick.size), "maxd": a.maxd, "block": a.block,
                      "L0": a.l0, "Lmax": a.lmax, "sieve_s": t_sieve, "scan_wall_s": t_scan,
                      "gcds": gcds, "gcd_wall_s": t_gcd, "gcd_share": t_gcd / t_scan,
                      "sd_pairs": pairs, "found": found, "u": int(pick.size) - found,
                      "results": a.out + ".results.txt"}))


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["square", "fft", "mul", "sieve", "sieve_wide", "gcd", "hgcd",
                                     "hgcd_many", "scan", "scan_step", "config4"])
    ap.add_argument("--r", type=int, default=136279841)
    ap.add_argument("--n", type=int, default=8)
    ap.add_argument("--k", type=int, default=3)
    ap.add_argument("--m", type=int, default=22)
    ap.add_argument("--depth", type=int, default=24)
    ap.add_argument("--dmin", type=int, default=2)
    ap.add_argument("--wide-from", type=int, default=32)
    ap.add_argument("--block", type=int, default=28)
    ap.add_argument("--maxd", type=int, default=20000)
    ap.add_argument("--l0", type=int, default=1024)
    ap.add_argument("--lmax", type=int, default=8192)
    ap.add_argument("--seed", type=int, default=4)
    ap.add_argument("--out", default="config4")
    a = ap.parse_args(argv)
    t0 = time.perf_counter()
    {"square": case_square, "fft": case_fft, "mul": case_mul, "sieve": case_sieve,
     "sieve_wide": case_sieve_wide, "gcd": case_gcd, "hgcd": case_hgcd,
     "hgcd_many": case_hgcd_many, "scan": case_scan, "scan_step": case_scan_step,
     "config4": case_config4}[a.case](a)
    print(f"{a.case}: done in {time.perf_counter() - t0:.3f} s")
    return 0


if __name__ == "__main__":
    sys.exit(main())
