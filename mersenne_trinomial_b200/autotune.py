"""Autotuner: FFT tile/stage settings, sieve strip width, scan gcd interval.

Follows the contract of the reference's FFT autotune (tsfactor.cu:1986-2080,
knobs of gf2_cantor_cuda.h:24-60): every candidate is verified on the device
against the default configuration before it is timed, the winner stays
active in this process, and the settings are printed as environment lines
that later runs pick up (GF2E_FFT_TILE_LOG, GF2E_FFT_CMIN, GF2E_FFT_TAYLOR_LV,
GF2E_FFT_BFLY_LV, GF2E_SIEVE_STRIP_LOG).  The scan's gcd interval schedule is
chosen from measured costs by gf2e_scan_choose_interval.

    python -m mersenne_trinomial_b200.autotune [--m 22] [--sieve-r R --sieve-depth D]
        [--scan-r R] [--json out.json]
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import sys
import time

from ._lib import Tune, call

ENV_NAMES = {
    "fft_tile_log": "GF2E_FFT_TILE_LOG",
    "fft_cmin": "GF2E_FFT_CMIN",
    "fft_taylor_lv": "GF2E_FFT_TAYLOR_LV",
    "fft_bfly_lv": "GF2E_FFT_BFLY_LV",
    "sieve_strip_log": "GF2E_SIEVE_STRIP_LOG",
}


def tune_default() -> dict:
    t = Tune()
    call("gf2e_tune_default", C.byref(t))
    return t.as_dict()


def tune_get() -> dict:
    t = Tune()
    call("gf2e_tune_get", C.byref(t))
    return t.as_dict()


def resolve_by_size(tune: dict, m: int) -> dict:
    """The FFT knobs a plan of size 2^m uses when they are 0 ("by size"),
    the same rule as the library's plan creation."""
    t = dict(tune)
    if t["fft_tile_log"] == 0:
        t["fft_tile_log"] = 11 if m <= 17 else (12 if m <= 21 else 13)
    if t["fft_cmin"] == 0:
        t["fft_cmin"] = 2 if m <= 17 else (4 if m <= 23 else 8)
    return t


def tune_set(**kw) -> dict:
    """Set some knobs (others keep their current value); returns the new tuning."""
    cur = tune_get()
    cur.update(kw)
    t = Tune(**cur)
    call("gf2e_tune_set", C.byref(t))
    return tune_get()


def _parse_report(text: str, keys: list) -> list:
    rows = []
    for line in text.splitlines():
        parts = line.split()
        if len(parts) != len(keys):
            continue
        row = {}
        for k, v in zip(keys, parts):
            row[k] = v if k == "status" else (float(v) if k == "ms" else int(v))
        rows.append(row)
    return rows


def fft_autotune(m: int, reps: int = 3) -> dict:
    """Verify + time every FFT candidate at size 2^m; the winner stays active."""
    best, ms = Tune(), C.c_double()
    buf = C.create_string_buffer(1 << 16)
    call("gf2e_fft_autotune", m, reps, C.byref(best), C.byref(ms), buf, len(buf))
    rows = _parse_report(buf.value.decode(),
                         ["fft_tile_log", "fft_cmin", "fft_taylor_lv", "fft_bfly_lv", "ms", "status"])
    return {"m": m, "best": best.as_dict(), "best_fwd_inv_ms": ms.value, "candidates": rows}


def sieve_autotune(r: int, depth: int, smax: int, reps: int = 3) -> dict:
    """Verify + time every strip width on one sieve; the winner stays active."""
    best, ms = Tune(), C.c_double()
    buf = C.create_string_buffer(1 << 12)
    call("gf2e_sieve_autotune", r, depth, smax, reps, C.byref(best), C.byref(ms), buf, len(buf))
    rows = []
    for line in buf.value.decode().splitlines():
        p = line.split()
        if len(p) == 3:
            rows.append({"sieve_strip_log": int(p[0]), "ms": float(p[1]), "status": p[2]})
    return {"r": r, "depth": depth, "smax": smax, "best": best.as_dict(),
            "best_ms": ms.value, "candidates": rows}


def choose_block(t_mul: float, t_sq: float) -> int:
    """Block size of the blocked DDF from the modmul and squaring costs."""
    m = C.c_int()
    call("gf2e_scan_choose_block", float(t_mul), float(t_sq), C.byref(m))
    return m.value


def choose_interval(k0: int, maxd: int, t_degree: float, t_gcd: float) -> dict:
    """gcd interval schedule (L0 doubling to Lmax) minimising expected scan cost."""
    L0, Lmax, cost = C.c_uint64(), C.c_uint64(), C.c_double()
    call("gf2e_scan_choose_interval", k0, maxd, float(t_degree), float(t_gcd),
         C.byref(L0), C.byref(Lmax), C.byref(cost))
    return {"L0": L0.value, "Lmax": Lmax.value, "expected_cost": cost.value,
            "k0": k0, "maxd": maxd, "t_degree": t_degree, "t_gcd": t_gcd}


def measure_scan_costs(r: int, nstates: int = 8, degrees: int = 16, gcd_pairs: int = 4) -> dict:
    """Per-degree cost of the batched scan step and per-gcd cost at size r
    (seconds per s), measured with the engine's own calls."""
    import numpy as np
    from . import engine as E

    s_vals = [1000 + 7 * i for i in range(nstates)]
    # per degree: square + accumulate for every resident s (TrinGPU per s)
    ctx = E.TrinGPU()
    ctx.init(r)
    ctx.set_s(s_vals[0])
    ctx.set_x()
    ctx.reset_acc()
    ctx.square_A()
    ctx.accumulate()
    E.stream_sync()
    t0 = time.perf_counter()
    for _ in range(degrees):
        ctx.square_A()
        ctx.accumulate()
    E.stream_sync()
    t_deg = (time.perf_counter() - t0) / degrees
    acc = ctx.read("ACC")
    ctx.fini()
    # gcd of an accumulator-like operand against T, batched like the scan
    nw = (r + 1 + 63) // 64
    pairs = []
    for i in range(gcd_pairs):
        T = np.zeros(nw, dtype=np.uint64)
        for e in (0, s_vals[i % len(s_vals)], r):
            T[e >> 6] |= np.uint64(1 << (e & 63))
        pairs.append((E.DeviceBuffer.from_array(acc), r, E.DeviceBuffer.from_array(T), r + 1))
    E.gcd_batch(pairs[:1])
    t0 = time.perf_counter()
    E.gcd_batch(pairs)
    t_gcd = (time.perf_counter() - t0) / len(pairs)
    return {"r": r, "t_degree_s": t_deg, "t_gcd_s": t_gcd}


def export_lines(t: dict) -> list:
    return [f"export {ENV_NAMES[k]}={v}" for k, v in t.items()]


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--m", type=int, nargs="*", default=[22], help="FFT sizes to tune (2^m points)")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--sieve-r", type=int, default=136279841)
    ap.add_argument("--sieve-depth", type=int, default=24)
    ap.add_argument("--sieve-smax", type=int, default=0, help="default floor(r/2)")
    ap.add_argument("--no-sieve", action="store_true")
    ap.add_argument("--scan-r", type=int, default=0, help="measure scan costs at this r")
    ap.add_argument("--k0", type=int, default=24)
    ap.add_argument("--maxd", type=int, default=20000)
    ap.add_argument("--json", default="")
    a = ap.parse_args(argv)
    out = {"default": tune_default()}
    for m in a.m:
        res = fft_autotune(m, a.reps)
        out.setdefault("fft", []).append(res)
        print(f"fft m={m}: best {res['best']} fwd+inv {res['best_fwd_inv_ms']:.3f} ms", flush=True)
    if not a.no_sieve:
        smax = a.sieve_smax or a.sieve_r // 2
        res = sieve_autotune(a.sieve_r, a.sieve_depth, smax, a.reps)
        out["sieve"] = res
        print(f"sieve r={a.sieve_r} d<={a.sieve_depth}: strip 2^{res['best']['sieve_strip_log']} "
              f"{res['best_ms']:.3f} ms", flush=True)
    if a.scan_r:
        costs = measure_scan_costs(a.scan_r)
        out["scan_costs"] = costs
        out["interval"] = choose_interval(a.k0, a.maxd, costs["t_degree_s"], costs["t_gcd_s"])
        print(f"scan r={a.scan_r}: t_degree {costs['t_degree_s']*1e3:.3f} ms, "
              f"t_gcd {costs['t_gcd_s']*1e3:.1f} ms -> L0 {out['interval']['L0']} "
              f"Lmax {out['interval']['Lmax']}", flush=True)
    out["final"] = tune_get()
    for line in export_lines(out["final"]):
        print(line)
    if a.json:
        with open(a.json, "w") as f:
            json.dump(out, f, indent=1)
    return 0


if __name__ == "__main__":
    sys.exit(main())
