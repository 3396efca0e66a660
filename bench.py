#!/usr/bin/env python
"""Benchmark: squarings/s at r = 136279841 (bit-exact), plus the sieve and the
other hot-path legs measured in the same run.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = `nstates` seeded s values (default 64, 17 MB state each, 1.1 GB in
HBM, larger than L2) each squared `k` times (default 256) from x:
F_k = x^(2^k) mod x^r + x^s + 1, r = 136279841.  Multi-GPU (torchrun): every
rank squares its own s values (independent states, no data-path
collective), so scaling is weak; the timing is the max over ranks of CUDA-event
time.  One JSON line is printed by rank 0.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

R = 136279841


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--nstates", type=int, default=64)
    ap.add_argument("--k", type=int, default=256)
    ap.add_argument("--no-extras", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    return ap.parse_args()


# ------------------------------------------------------------------ clocks
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.gpu_id = gpu_id
        self.proc = None
        self.path = None

    def start(self):
        if not shutil.which("nvidia-smi"):
            return
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        self.proc = subprocess.Popen(
            ["nvidia-smi", "-i", self.gpu_id, "--query-gpu=" + self.FIELDS,
             "--format=csv,noheader,nounits", "-lms", "200"],
            stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                p = [x.strip() for x in line.split(",")]
                if len(p) < 8:
                    continue
                try:
                    sm.append(float(p[0]))
                    mx = float(p[1])
                except ValueError:
                    continue
                for i, nm in enumerate(names):
                    if p[4 + i].lower().startswith("active"):
                        reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def gpu_uuid(torch, dev):
    try:
        return "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        return str(dev)


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic(name):
    p = os.path.join(ROOT, "profiles", name)
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return None


# --------------------------------------------------------- CPU baselines
def cpu_stage2_reference(r, s_list, k, procs):
    """The reference's own squaring kernels (trinomial_stage2 run) under its CPU
    emulation header, `procs` concurrent processes, one s each."""
    exe = os.path.join(ROOT, "oracle", "_ref", "trinomial_stage2_emul")
    td = tempfile.mkdtemp(prefix="gf2e_cpu_")
    try:
        t0 = time.perf_counter()
        ps = [subprocess.Popen([exe, "run", str(r), str(int(s)), str(k + 1), str(k),
                                os.path.join(td, f"p{i}")],
                               stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
              for i, s in enumerate(s_list[:procs])]
        rc = [p.wait() for p in ps]
        wall = time.perf_counter() - t0
    finally:
        shutil.rmtree(td, ignore_errors=True)
    if any(rc):
        raise RuntimeError(f"reference CPU run failed: {rc}")
    return len(ps) * k / wall, wall


def cpu_stage2_port(r, s_list, k, procs):
    """The oracle's restatement of the reference squaring, threads (ctypes
    releases the GIL), when the reference build is absent."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle import oracle as O
    O.lib()

    def one(s):
        O.trin_square_k(O.x_state(r), r, int(s), k)
    t0 = time.perf_counter()
    with ThreadPoolExecutor(procs) as ex:
        list(ex.map(one, s_list[:procs]))
    wall = time.perf_counter() - t0
    return procs * k / wall, wall


def cpu_squaring_baseline(r, s_list, k):
    procs = max(1, min(os.cpu_count() or 1, len(s_list)))
    if os.path.exists(os.path.join(ROOT, "oracle", "_ref", "trinomial_stage2_emul")):
        v, wall = cpu_stage2_reference(r, s_list, k, procs)
        kind = "reference"
        what = "reference trinomial_stage2 kernels (cuda_emul.h CPU emulation)"
    else:
        v, wall = cpu_stage2_port(r, s_list, k, procs)
        kind = "port"
        what = "oracle restatement of the reference squaring"
    return {"value": v, "unit": "squarings/s", "cores": procs, "kind": kind,
            "sample": f"{procs} concurrent s values x {k} squarings at r={r} by {what}; "
                      f"{wall:.1f} s wall"}


# ---------------------------------------------------------------- reference arm
def run_reference_arm(args, rank):
    if rank != 0:
        return 0
    from mersenne_trinomial_b200 import workloads as W
    rng = np.random.default_rng(7)
    s_all = rng.integers(3, R // 2, size=4096).astype(np.uint64)
    procs = os.cpu_count() or 1
    ksq = 12                                   # squarings per process per step
    vals = []
    kind = "reference" if os.path.exists(os.path.join(ROOT, "oracle", "_ref",
                                                      "trinomial_stage2_emul")) else "port"
    fn = cpu_stage2_reference if kind == "reference" else cpu_stage2_port
    for i in range(args.warmup + args.steps):
        s = s_all[(i * procs) % 4096:][:procs]
        v, wall = fn(R, s, ksq, procs)
        if i >= args.warmup:
            vals.append((v, wall))
    v = statistics.median(x[0] for x in vals)
    wall = statistics.median(x[1] for x in vals)
    line = {
        "impl": "reference", "metric": "squarings/s at r=136279841 (bit-exact)",
        "value": v, "unit": "squarings/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": wall * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
        "config": {"workload": "x^(2^k) mod x^r+x^s+1, r=136279841, seeded s",
                   "sample": f"{procs} s x {ksq} squarings per step"},
        "cpu_baseline": {"value": v, "unit": "squarings/s", "cores": procs, "kind": kind,
                         "sample": f"{procs} concurrent s values x {ksq} squarings per step"},
        "e2e": {"value": v, "unit": "squarings/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------- ours
def main():
    args = parse()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        return run_reference_arm(args, rank)

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    import mersenne_trinomial_b200 as M
    from mersenne_trinomial_b200 import workloads as W
    M.lib()

    def barrier_sync():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    from mersenne_trinomial_b200 import multi

    def max_over_ranks(x):
        return multi.max_over_ranks(x, dist, device="cuda")

    r, n, k = R, args.nstates, args.k
    nw = (r + 63) // 64
    stride = nw + (nw & 1)
    s_host = multi.rank_s_values(r, n, rank)             # disjoint seeded s per rank
    states = torch.empty(stride * n, dtype=torch.int64, device="cuda")
    scratch = torch.empty_like(states)
    s_dev = torch.from_numpy(s_host.view(np.int64)).cuda()
    per_pass = M.engine.squarings_per_pass(r, stride, n)
    # passes of the squaring kernel per step (an odd pass count gets one
    # fused pass split in two, as gf2e_trin_square_batch does)
    n4 = k // 2 if per_pass == 2 else 0
    n1 = k - 2 * n4
    if (n4 + n1) % 2 and n4 > 0:
        n4, n1 = n4 - 1, n1 + 2
    copy_back = (n4 + n1) % 2
    launches_per_step = 1 + n4 + n1 + copy_back
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]

    def step(i=None):
        M.trin_set_x(states, stride, n, r)
        if i is not None:
            ev[i][0].record()
        M.trin_square_batch(states, scratch, stride, n, r, s_dev, k)
        if i is not None:
            ev[i][1].record()

    for _ in range(args.warmup):
        step()
    barrier_sync()
    # the timed result is checked: state 0 of rank 0 against x^(2^k) mod T as
    # the reference's own squaring kernels computed it (a committed fixture)
    if rank == 0:
        fx = [c for c in json.load(open(os.path.join(ROOT, "tests", "golden", "square.json")))
              ["cases"] if c["r"] == r and c["s"] == int(s_host[0]) and c["k"] == k]
        if fx:
            import hashlib
            got = states[:nw].cpu().numpy().view(np.uint64)
            if hashlib.sha256(np.ascontiguousarray(got).tobytes()).hexdigest() != fx[0]["sha256"]:
                raise RuntimeError(f"F_{k} for s={int(s_host[0])} differs from the reference's")
    clk = ClockSampler(gpu_uuid(torch, local))
    clk.start()
    barrier_sync()
    t_all0 = torch.cuda.Event(enable_timing=True)
    t_all1 = torch.cuda.Event(enable_timing=True)
    t_all0.record()
    for i in range(args.steps):
        step(i)
    t_all1.record()
    barrier_sync()
    clocks = clk.stop()
    total_ms = max_over_ranks(t_all0.elapsed_time(t_all1))
    step_ms = total_ms / args.steps
    sq_per_step = n * k
    value = world * sq_per_step / (step_ms / 1e3)
    # dominant kernel: the batched squaring pass (n4 two-squaring passes per
    # step at r = 136279841; each reads and writes every state once)
    passes = n4 + n1
    kern_ms = statistics.mean(a.elapsed_time(b) for a, b in ev) / passes
    kern_name = "k_frob4_batch" if n4 else "k_square_batch"
    algo_bytes = n * 2 * nw * 8                      # read + write each state once
    peak, peak_kind = measured_peaks()
    achieved = algo_bytes / (kern_ms / 1e3) / 1e9
    prof = profile_traffic("frob4_r136279841.json" if n4 else "square_r136279841.json")
    traffic = None
    if prof and prof.get("dram_bytes_per_state_pass"):
        traffic = prof["dram_bytes_per_state_pass"] * n

    # parity spot check of one state against the engine's independent FFT path
    # is in the tests; here the first state is checked against F_k from the
    # host-buffer API to make sure both paths agree.
    pinned = torch.empty((n, nw), dtype=torch.int64, pin_memory=True)
    out_np = pinned.numpy().view(np.uint64)
    # e2e: host s values in, host states out, through the C ABI
    M.frobenius_host(r, s_host, k, out=out_np)
    dev_first = states[:nw].cpu().numpy().view(np.uint64)
    if not (out_np[0] == dev_first).all():
        raise RuntimeError("host-buffer path disagrees with the device path")
    barrier_sync()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        M.frobenius_host(r, s_host, k, out=out_np)
    e2e_wall = max_over_ranks(time.perf_counter() - t0)
    e2e_value = world * sq_per_step * args.steps / e2e_wall

    extras = {}
    if rank == 0 and not args.no_extras:
        extras = run_extras(torch, M, W, sq_rate=value / world)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        ksq = 12
        cpu = cpu_squaring_baseline(r, s_host, ksq)

    if rank == 0:
        line = {
            "metric": "squarings/s at r=136279841 (bit-exact)",
            "value": value, "unit": "squarings/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": {"workload": f"x^(2^k) mod x^r+x^s+1, r={r}, {n} seeded s per GPU, "
                                   f"k={k} squarings per step from x",
                       "state_mb": round(nw * 8 / 2**20, 2),
                       "l2": "inputs (1.1 GB) larger than L2; no flush needed",
                       "parallelism": f"dp{world} (independent s per rank)"},
            "e2e": {"value": e2e_value, "unit": "squarings/s", "h2d_bytes_per_step": n * 8,
                    "d2h_bytes_per_step": n * nw * 8},
            "roofline": {"bound": "hbm", "achieved": achieved,
                         "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic, "kernel": kern_name,
                         "squarings_per_launch": 2 if n4 else 1,
                         "peak_source": peak_kind,
                         "algorithmic_bytes_per_launch": algo_bytes,
                         "launch_ms": kern_ms},
            "gpu_launches": launches_per_step * args.steps,
            "clocks": clocks,
            "cpu_baseline": cpu,
            "extras": extras,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def _ev_time(torch, fn, reps=3, flush=None):
    ts = []
    for _ in range(reps):
        if flush is not None:
            flush()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        torch.cuda.synchronize()
        ts.append(a.elapsed_time(b))
    return statistics.median(ts)


def run_extras(torch, M, W, sq_rate=None):
    """The other hot-path legs named by the metric / configurations."""
    out = {}
    flush_buf = torch.empty(64 * 2**20, dtype=torch.int64, device="cuda")   # 512 MB > L2

    def flush():
        flush_buf.fill_(1)

    # sieve at r = 136279841, d <= 24, every s <= floor(r/2)
    smax = R // 2
    best = torch.empty(smax + 1, dtype=torch.int64, device="cuda")
    ws = M.engine.SieveWorkspace(24)
    run = lambda: M.sieve_device(R, 24, smax, best, workspace=ws)
    run()
    ms = _ev_time(torch, run, 3, flush)
    out["sieve_r136279841_d24"] = {"pairs_per_s": smax * 23 / (ms / 1e3), "ms": ms,
                                   "pairs": smax * 23}
    # the reference's published full-range run: d <= 29 (7.52 s on its GPU,
    # coarse_sieve.log:9-40) and the dense-table limit d <= 31
    for dmax in (29, 31):
        wsd = M.engine.SieveWorkspace(dmax)
        rund = lambda: M.sieve_device(R, dmax, smax, best, workspace=wsd)
        rund()
        ms = _ev_time(torch, rund, 3)
        out[f"sieve_r136279841_d{dmax}"] = {"pairs_per_s": smax * (dmax - 1) / (ms / 1e3),
                                            "ms": ms, "pairs": smax * (dmax - 1)}
        if dmax == 29:
            h = best[1:].cpu().numpy().view(np.uint64)
            surv = int(np.count_nonzero(h == np.uint64(0xFFFFFFFFFFFFFFFF)))
            out["sieve_r136279841_d29"].update({"survivors": surv, "factors": smax - surv,
                                                "reference_published_s": 7.52})
        del wsd
    # the wide degrees 32..36 one at a time on the d <= 31 result (the
    # reference's coarse_sieve_wide runs, coarse_sieve.log:42-124); a repeat
    # of a degree is idempotent (min-merge of the same keys), so the second
    # run is the timed one
    published = {32: 162.86, 33: 593.48, 34: 2494.17, 35: None, 36: 44323.71}
    wide = {}
    for d in range(32, 37):
        wsd = M.engine.SieveWorkspace(d)
        rund = lambda: M.sieve_device(R, d, smax, best, dmin=d, fill=False, workspace=wsd)
        rund()
        ms = _ev_time(torch, rund, 1)
        h = best[1:].cpu().numpy().view(np.uint64)
        wide[f"d{d}"] = {"ms": ms, "workspace_GB": wsd.buf.nbytes / 2**30,
                         "survivors": int(np.count_nonzero(h == np.uint64(0xFFFFFFFFFFFFFFFF))),
                         "reference_published_s": published[d]}
        del wsd
    out["sieve_r136279841_wide_d32_d36"] = wide
    # config 1: r in [40000, 50000], d <= 20
    c1 = W.sieve_config(1)
    best1 = torch.empty(c1["smax"] + 1, dtype=torch.int64, device="cuda")
    ws1 = M.engine.SieveWorkspace(20)
    run1 = lambda: M.sieve_device(c1["r"], 20, c1["smax"], best1, workspace=ws1)
    run1()
    ms = _ev_time(torch, run1, 5)
    npairs = (c1["smax"] - 1) * 19
    out["sieve_config1"] = {"r": c1["r"], "pairs_per_s": npairs / (ms / 1e3), "ms": ms}
    # config 2: r ~ 1e6, 256 s, 4096 squarings
    c2 = W.squaring_config(1)
    r2 = c2["r"]
    nw2 = (r2 + 63) // 64
    st2 = nw2 + (nw2 & 1)
    a2 = torch.empty(st2 * 256, dtype=torch.int64, device="cuda")
    b2 = torch.empty_like(a2)
    s2 = torch.from_numpy(c2["s"].view(np.int64)).cuda()

    def run2():
        M.trin_set_x(a2, st2, 256, r2)
        M.trin_square_batch(a2, b2, st2, 256, r2, s2, 4096)
    run2()
    ms = _ev_time(torch, run2, 3, flush)
    out["squaring_config2"] = {"r": r2, "squarings_per_s": 256 * 4096 / (ms / 1e3), "ms": ms}
    # config 3: 64 uneven products
    c3 = W.mul_config(1)
    bufs, jobs = [], []
    for i, (ab, bb) in enumerate(c3["sizes"]):
        a = torch.from_numpy(W.random_bits(ab, 10 + i).view(np.int64)).cuda()
        b = torch.from_numpy(W.random_bits(bb, 500 + i).view(np.int64)).cuda()
        o = torch.empty(M.mul_out_words(ab, bb), dtype=torch.int64, device="cuda")
        bufs.append((a, b, o))
        jobs.append((a, ab, b, bb, o))
    wsb = M.mul_batch_dev(jobs)
    torch.cuda.synchronize()
    ms = _ev_time(torch, lambda: M.mul_batch_dev(jobs, workspace=wsb), 3, flush)
    tot_bits = sum(ab + bb for ab, bb in c3["sizes"])
    bytes3 = sum(48 * (1 << M.engine.fft_m_for(ab, bb)) + (ab + bb) // 4 for ab, bb in c3["sizes"])
    peak = measured_peaks()[0]

    def pass_bytes():
        # bytes the tile passes must move: each forward/inverse pass reads and
        # writes the n points once (two forwards and one inverse per product),
        # plus the 48 n of packing, pointwise product and overlap-add
        tot = 0
        for ab, bb in c3["sizes"]:
            m = M.engine.fft_m_for(ab, bb)
            F = M.CudaFFT()
            F.init(m)
            f, i = F.passes()
            F.fini()
            tot += 16 * (1 << m) * (2 * f + i) + 48 * (1 << m) + (ab + bb) // 4
        return tot
    pb3 = pass_bytes()
    out["mul_config3"] = {"products_per_s": 64 / (ms / 1e3), "ms": ms,
                          "algorithmic_GBps": bytes3 / (ms / 1e3) / 1e9,
                          "frac_of_measured_hbm": bytes3 / (ms / 1e3) / 1e9 / peak,
                          "pass_GBps": pb3 / (ms / 1e3) / 1e9,
                          "pass_frac_of_measured_hbm": pb3 / (ms / 1e3) / 1e9 / peak,
                          "operand_bits": tot_bits, "tuning": "built-in default"}
    # autotune the transform at the largest config-3 size (2^23 points), then
    # the same 64 products under the chosen settings
    from mersenne_trinomial_b200 import autotune as A
    dflt = A.resolve_by_size(A.tune_default(), 23)
    t0 = time.perf_counter()
    tuned = A.fft_autotune(23, reps=2)
    tune_s = time.perf_counter() - t0
    ms_t = _ev_time(torch, lambda: M.mul_batch_dev(jobs, workspace=wsb), 3, flush)
    dflt_row = [c for c in tuned["candidates"]
                if all(c[k] == dflt[k] for k in ("fft_tile_log", "fft_cmin", "fft_taylor_lv",
                                                  "fft_bfly_lv"))]
    pb3t = pass_bytes()
    out["mul_config3_tuned"] = {
        "products_per_s": 64 / (ms_t / 1e3), "ms": ms_t,
        "algorithmic_GBps": bytes3 / (ms_t / 1e3) / 1e9,
        "frac_of_measured_hbm": bytes3 / (ms_t / 1e3) / 1e9 / peak,
        "pass_GBps": pb3t / (ms_t / 1e3) / 1e9,
        "pass_frac_of_measured_hbm": pb3t / (ms_t / 1e3) / 1e9 / peak,
        "tuning": {k: v for k, v in tuned["best"].items() if k.startswith("fft_")},
        "autotune_s": tune_s, "candidates_verified": len(tuned["candidates"]),
        "fwd_inv_ms_m23": {"tuned": tuned["best_fwd_inv_ms"],
                           "default": dflt_row[0]["ms"] if dflt_row else None}}
    del bufs, jobs, wsb
    out["deep_scan_r136279841"] = deep_scan_sample(torch, M)
    # blocked DDF: block size from the measured modmul (per-degree sample) and
    # batched squaring costs
    from mersenne_trinomial_b200 import autotune as A
    t_mul = out["deep_scan_r136279841"]["ms_per_degree_per_s"] / 1e3
    t_sq = 1.0 / sq_rate if sq_rate else 7.2e-6          # batched state-squaring
    mblk = A.choose_block(t_mul, t_sq)
    out["deep_scan_r136279841_blocked"] = deep_scan_sample(torch, M, nsurv=8, degrees=4 * mblk,
                                                           block=mblk)
    out["deep_scan_r136279841_blocked"]["block_from"] = {"t_mul_s": t_mul, "t_sq_s": t_sq}
    out["deep_scan_r136279841_with_gcd"] = deep_scan_gcd_sample(M, block=32)
    # gcd interval schedule for config 4 (k0 = 24, d <= 20000) from this run's
    # per-degree cost (blocked) and amortised per-s gcd cost
    g = out["deep_scan_r136279841_with_gcd"]
    t_deg = out["deep_scan_r136279841_blocked"]["ms_per_degree_per_s"] / 1e3
    ns = len(g["survivors"])
    t_gcd = max(1e-3, g["wall_s"] - ns * (g["maxd"] - g["k0"]) * t_deg) / ns
    out["config4_interval_choice"] = A.choose_interval(24, 20000, t_deg, t_gcd)
    out["serving"] = serving_sample()
    return out


def deep_scan_sample(torch, M, nsurv=4, degrees=32, block=1):
    """Config 4's per-degree leg at full size: F <- F^2 and ACC <- ACC*(F+x)
    mod T for `nsurv` d<=24 survivors of r = 136279841, batched, degrees
    25..24+degrees; the interval-end half-gcds are measured by
    deep_scan_gcd_sample."""
    import ctypes as C
    from mersenne_trinomial_b200._lib import call
    smax = 200000
    best = M.run_sieve(R, 24, smax)
    surv = [s for s in range(3, smax + 1) if int(best[s]) == 0xFFFFFFFFFFFFFFFF][:nsurv]
    h = C.c_void_p()
    call("gf2e_scanner_create_blocked", R, nsurv, block, C.byref(h))
    s_arr = np.asarray(surv, dtype=np.uint64)
    call("gf2e_scanner_submit", h.value, s_arr.ctypes.data, nsurv, 24, 24 + 1000000, 1 << 30,
         1 << 30, 0)
    call("gf2e_scanner_step", h.value, block, None)          # ramp + first step (warm-up)
    torch.cuda.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record()
    call("gf2e_scanner_step", h.value, degrees, None)
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b)
    M.lib().gf2e_scanner_destroy(h.value)
    return {"survivors": surv, "degrees": degrees, "block": block, "ms": ms,
            "sd_pairs_per_s": nsurv * degrees / (ms / 1e3),
            "ms_per_degree_per_s": ms / degrees / nsurv,
            "note": ("square + running product per degree" if block == 1 else
                     f"blocked DDF, {block} degrees per step: Horner product, one modmul, "
                     f"{block}x{block} squarings") + " (no interval end in the sample)"}


def deep_scan_gcd_sample(M, nsurv=8, maxd=88, block=1):
    """Config 4's full cycle at r = 136279841 on a bounded sample: `nsurv`
    d<=24 survivors (s = 474 first, the reference's known answer
    `474 41 p3991ef16129`), ramp to k0 = 24, running products for degrees
    25..maxd, then the interval-end gcds (one lockstep half-gcd batch) and hit
    resolution; wall time of the whole scan call."""
    smax = 200000
    best = M.run_sieve(R, 24, smax)
    surv = [474] + [s for s in range(3, smax + 1)
                    if int(best[s]) == 0xFFFFFFFFFFFFFFFF and s != 474][:nsurv - 1]
    t0 = time.perf_counter()
    lines = M.scan(R, surv, 24, maxd, L0=maxd - 24, Lmax=4096, batch=nsurv, block=block)
    wall = time.perf_counter() - t0
    return {"survivors": surv, "k0": 24, "maxd": maxd, "results": lines, "wall_s": wall,
            "sd_pairs_per_s": nsurv * (maxd - 24) / wall,
            "known_answer_474": "474 41 p3991ef16129" in lines, "block": block,
            "note": "one interval of 64 degrees then one half-gcd per s (one lockstep batch)"}


def serving_sample(n_jobs=24, rate=16.0, seed=1):
    """Config 5: a seeded Poisson stream of (r, s-set, d-range) jobs.  Latency
    p50/p99 from the stream served in real time; throughput of continuous
    batching from the same jobs queued at once, against the plain path (each
    job alone on the GPU, back to back); every job's lines compared."""
    from mersenne_trinomial_b200 import serve
    # deep jobs at r = 136279841 (each s at least one 25 s half-gcd, 4 s when
    # 8-16 run at once) are measured by profile case serve_deep, not here
    jobs = serve.job_stream(seed, n_jobs, rate, deep_max=600, s_lo=16, s_hi=4096,
                            deep_s_cap={"1e7": 8}, deep_classes=("1e5", "1e6", "1e7"))
    lat, wall, lines, _ = serve.run_stream(jobs, slots=64)
    _, sat_wall, sat_lines, pairs = serve.run_stream(jobs, slots=64, realtime=False)
    plain_wall, plain_lines, plain_pairs = serve.run_one_at_a_time(jobs, slots=64)
    v = sorted(lat.values())
    same = all(lines[k] == plain_lines[k] == sat_lines[k] for k in lines)
    return {"jobs": n_jobs, "rate_per_s": rate, "p50_s": float(np.percentile(v, 50)),
            "p99_s": float(np.percentile(v, 99)), "realtime_wall_s": wall,
            "r_classes": sorted({int(j["r"]) for j in jobs}),
            "deep_jobs": sum(1 for j in jobs if j["dmax"] > 24),
            "s_per_job_max": max(int(j["s"].size) for j in jobs),
            "sieved_scanned_pairs": list(pairs),
            "sd_pairs_per_s_batched": sum(pairs) / sat_wall,
            "sd_pairs_per_s_plain_one_at_a_time": sum(plain_pairs) / plain_wall,
            "batched_over_plain": plain_wall / sat_wall,
            "results_identical_alone_vs_mixed": same}


if __name__ == "__main__":
    sys.exit(main())
