"""Regenerate the golden fixtures in tests/golden/ from the reference itself.

Runs the reference's own code built by oracle/build_ref.sh into oracle/_ref/
(sieve_ref, the reference engine's gf2x_fft_mul / CantorFFT through
libref_cantor.so, and the reference kernels of trinomial_stage2 /
trinomial_scan executed by the reference's CPU-emulation header).  Only this
container has the reference sources; the fixtures are committed so the tests
need neither the reference nor this script.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import gzip
import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from mersenne_trinomial_b200 import multi, workloads as W  # noqa: E402

REF = O.REF_DIR


def sha(data: bytes) -> str:
    return hashlib.sha256(data).hexdigest()


def run(cmd, **kw):
    return subprocess.run(cmd, check=True, capture_output=True, text=True, **kw)


def gen_sieve():
    out = {"cases": []}
    cfgs = [W.sieve_config(seed) for seed in (1, 2, 3)]
    for c in cfgs:
        txt = run([os.path.join(REF, "sieve_ref"), "run", str(c["r"]), str(c["dmax"]),
                   str(c["smax"])]).stdout
        name = f"sieve_r{c['r']}_d{c['dmax']}.txt.gz"
        with gzip.open(os.path.join(HERE, name), "wt") as f:
            f.write(txt)
        out["cases"].append({"r": c["r"], "depth": c["dmax"], "smax": c["smax"], "file": name,
                             "lines": txt.count("\n"), "sha256": sha(txt.encode())})
    # the reference GPU selftest configuration and the reference CPU selftests
    # (d <= 27 at r = 136279841: about 3 minutes of the reference CPU sieve)
    for r, depth, smax in [(136279841, 20, 999999), (136279841, 11, 30000),
                           (74207281, 10, 20000), (101, 9, 100), (136279841, 27, 999999)]:
        txt = run([os.path.join(REF, "sieve_ref"), "run", str(r), str(depth), str(smax)]).stdout
        out["cases"].append({"r": r, "depth": depth, "smax": smax, "file": None,
                             "lines": txt.count("\n"), "sha256": sha(txt.encode()),
                             "head": txt.splitlines()[:20]})
    sel = run([os.path.join(REF, "sieve_ref"), "selftest"]).stdout
    out["ref_selftest"] = sel.splitlines()
    with open(os.path.join(HERE, "sieve.json"), "w") as f:
        json.dump(out, f, indent=1)


def stage2(r, s, k0, k1):
    with tempfile.TemporaryDirectory() as td:
        pre = os.path.join(td, "o")
        run([os.path.join(REF, "trinomial_stage2_emul"), "run", str(r), str(s), str(k0), str(k1),
             pre])
        fk = np.fromfile(pre + ".fk", dtype="<u8")
        acc = np.fromfile(pre + ".acc", dtype="<u8")
    return fk, acc


def gen_square():
    cases = []
    def add(r, s, k, full):
        fk, _ = stage2(r, s, k + 1, k)
        c = {"r": r, "s": s, "k": k, "sha256": sha(fk.tobytes())}
        if full:
            c["words"] = [format(int(x), "x") for x in fk]
        cases.append(c)
    for k in (1, 2, 5, 31, 40):
        add(31, 3, k, True)                                  # trinomial_stage2.cu:75-99
    add(4423, 1200, 24, True)                                # trinomial_stage2.cu:100-121
    for s in (1, 2, 63, 64, 65, 127, 128, 129, 1000, 2211):  # word-boundary s (tsfactor.cu:1433-1438)
        add(4423, s, 50, True)
    for r in (127, 129, 191, 193, 255, 257):
        add(r, (r - 1) // 2, 37, True)
        add(r, 1, 37, True)
    cfg = W.squaring_config(1)
    for s in [int(x) for x in cfg["s"][:4]]:
        add(cfg["r"], s, 4096, False)
    # the benchmark's workload: F_256 at r = 136279841 for the first two s of
    # the default bench's seeded s values (state 0 is checked by bench.py),
    # and short runs at word-boundary s
    R = 136279841
    for s in [int(x) for x in multi.rank_s_values(R, 64, 0)[:2]]:
        add(R, s, 256, False)
    for s in (1, 63, 64, 65, 474, (R - 1) // 2):
        add(R, s, 3, False)
    # interval product ACC = prod_{k=5..12} (F_k + x) (trinomial_stage2.cu:123-146)
    _, acc = stage2(4423, 1200, 5, 12)
    prods = [{"r": 4423, "s": 1200, "k0": 5, "k1": 12, "words": [format(int(x), "x") for x in acc]}]
    _, acc = stage2(cfg["r"], int(cfg["s"][0]), 100, 103)
    prods.append({"r": cfg["r"], "s": int(cfg["s"][0]), "k0": 100, "k1": 103,
                  "sha256": sha(acc.tobytes())})
    sel = run([os.path.join(REF, "trinomial_stage2_emul"), "selftest"]).stdout
    with open(os.path.join(HERE, "square.json"), "w") as f:
        json.dump({"cases": cases, "products": prods, "ref_selftest": sel.splitlines()}, f, indent=1)


def gen_stage2_cli():
    """The reference's trinomial_stage2 run mode (under its CPU emulation):
    output files and the state file of a run stopped at k = 1030 and resumed
    to k = 2100, and of the same run without a state file
    (trinomial_stage2.cu:195-277)."""
    exe = os.path.join(REF, "trinomial_stage2_emul")
    out = {"runs": []}

    def files(pre, state=None):
        d = {}
        for ext in (".fk", ".acc", ".meta"):
            with open(pre + ext, "rb") as f:
                d[ext] = sha(f.read())
        if state:
            with open(state, "rb") as f:
                d["state"] = sha(f.read())
        return d
    with tempfile.TemporaryDirectory() as td:
        st = os.path.join(td, "state.bin")
        for name, args, use_state in [("stop", ["4423", "1200", "1000", "1030"], True),
                                      ("resume", ["4423", "1200", "1000", "2100"], True),
                                      ("straight", ["4423", "1200", "1000", "2100"], False)]:
            pre = os.path.join(td, name)
            run([exe, "run"] + args + [pre] + ([st] if use_state else []))
            out["runs"].append({"name": name, "args": args, "state": use_state,
                                "sha256": files(pre, st if use_state else None)})
        cfg = W.squaring_config(1)
        args = [str(cfg["r"]), str(int(cfg["s"][0])), "100", "103"]
        pre = os.path.join(td, "cfg2")
        run([exe, "run"] + args + [pre])
        out["runs"].append({"name": "config2", "args": args, "state": False,
                            "sha256": files(pre)})
    out["ref_selftest"] = run([exe, "selftest"]).stdout.splitlines()
    with open(os.path.join(HERE, "stage2_cli.json"), "w") as f:
        json.dump(out, f, indent=1)


def gen_fft():
    L = O.ref_cantor()
    cases = []
    for i, (ab, bb) in enumerate([(1, 1), (31, 33), (64, 64), (100, 77), (4096, 4096),
                                  (100000, 77777), (1 << 20, 1 << 19), (8000000, 8000000),
                                  (65536, 134217728 // 16), (3, 1 << 21)]):
        a = W.random_bits(ab, 1000 + i)
        b = W.random_bits(bb, 2000 + i)
        out = np.zeros(O.mul_out_words(ab, bb), dtype=np.uint64)
        L.ref_fft_mul(a, ab, b, bb, out)
        c = {"abits": ab, "bbits": bb, "seed_a": 1000 + i, "seed_b": 2000 + i,
             "sha256": sha(out.tobytes())}
        if out.size <= 300:
            c["words"] = [format(int(x), "x") for x in out]
        cases.append(c)
    tr = []
    for m in range(1, 15):
        f = W.splitmix64(77 + m, 1 << m)
        g = f.copy()
        L.ref_fft_fwd(g, m)
        t = {"m": m, "seed": 77 + m, "fwd_sha256": sha(g.tobytes())}
        if m <= 4:
            t["fwd_words"] = [format(int(x), "x") for x in g]
        tr.append(t)
    basis = np.zeros(64, dtype=np.uint64)
    n = L.ref_basis(basis)
    W10 = np.zeros(512, dtype=np.uint64)
    L.ref_twiddles(10, W10)
    sel = run([os.path.join(REF, "cantor_ref"), "selftest"]).stdout
    with open(os.path.join(HERE, "fft.json"), "w") as f:
        json.dump({"products": cases, "transforms": tr,
                   "basis": [format(int(x), "x") for x in basis[:n]],
                   "twiddles_m10_sha256": sha(W10.tobytes()),
                   "ref_selftest": sel.splitlines()}, f, indent=1)


def gen_scan():
    r, k0, maxd = 4423, 5, 200
    best = O.sieve(r, k0, 350)
    surv = [s for s in range(2, 351) if int(best[s]) == 0xFFFFFFFFFFFFFFFF]
    with tempfile.TemporaryDirectory() as td:
        sf = os.path.join(td, "surv.txt")
        with open(sf, "w") as f:
            f.write("".join(f"{s}\n" for s in surv))
        pre = os.path.join(td, "scan")
        run([os.path.join(REF, "trinomial_scan_emul"), str(r), sf, str(k0), str(maxd), pre,
             "--verbose", "0"])
        with open(pre + ".results.txt") as f:
            results = f.read().splitlines()
    sel = run([os.path.join(REF, "trinomial_scan_emul"), "--selftest"]).stdout
    with open(os.path.join(HERE, "scan.json"), "w") as f:
        json.dump({"r": r, "k0": k0, "maxd": maxd, "survivors": surv, "results": results,
                   "ref_selftest": sel.splitlines()}, f, indent=1)


def gen_verify():
    """Divisibility verdicts of the reference's Python verifier (verify_gf2_trinomial.py)."""
    src = os.environ.get("GF2E_REFERENCE_SRC")
    if not src or not os.path.isdir(src):
        raise SystemExit("make_golden: set GF2E_REFERENCE_SRC to the reference's src/ directory")
    sys.path.insert(0, src)
    import verify_gf2_trinomial as V  # the reference's own checker
    lines = [(136279841, "474 41 p3991ef16129"), (136279841, "33 5 p29"),
             (136279841, "474 41 p3991ef16128"), (136279841, "33 5 p2b"),
             (44687, "1 2 p7")]
    cert = gzip.open(os.path.join(HERE, f"sieve_r{W.sieve_config(1)['r']}_d20.txt.gz"), "rt").read()
    for ln in cert.splitlines()[:200:7]:
        lines.append((W.sieve_config(1)["r"], ln))
    out = []
    for r, ln in lines:
        s, d, p = ln.split()
        pi = int(p[1:], 16)
        ok = bool(V.divides_trinomial(pi, pi.bit_length() - 1, r, int(s))) and pi.bit_length() - 1 == int(d)
        out.append({"r": r, "line": ln, "divides": ok})
    with open(os.path.join(HERE, "verify.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    if not os.environ.get("GF2E_REFERENCE_SRC"):
        raise SystemExit("make_golden: set GF2E_REFERENCE_SRC to the reference's src/ directory")
    if not os.path.exists(os.path.join(REF, "sieve_ref")):
        O.build()
    gen_sieve()
    gen_square()
    gen_fft()
    gen_scan()
    gen_stage2_cli()
    gen_verify()
    print("golden fixtures written to", HERE)
