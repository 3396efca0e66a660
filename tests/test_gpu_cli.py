"""The drop-in command-line tools on the GPU, against what the reference's own
tools produce for the same invocations (their outputs recorded in
tests/golden by make_golden.py, the reference run under its CPU emulation):

  trinomial_stage2 selftest | run r s k0 k1 prefix [state]
      .fk / .acc / .meta and the state file byte-equal to the reference's,
      including a run stopped at k = 1030 and resumed from its state file
      (trinomial_stage2.cu:195-277);
  trinomial_scan r survivors k0 maxd prefix [--state f]
      prefix.results.txt line for line equal to the reference's (ties, which
      the reference leaves as "s d g<file>", resolved to the least factor),
      a second run over the same file adding nothing, and runs resumed from
      state files in the reference's layout {0x4E435354, r, s, k, nw} + F_k
      (one written as the reference writes it, and the tool's own) giving
      the same lines (trinomial_scan.cu:144-170, 542-697);
  cantor_cuda selftest | bench bits
      the reference's report lines and residue checks (cantor_cuda.cu:103-189).
"""
import hashlib
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, load_json

pytestmark = pytest.mark.gpu

BIN = os.path.join(ROOT, "mersenne_trinomial_b200", "bin")


@pytest.fixture(scope="module")
def tools(engine):
    from mersenne_trinomial_b200 import build
    build.build_tools()
    return BIN


def run(args, cwd=None, timeout=900):
    p = subprocess.run(args, capture_output=True, text=True, cwd=cwd, timeout=timeout)
    return p.returncode, p.stdout, p.stderr


def sha_file(path):
    with open(path, "rb") as f:
        return hashlib.sha256(f.read()).hexdigest()


def test_stage2_selftest(tools):
    rc, out, err = run([os.path.join(tools, "trinomial_stage2"), "selftest"])
    assert rc == 0, err
    assert "STAGE2 SELFTEST: ALL PASS" in out


def test_stage2_runs_and_resume_match_reference(tools, tmp_path):
    fx = load_json("stage2_cli.json")
    exe = os.path.join(tools, "trinomial_stage2")
    state = tmp_path / "state.bin"
    for case in fx["runs"]:
        pre = str(tmp_path / case["name"])
        args = [exe, "run"] + case["args"] + [pre] + ([str(state)] if case["state"] else [])
        rc, out, err = run(args)
        assert rc == 0, err
        if case["name"] == "resume":
            assert "resumed at k=1030" in err
        for ext in (".fk", ".acc", ".meta"):
            assert sha_file(pre + ext) == case["sha256"][ext], (case["name"], ext)
        if case["state"]:
            assert sha_file(state) == case["sha256"]["state"], case["name"]


def test_scan_results_file_matches_reference(tools, tmp_path, oracle):
    fx = load_json("scan.json")
    r, k0, maxd = fx["r"], fx["k0"], fx["maxd"]
    surv = tmp_path / "surv.txt"
    surv.write_text("".join(f"{s}\n" for s in fx["survivors"]))
    pre = str(tmp_path / "scan")
    exe = os.path.join(tools, "trinomial_scan")
    rc, out, err = run([exe, str(r), str(surv), str(k0), str(maxd), pre, "--verbose", "0"])
    assert rc == 0, err
    got = open(pre + ".results.txt").read().splitlines()
    assert len(got) == len(fx["results"]) == len(fx["survivors"])
    # every line as the reference's; its three "s d g<file>" ties (several
    # factors of the least degree, left unresolved without NTL) resolved to
    # the least factor, checked as in test_gpu_scan
    from test_gpu_scan import check_against_reference
    assert check_against_reference(got, fx, oracle) == (104, 102, 2)
    # a second run over the same results file answers nothing twice
    rc, out, err = run([exe, str(r), str(surv), str(k0), str(maxd), pre, "--verbose", "0"])
    assert rc == 0, err
    assert open(pre + ".results.txt").read().splitlines() == got


def test_cantor_cuda_selftest_and_bench(tools):
    exe = os.path.join(tools, "cantor_cuda")
    rc, out, err = run([exe, "selftest"])
    assert rc == 0, err
    assert "GPU SELFTEST: ALL PASS" in out
    rc, out, err = run([exe, "bench", "8388608"])
    assert rc == 0, err
    lines = [l for l in out.splitlines() if l.startswith("residue check mod 0x")]
    assert len(lines) == 3 and all(l.endswith(": PASS") for l in lines), out


def _scan(exe, r, surv_path, k0, maxd, pre, *extra, env=None):
    return subprocess.run([exe, str(r), str(surv_path), str(k0), str(maxd), pre, "--verbose", "0",
                           *map(str, extra)], capture_output=True, text=True, timeout=900,
                          env=env)


def _read_states(path, r):
    nw = (r + 63) // 64
    raw = np.fromfile(path, dtype="<u8")
    recs, i = [], 0
    while i + 5 <= raw.size:
        magic, rr, s, k, n = (int(x) for x in raw[i:i + 5])
        assert magic == 0x4E435354 and rr == r and n == nw
        recs.append((s, k, raw[i + 5:i + 5 + nw].copy()))
        i += 5 + nw
    assert i == raw.size
    return recs


def test_scan_resume_from_state_files(tools, tmp_path, oracle):
    fx = load_json("scan.json")
    r, k0, maxd = fx["r"], fx["k0"], fx["maxd"]
    exe = os.path.join(tools, "trinomial_scan")
    surv = tmp_path / "surv.txt"
    surv.write_text("".join(f"{s}\n" for s in fx["survivors"]))
    # the uninterrupted run, saving its state at every step
    env = dict(os.environ, GF2E_SCAN_STATE_SECS="0")
    st1 = tmp_path / "run1.state"
    p = _scan(exe, r, surv, k0, maxd, str(tmp_path / "run1"), "--state", st1, "--l0", 8,
              "--interval", 8, "--batch", 16, env=env)
    assert p.returncode == 0, p.stderr
    want = open(str(tmp_path / "run1") + ".results.txt").read().splitlines()
    by_s = {int(l.split()[0]): l for l in want}
    recs = _read_states(st1, r)
    assert recs
    for s, k, F in recs:
        assert k0 < k < maxd
        assert (F == oracle.trin_square_k(oracle.x_state(r), r, s, k)).all(), (s, k)
    # a fresh results file resumed from that state: same lines
    p = _scan(exe, r, surv, k0, maxd, str(tmp_path / "run2"), "--state", st1)
    assert p.returncode == 0, p.stderr
    got = open(str(tmp_path / "run2") + ".results.txt").read().splitlines()
    assert sorted(got) == sorted(want)
    # a one-record file as the reference writes it, for an s whose least
    # degree lies beyond its frontier, and one whose frontier passed maxd
    d_of = {s: int(l.split()[1]) for s, l in by_s.items() if l.split()[1] != "u"}
    s1 = max(d_of, key=d_of.get)
    k1 = d_of[s1] - 3
    nw = (r + 63) // 64
    for s_, k_, expect in [(s1, k1, by_s[s1]), (s1, maxd + 5, f"{s1} u")]:
        st = tmp_path / f"ref_{k_}.state"
        F = oracle.trin_square_k(oracle.x_state(r), r, s_, min(k_, 4 * maxd))
        np.concatenate([np.array([0x4E435354, r, s_, k_, nw], dtype=np.uint64), F]).astype(
            "<u8").tofile(st)
        one = tmp_path / f"one_{k_}.txt"
        one.write_text(f"{s_}\n")
        pre = str(tmp_path / f"one_{k_}")
        p = _scan(exe, r, one, k0, maxd, pre, "--state", st)
        assert p.returncode == 0, p.stderr
        assert open(pre + ".results.txt").read().splitlines() == [expect]
