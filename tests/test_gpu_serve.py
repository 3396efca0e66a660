"""Serving (continuous batching): every job's result is the same alone and in
the mix, the scanner path matches the oracle scan at small r, and jobs of
different r are resident together."""
import numpy as np
import pytest

from conftest import load_json

pytestmark = pytest.mark.gpu


def test_scanner_scan_matches_reference(engine):
    fx = load_json("scan.json")
    got = engine.scan(fx["r"], fx["survivors"], fx["k0"], fx["maxd"], L0=32, Lmax=4096, batch=32)
    want = {l.split()[0]: l for l in fx["results"]}
    for line in got:
        w = want[line.split()[0]]
        if " g" not in w:
            assert line == w


def test_job_alone_equals_job_in_mix(engine, oracle):
    from mersenne_trinomial_b200 import serve
    jobs = serve.job_stream(seed=5, n_jobs=8, rate=1000.0, deep_max=300, s_lo=8, s_hi=24,
                            deep_classes=("1e5", "1e6"))
    # the mix: everything submitted at once, stepped together
    lat, wall, mixed, pairs = serve.run_stream(jobs, slots=16, realtime=False)
    alone_wall, alone, alone_pairs = serve.run_one_at_a_time(jobs, slots=16)
    # pairs actually worked: the same sieve either way, and scanned pairs no
    # more than every deep s over its whole range
    assert pairs[0] == alone_pairs[0] > 0
    assert 0 < pairs[1] <= sum(int(j["s"].size) * int(j["dmax"]) for j in jobs if j["dmax"] > 24)
    assert set(mixed) == {j["id"] for j in jobs}
    for j in jobs:
        assert mixed[j["id"]] == alone[j["id"]], j["id"]
        assert len(mixed[j["id"]]) == j["s"].size
    # every reported factor divides its trinomial (check-ntl restatement)
    for j in jobs:
        for ln in mixed[j["id"]]:
            p = ln.split()
            if len(p) == 3 and p[2].startswith("p"):
                assert oracle.factor_divides(j["r"], int(p[0]), int(p[1]), p[2][1:]) == 1, ln
            else:
                assert p[1] == "u" and j["dmax"] >= 2


def test_sieve_only_job_matches_oracle(engine, oracle):
    from mersenne_trinomial_b200.serve import Server
    r = 44687
    s = np.arange(1, 400, dtype=np.uint64)
    srv = Server(8 << 30, 8)
    srv.submit(1, r, s, 12)
    done = []
    while not done:
        srv.step(4)
        done = srv.poll()
    lines = srv.lines(1)
    best = oracle.sieve(r, 12, 400)
    want = []
    for v in s.tolist():
        k = int(best[v])
        want.append(f"{v} u" if k == 0xFFFFFFFFFFFFFFFF else f"{v} {k >> 48} p{k & 0xFFFFFFFFFFFF:x}")
    assert lines == want
    srv.close()


def test_blocked_server_matches_per_degree_server(engine):
    """Scanners in blocked-DDF mode give every job the same lines as the
    per-degree scanners."""
    from mersenne_trinomial_b200 import serve
    jobs = serve.job_stream(seed=7, n_jobs=6, rate=1000.0, deep_max=300, s_lo=8, s_hi=24,
                            deep_classes=("1e5", "1e6"))
    _, _, plain, _ = serve.run_stream(jobs, slots=16, realtime=False)
    _, _, blocked, _ = serve.run_stream(jobs, slots=16, realtime=False, block=8)
    assert plain == blocked


def test_deep_jobs_at_large_r_in_the_mix(engine, oracle):
    """Deep (squaring + gcd) jobs at r ~ 1e7 and r = 136279841 beside small
    ones, s-sets up to a few thousand for sieve-only jobs: each job's lines
    equal the job alone, and every factor divides its trinomial."""
    from mersenne_trinomial_b200 import serve
    jobs = serve.job_stream(seed=11, n_jobs=8, rate=1000.0, deep_max=60, s_lo=16, s_hi=4096,
                            deep_s_cap={"1e7": 4, "deep": 2})
    assert any(j["r"] == 136279841 and j["dmax"] > 24 for j in jobs)
    assert any(j["r"] > 5_000_000 and j["r"] != 136279841 and j["dmax"] > 24 for j in jobs)
    _, _, mixed, pairs = serve.run_stream(jobs, slots=16, realtime=False)
    _, alone, _ = serve.run_one_at_a_time(jobs, slots=16)
    for j in jobs:
        assert mixed[j["id"]] == alone[j["id"]], j["id"]
        for ln in mixed[j["id"]]:
            p = ln.split()
            if len(p) == 3 and p[2].startswith("p"):
                assert oracle.factor_divides(j["r"], int(p[0]), int(p[1]), p[2][1:]) == 1, ln
