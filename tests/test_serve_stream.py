"""The serving benchmark's job stream (config 5's request mix), host logic
only: seeded and reproducible, r from the config's four values, s-sets of
16..4096 values, d-ranges 2..24 for sieve jobs and 25..deep_max for deep
(squaring + gcd) jobs, deep s-sets capped per r class, Poisson arrivals."""
import numpy as np

from mersenne_trinomial_b200 import serve
from mersenne_trinomial_b200 import workloads as W


def test_stream_is_seeded_and_within_the_config():
    a = serve.job_stream(5, 60, rate=16.0, deep_max=600)
    b = serve.job_stream(5, 60, rate=16.0, deep_max=600)
    assert [(j["r"], j["dmax"], j["t"]) for j in a] == [(j["r"], j["dmax"], j["t"]) for j in b]
    assert all((x["s"] == y["s"]).all() for x, y in zip(a, b))
    assert [j["id"] for j in a] == list(range(1, 61))
    ts = [j["t"] for j in a]
    assert all(t1 > t0 for t0, t1 in zip(ts, ts[1:]))
    centres = dict(serve.R_CLASSES)
    rs = {j["r"] for j in a}
    assert len(rs) <= 4
    for r in rs:
        if r == W.R_DEEP:
            continue
        assert r % 8 in (1, 7) and r not in serve.BAD_R
        assert any(abs(r - c) <= 3000 for c in centres.values())
    for j in a:
        r, s, dmax = j["r"], j["s"], j["dmax"]
        assert 1 <= s.size <= 4096
        assert (np.diff(s.astype(np.int64)) > 0).all()           # sorted, no repeats
        assert int(s.min()) >= 3 and int(s.max()) < r // 2
        assert 2 <= dmax <= 600
        if dmax >= 25:                                          # a deep job
            cls = "deep" if r == W.R_DEEP else next(k for k, c in centres.items()
                                                     if abs(r - c) <= 3000)
            assert s.size <= serve.DEEP_S_CAP[cls]


def test_deep_jobs_only_where_asked():
    jobs = serve.job_stream(11, 80, rate=16.0, deep_max=300, deep_frac=1.0,
                            deep_classes=("1e5",))
    near_1e5 = [j for j in jobs if abs(j["r"] - serve.R_CLASSES["1e5"]) <= 3000]
    assert near_1e5 and all(j["dmax"] >= 25 for j in near_1e5)
    assert all(j["dmax"] <= 24 for j in jobs if j not in near_1e5)
    none = serve.job_stream(11, 80, rate=16.0, deep_max=300, deep_frac=0.0)
    assert all(j["dmax"] <= 24 for j in none)


def test_deep_caps_can_be_raised_per_class():
    jobs = serve.job_stream(3, 120, rate=16.0, deep_max=100, deep_frac=1.0, s_lo=4096,
                            deep_s_cap={"1e7": 1000}, deep_classes=("1e7",))
    deep = [j for j in jobs if j["dmax"] >= 25]
    assert deep and all(j["s"].size <= 1000 for j in deep)
    assert max(j["s"].size for j in deep) > serve.DEEP_S_CAP["1e7"]
