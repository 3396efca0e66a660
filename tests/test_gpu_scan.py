"""Batched deep scan (gf2e_scan) against the reference's trinomial_scan results
at r = 4423 (tests/golden/scan.json: 104 survivors, 102 found, 2 u, 3 ties)
under the reference selftest's two interval policies, and every reported
factor re-verified by the check-ntl restatement."""
import pytest

from conftest import load_json

pytestmark = pytest.mark.gpu


def gf2_divmod(a: int, b: int):
    """Quotient and remainder of GF(2)[x] polynomials held as Python ints."""
    q, db = 0, b.bit_length() - 1
    while a and a.bit_length() - 1 >= db:
        sh = a.bit_length() - 1 - db
        q |= 1 << sh
        a ^= b << sh
    return q, a


def check_against_reference(got, fx, oracle):
    """Every line of `got` against the reference's selftest results; returns
    (lines, found, u)."""
    r, k0, maxd = fx["r"], fx["k0"], fx["maxd"]
    want = {int(l.split()[0]): l for l in fx["results"]}
    nfound = nu = 0
    for line in got:
        s = int(line.split()[0])
        w = want[s].split()
        g = line.split()
        if w[1] == "u":
            assert g[1] == "u", line
            nu += 1
            continue
        nfound += 1
        assert g[1] == w[1] and g[2].startswith("p"), (line, want[s])
        if w[2].startswith("p"):
            assert g[2] == w[2], (line, want[s])
        else:
            # the reference without NTL defers this tie-break ('g<file>')
            st, d, gdeg, gh, mask = oracle.scan_one(r, s, k0, maxd)
            if mask is not None:                  # single factor: it is the gcd
                assert g[2] == "p" + mask
            else:                                 # two factors of degree d
                assert gdeg == 2 * d
                p, G = int(g[2][1:], 16), int(gh, 16)
                q, rem = gf2_divmod(G, p)
                assert rem == 0 and q.bit_length() - 1 == d and p < q
        assert oracle.factor_divides(r, s, int(g[1]), g[2][1:]) == 1
    return len(got), nfound, nu


@pytest.mark.parametrize("L0,Lmax,batch", [(32, 4096, 128), (8, 8, 16), (64, 4096, 7)])
def test_scan_matches_reference(engine, oracle, L0, Lmax, batch):
    fx = load_json("scan.json")
    r, k0, maxd = fx["r"], fx["k0"], fx["maxd"]
    got = engine.scan(r, fx["survivors"], k0, maxd, L0=L0, Lmax=Lmax, batch=batch)
    assert check_against_reference(got, fx, oracle) == (104, 102, 2)


def test_scan_results_in_input_order_and_retire_refill(engine):
    fx = load_json("scan.json")
    surv = list(reversed(fx["survivors"]))[:40]
    got = engine.scan(fx["r"], surv, fx["k0"], fx["maxd"], L0=16, Lmax=64, batch=5)
    assert [int(l.split()[0]) for l in got] == surv


def test_scan_rejects_bad_arguments(engine):
    with pytest.raises(engine.Gf2eError):
        engine.scan(4423, [2212], 5, 200)
    with pytest.raises(engine.Gf2eError):
        engine.scan(4423, [3], 5, 5)


@pytest.mark.timeout(900)
def test_scan_r136279841_known_answer(engine, oracle):
    """Config-4 path end to end at r = 136279841: ramp to k0 = 24, running
    product of (x^(2^k) + x) mod T for k = 25.., half-gcd at the interval
    end, hit resolution.  The reference's certificate for s = 474 is
    `474 41 p3991ef16129` (tsfactor_handoff.md:337)."""
    got = engine.scan(136279841, [474], 24, 200, L0=64, Lmax=4096, batch=1)
    assert got == ["474 41 p3991ef16129"]
    assert oracle.factor_divides(136279841, 474, 41, "3991ef16129") == 1


@pytest.mark.parametrize("block,L0,batch", [(2, 32, 128), (8, 8, 16), (16, 64, 7), (62, 64, 33)])
def test_blocked_scan_matches_per_degree_scan(engine, block, L0, batch):
    """tsfactor's blocked DDF (m degrees per step) gives the per-degree
    scanner's result for every survivor of the reference selftest at r = 4423
    (whose lines the per-degree scan reproduces exactly)."""
    fx = load_json("scan.json")
    r, k0, maxd = fx["r"], fx["k0"], fx["maxd"]
    want = engine.scan(r, fx["survivors"], k0, maxd, L0=32, Lmax=4096, batch=128)
    got = engine.scan(r, fx["survivors"], k0, maxd, L0=L0, Lmax=4096, batch=batch, block=block)
    assert got == want


def test_blocked_scan_rejects_bad_block(engine):
    for m in (3, 0, 64, -2):
        with pytest.raises(engine.Gf2eError):
            engine.scan(4423, [3], 5, 200, block=m)


@pytest.mark.timeout(900)
def test_blocked_scan_r136279841_known_answer(engine):
    """The blocked DDF at full size: `474 41 p3991ef16129` (blocks of 32
    degrees from k0 = 24, one gcd after two blocks)."""
    got = engine.scan(136279841, [474], 24, 200, L0=64, Lmax=4096, batch=1, block=32)
    assert got == ["474 41 p3991ef16129"]


@pytest.mark.gpu
@pytest.mark.parametrize("block,sched,kw", [(1, "linear", {"q0": 40}), (4, "linear", {"q0": 3}),
                                            (6, "opt", {"G": 60}), (2, "opt", {"G": 100, "rho": 1.1}),
                                            (8, "linear", {"q0": 2, "qcap": 5})])
def test_scheduled_scan_matches_doubling(engine, block, sched, kw):
    """tsfactor's interval schedules (QSched linear / Euler-optimal, --Zq)
    change only the gcd cadence: every result line of the r = 4423 selftest
    survivors equals the doubling schedule's."""
    fx = load_json("scan.json")
    r, k0, maxd = fx["r"], fx["k0"], fx["maxd"]
    want = engine.scan(r, fx["survivors"], k0, maxd, L0=32, Lmax=4096, batch=128)
    got = engine.scan(r, fx["survivors"], k0, maxd, batch=64, block=block, sched=sched, **kw)
    assert got == want


def test_late_hit_resolves_without_testing_cleared_degrees(engine, oracle):
    """Hits in intervals that start past 2 k0 are resolved from the gcd
    alone (the clear intervals exclude every lower factor degree); with
    8-degree intervals most of the selftest's hits are such, and every line
    still equals the reference's."""
    fx = load_json("scan.json")
    r, k0, maxd = fx["r"], fx["k0"], fx["maxd"]
    got = engine.scan(r, fx["survivors"], k0, maxd, L0=8, Lmax=8, batch=128)
    deep = [l for l in got if l.split()[1] != "u" and int(l.split()[1]) > 2 * k0 + 8]
    assert len(deep) >= 10
    assert check_against_reference(got, fx, oracle) == (104, 102, 2)


@pytest.mark.timeout(1200)
def test_deep_known_degree_r136279841(engine, oracle):
    """A degree-only known answer from the reference's own runs: at
    r = 136279841 the least factor of x^r + x^7458 + 1 has degree 30775
    (so the deep-scan workload, d <= 20000, reports it as u).  Blocked scan
    with long intervals (three interval gcds at this size), the factor
    re-verified by the check-ntl restatement."""
    r, s = 136279841, 7458
    got = engine.scan(r, [s], 24, 31000, L0=8192, Lmax=16384, batch=1, block=26)
    parts = got[0].split()
    assert parts[:2] == [str(s), "30775"], got
    mask = parts[2][1:]
    assert int(mask, 16).bit_length() == 30776
    assert oracle.factor_divides(r, s, 30775, mask) == 1
