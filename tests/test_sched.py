"""Interval schedules of the deep scan (gf2e_sched_widths) against a
restatement of the reference's QSched (tsfactor.cu:831-894): linear growth
q += q0, the Euler-optimal recurrence with its first-interval argmin, the
--Zq cap; and trinomial_scan's doubling L0, 2 L0, ... Lmax.  CPU only."""
import math
import sys

import pytest

from conftest import ROOT

sys.path.insert(0, ROOT)


def qsched(opt: bool, m: int, q0: int, G: int, rho: float, zq: int, k_start: int, n: int):
    """tsfactor.cu:834-894 restated (test infrastructure): widths in degrees
    of the first n intervals, the first starting at degree k_start."""
    q = 0
    out = []
    k = k_start                         # grow(k) before the first interval

    def grow(k_end):
        nonlocal q
        if not opt:
            q = q + q0
            return
        w = q * m
        if not w:
            k0 = k_end
            C = 16.0 / 9.0
            best, bestk1 = 1e300, 0
            lo = int(1.02 * math.sqrt(float(k0) * float(G))) + 1
            if lo <= k0:
                lo = k0 + m
            for i in range(96):
                k1 = lo + int(float(lo) * 0.06 * i)
                E, kp, kc = 0.0, float(k0), float(k1)
                for _ in range(200):
                    if not kp < 4e18:
                        break
                    E += (C / kp) * ((kc - kp) + float(G))
                    nx = kc * kc / kp - float(G)
                    wn = nx - kc
                    wc = kc - kp
                    if wn < wc:
                        wn = wc
                    if wn < (rho - 1.0) * kc:
                        wn = (rho - 1.0) * kc
                    kp = kc
                    kc = kc + wn
                    if kp > 1e14:
                        break
                if E < best:
                    best, bestk1 = E, k1
            w = bestk1 - k0 if bestk1 > k0 else m
        else:
            kd, wd = float(k_end), float(w)
            wn = wd * kd / (kd - wd) - float(G)
            if wn < wd:
                wn = wd
            if wn < (rho - 1.0) * kd:
                wn = (rho - 1.0) * kd
            w = int(wn)
        q = (w + m - 1) // m
        if q < 1:
            q = 1

    grow(k)
    if zq and q > zq:
        q = zq
    for _ in range(n):
        out.append(q * m)
        k = k + q * m
        grow(k - 1)
        if zq and q > zq:
            q = zq
    return out


@pytest.fixture(scope="module")
def E():
    from mersenne_trinomial_b200 import engine
    return engine


@pytest.mark.parametrize("m,q0,k_start", [(4, 3, 25), (8, 2, 31), (14, 15, 100), (1, 600, 25),
                                          (46, 14, 25)])
def test_linear_matches_qsched(E, m, q0, k_start):
    got = E.sched_widths("linear", m, k_start, 40, q0=q0)
    assert got == qsched(False, m, q0, 4000, 1.25, 0, k_start, 40)


@pytest.mark.parametrize("m,G,rho,k_start", [(6, 60, 1.25, 25), (46, 4000, 1.25, 25),
                                             (1, 4000, 1.25, 1000), (32, 20000, 1.5, 31),
                                             (2, 100, 1.1, 3)])
def test_opt_matches_qsched(E, m, G, rho, k_start):
    got = E.sched_widths("opt", m, k_start, 60, G=G, rho=rho)
    want = qsched(True, m, 0, G, rho, 0, k_start, 60)
    # compare while the scanned degree stays below 10^12 (far past any run)
    n, k = 0, k_start
    while n < 60 and k + want[n] < 10 ** 12:
        k += want[n]
        n += 1
    assert n >= 8
    assert got[:n] == want[:n]
    # widths never shrink
    assert all(b >= a for a, b in zip(got[:n], got[1:n]))


def test_qcap_caps_both_modes(E):
    assert E.sched_widths("linear", 4, 25, 30, q0=3, qcap=20) == \
        qsched(False, 4, 3, 4000, 1.25, 20, 25, 30)
    assert E.sched_widths("opt", 6, 25, 30, G=60, qcap=7) == \
        qsched(True, 6, 0, 60, 1.25, 7, 25, 30)


def test_doubling_is_trinomial_scan(E):
    assert E.sched_widths("doubling", 1, 25, 10, L0=64, Lmax=4096) == \
        [64, 128, 256, 512, 1024, 2048, 4096, 4096, 4096, 4096]
    # blocked: whole blocks
    assert E.sched_widths("doubling", 46, 25, 4, L0=64, Lmax=4096)[:2] == [92, 184]


def test_bad_schedules_are_rejected(E):
    from mersenne_trinomial_b200 import Gf2eError
    with pytest.raises(Gf2eError):
        E.sched_widths("linear", 4, 25, 3, q0=0)
    with pytest.raises(Gf2eError):
        E.sched_widths("opt", 4, 25, 3, G=0)
    with pytest.raises(Gf2eError):
        E.sched_widths("opt", 4, 25, 3, rho=1.0)
    with pytest.raises(ValueError):
        E.make_sched("weekly")
