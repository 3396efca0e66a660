"""coarse_sieve checkpoints on the GPU: a run stopped at degree boundaries
(the reference's COARSE_TEST_STOP_AFTER_BUCKETS hook, one degree per unit
here) and resumed, possibly several times, writes the same outputs as an
uninterrupted run, and those equal the oracle sieve.  Covers full-image
and delta checkpoints (--load baseline), a checkpoint in the reference's
layout stopped inside a degree, and periodic saves."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from test_sieve_ckpt import parse, ref_file

pytestmark = pytest.mark.gpu

TOOL = os.path.join(ROOT, "mersenne_trinomial_b200", "bin", "coarse_sieve")
R, DEPTH, SMAX = 44687, 20, 22343


def sieve(*args, stop_after=None):
    env = dict(os.environ)
    env.pop("COARSE_TEST_STOP_AFTER_BUCKETS", None)
    if stop_after:
        env["COARSE_TEST_STOP_AFTER_BUCKETS"] = str(stop_after)
    p = subprocess.run([TOOL] + [str(a) for a in args], capture_output=True, text=True,
                       timeout=300, env=env)
    assert p.returncode == 0, p.stderr
    return p.stderr


def found(prefix):
    return np.fromfile(f"{prefix}.found.bin", dtype="<u8")


@pytest.fixture(scope="module")
def full(oracle, tmp_path_factory):
    if not os.path.exists(TOOL):
        from mersenne_trinomial_b200 import build
        build.build_lib()
        build.build_tools()
    d = tmp_path_factory.mktemp("full")
    sieve(R, DEPTH, d / "a", "--found")
    want = oracle.sieve(R, DEPTH, SMAX)[1:]
    got = found(d / "a")
    assert (got == want).all()
    return d / "a", got


def test_stop_twice_then_resume(full, tmp_path):
    prefix, want = full
    ck = tmp_path / "ck"
    err = sieve(R, DEPTH, tmp_path / "b", "--found", "--checkpoint", ck, stop_after=6)
    assert "stopping on request; resume with --resume" in err
    assert not os.path.exists(f"{tmp_path / 'b'}.found.bin")
    f = parse(ck)
    assert (f["d"], f["next"], f["kind"], f["r"], f["smax"], f["depth"]) == (8, 0, 0, R, SMAX, DEPTH)
    err = sieve(R, DEPTH, tmp_path / "b", "--found", "--resume", ck, stop_after=5)
    assert "continuing at degree 8" in err
    assert parse(ck)["d"] == 13 and parse(f"{ck}.1")["d"] == 8
    err = sieve(R, DEPTH, tmp_path / "b", "--found", "--resume", ck)
    assert "continuing at degree 13" in err
    assert (found(tmp_path / "b") == want).all()
    for ext in ("found.cert", "survivors.txt"):
        assert open(f"{tmp_path / 'b'}.{ext}").read() == open(f"{prefix}.{ext}").read()


def test_delta_checkpoint_against_load(full, tmp_path):
    _, want = full
    sieve(R, 12, tmp_path / "lo", "--found")
    lo = f"{tmp_path / 'lo'}.found.bin"
    ck = tmp_path / "ck"
    sieve(R, DEPTH, tmp_path / "c", "--found", "--load", lo, "--min-depth", 13, "--checkpoint", ck,
          stop_after=3)
    f = parse(ck)
    assert (f["kind"], f["bpath"], f["d"]) == (1, lo, 16)
    assert f["size"] == 80 + len(lo) + 16 * f["ndelta"] < 8 * SMAX
    sieve(R, DEPTH, tmp_path / "c", "--found", "--resume", ck)
    assert (found(tmp_path / "c") == want).all()


def test_reference_checkpoint_inside_a_degree(full, tmp_path):
    """A reference checkpoint saved after 3 of 8 buckets of degree 15: this
    engine runs degree 15 whole from the saved best[]."""
    _, want = full
    sieve(R, 14, tmp_path / "lo", "--found")
    image = found(tmp_path / "lo")
    ref_file(tmp_path / "ck", 15, 3, 8, r=R, smax=SMAX, depth=DEPTH, image=image)
    err = sieve(R, DEPTH, tmp_path / "d", "--found", "--resume", tmp_path / "ck")
    assert "degree 15 runs again whole" in err
    assert (found(tmp_path / "d") == want).all()


def test_periodic_saves(full, oracle, tmp_path):
    _, want = full
    ck = tmp_path / "ck"
    err = sieve(R, DEPTH, tmp_path / "e", "--found", "--checkpoint", ck, "--checkpoint-mins",
                1e-6, "--checkpoint-keep", 2)
    # a save after each degree whose end is at least the period after the
    # last save: most of degrees 2..19 (the smallest finish within 60 us)
    assert err.count("[checkpoint: d=") >= 8
    assert (found(tmp_path / "e") == want).all()
    newest, older = parse(ck), parse(f"{ck}.1")
    assert older["d"] < newest["d"] <= DEPTH and newest["period"] == 0
    assert not os.path.exists(f"{ck}.2")
    for f in (newest, older):                       # each image: degrees below d done
        assert (f["image"] == oracle.sieve(R, f["d"] - 1, SMAX)[1:]).all()
