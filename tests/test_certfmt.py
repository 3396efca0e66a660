"""Result text (mersenne_trinomial_b200/csrc/tools/certfmt.h): certificate
lines "s d p<hex>", survivor lines and bin2cert's "s u" lines, formatted by
several threads, byte-identical to printf("%" PRIu64 " %u p%" PRIx64 "\\n")
(coarse_sieve.cu:1510-1558, bin2cert.c), including edge keys and line
counts that cross the formatter's 2^22-key rounds.  Host only."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

HDR = os.path.join(ROOT, "mersenne_trinomial_b200", "csrc", "tools")
SRC = os.path.join(ROOT, "tests", "certfmt_driver.cpp")
BIN = os.path.join(ROOT, "mersenne_trinomial_b200", "bin")
REF = os.path.join(ROOT, "oracle", "_ref")
NONE = (1 << 64) - 1


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    exe = tmp_path_factory.mktemp("fmt") / "certfmt_driver"
    subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", "-I", HDR, "-o", str(exe), SRC],
                   check=True, timeout=180)
    return exe


def keys(n, seed):
    rng = np.random.default_rng(seed)
    d = rng.integers(1, 48, size=n).astype(np.uint64)
    mask = rng.integers(1, 1 << 48, size=n, dtype=np.uint64) >> rng.integers(0, 48, size=n).astype(np.uint64)
    k = (d << np.uint64(48)) | mask
    k[rng.random(n) < 0.2] = np.uint64(NONE)
    k[rng.random(n) < 0.01] = np.uint64(0)
    edge = [NONE, 0, (1 << 48) - 1, (65535 << 48) | 1, 1 << 48, (2 << 48) | 0x3]
    k[: len(edge)] = np.array(edge, dtype=np.uint64)
    return k


def expected(k, s0, kind):
    out = []
    for i, v in enumerate(k.tolist()):
        s = s0 + i
        if kind == "cert":
            if v in (NONE, 0):
                continue
            out.append(f"{s} {v >> 48} p{v & 0xFFFFFFFFFFFF:x}\n")
        elif kind == "survivors":
            if v == NONE:
                out.append(f"{s}\n")
        else:
            out.append(f"{s} u\n" if v == NONE else f"{s} {v >> 48} p{v & 0xFFFFFFFFFFFF:x}\n")
    return "".join(out)


@pytest.mark.parametrize("kind", ["cert", "survivors", "bin2cert"])
@pytest.mark.parametrize("threads", [1, 7])
def test_lines_match_printf_format(driver, tmp_path, kind, threads):
    k = keys(200_003, 1)
    k.astype("<u8").tofile(tmp_path / "k.bin")
    s0 = 18446744073709000000 if kind == "survivors" else 1   # widest decimal s too
    p = subprocess.run([str(driver), kind, str(tmp_path / "k.bin"), str(s0), str(threads)],
                       capture_output=True, text=True, timeout=120)
    assert p.returncode == 0
    want = expected(k, s0, kind)
    assert p.stdout == want
    assert int(p.stderr) == want.count("\n")


def test_bin2cert_large_image_matches_reference(tmp_path):
    """4.5 M records (two formatter rounds) against the reference's own
    bin2cert built from its sources, and the text back through cert2bin."""
    ours, ref = os.path.join(BIN, "bin2cert"), os.path.join(REF, "bin2cert")
    for p in (ours, ref):
        if not os.path.exists(p):
            pytest.skip(f"{p} not built")
    k = keys(4_500_000, 2)
    img = tmp_path / "big.found.bin"
    k.astype("<u8").tofile(img)
    a = subprocess.run([ours, str(img)], capture_output=True, timeout=300)
    b = subprocess.run([ref, str(img)], capture_output=True, timeout=300)
    assert a.returncode == b.returncode == 0
    assert a.stdout == b.stdout
    # and back (about 90 MB of text: more than one 64 MB read block of the
    # parallel cert2bin), against the reference's cert2bin
    c2b, rc2b = os.path.join(BIN, "cert2bin"), os.path.join(REF, "cert2bin")
    if os.path.exists(c2b) and os.path.exists(rc2b):
        rng = np.random.default_rng(3)                 # valid keys: masks of exactly d+1 bits
        d = rng.integers(2, 48, size=k.size).astype(np.uint64)
        m = rng.integers(0, 1 << 48, size=k.size, dtype=np.uint64)
        m = (m & ((np.uint64(1) << d) - np.uint64(1))) | (np.uint64(1) << d)
        k = (d << np.uint64(48)) | m
        k[rng.random(k.size) < 0.2] = np.uint64(NONE)
        k.astype("<u8").tofile(img)
        cert = tmp_path / "big.cert"
        cert.write_bytes(subprocess.run([ours, str(img)], capture_output=True, timeout=300).stdout)
        for lim in (20, 47):
            ro = subprocess.run([c2b, str(cert), str(tmp_path / "o.bin"), str(lim)], timeout=300)
            rr = subprocess.run([rc2b, str(cert), str(tmp_path / "r.bin"), str(lim)], timeout=300)
            assert ro.returncode == rr.returncode == 0
            assert (tmp_path / "o.bin").read_bytes() == (tmp_path / "r.bin").read_bytes()
        assert (tmp_path / "o.bin").read_bytes() == img.read_bytes()   # LIMIT 47: the image itself
        assert (tmp_path / "o.bin").stat().st_size == 8 * k.size
