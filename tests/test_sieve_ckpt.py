"""Sieve checkpoint files (coarse_sieve --checkpoint / --resume) in the
reference's version-2 layout (coarse_sieve.cu:509-831): files built here byte
by byte from that layout are read by the engine's reader
(mersenne_trinomial_b200/csrc/tools/sieve_ckpt.h), and the files it writes
parse back under the layout.  Host only: a small driver over the header."""
import os
import struct
import subprocess

import numpy as np
import pytest

from conftest import ROOT

HDR = os.path.join(ROOT, "mersenne_trinomial_b200", "csrc", "tools")
SRC = os.path.join(ROOT, "tests", "ckpt_driver.cpp")
R, SMAX = 44687, 5000
ALL = (1 << 64) - 1


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    exe = tmp_path_factory.mktemp("drv") / "ckpt_driver"
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", HDR, "-o", str(exe), SRC], check=True,
                   timeout=180)
    return exe


def run(*args):
    return subprocess.run([str(a) for a in args], capture_output=True, text=True, timeout=60)


def keys(seed, smax=SMAX):
    """A best[] image: mostly keys (d << 48) | mask, some all-ones."""
    rng = np.random.default_rng(seed)
    d = rng.integers(2, 25, size=smax).astype(np.uint64)
    mask = rng.integers(1, 1 << 24, size=smax).astype(np.uint64)
    k = (d << np.uint64(48)) | mask
    k[rng.random(smax) < 0.3] = np.uint64(ALL)
    return k


def save(path, k):
    np.ascontiguousarray(k, dtype="<u8").tofile(path)


def load(path):
    return np.fromfile(path, dtype="<u8")


def fnv1a(k):
    h = 0xCBF29CE484222325
    for v in k.tolist():
        h = ((h ^ v) * 0x100000001B3) & ALL
    return h


def ref_file(path, d, nxt, nb, r=R, smax=SMAX, depth=24, period=0, kind=0, bpath=b"",
             bhash=0, image=None, pairs=()):
    """A checkpoint laid out as coarse_sieve.cu ckpt_write (600-640) writes it."""
    nd = len(pairs) if kind else 0
    body = b"GF2SVCK2" + struct.pack("<6I", 2, d, nxt, nb, kind, len(bpath))
    body += struct.pack("<6Q", r, smax, depth, period, bhash, nd) + bpath
    if kind:
        body += b"".join(struct.pack("<2Q", s, v) for s, v in pairs)
    else:
        body += np.ascontiguousarray(image, dtype="<u8").tobytes()
    with open(path, "wb") as f:
        f.write(body)


def parse(path):
    b = open(path, "rb").read()
    assert b[:8] == b"GF2SVCK2"
    h32 = struct.unpack_from("<6I", b, 8)
    h64 = struct.unpack_from("<6Q", b, 32)
    off = 80 + h32[5]
    out = {"version": h32[0], "d": h32[1], "next": h32[2], "nbuckets": h32[3], "kind": h32[4],
           "bpath": b[80:off].decode(), "r": h64[0], "smax": h64[1], "depth": h64[2],
           "period": h64[3], "hash": h64[4], "ndelta": h64[5], "size": len(b)}
    if h32[4]:
        out["pairs"] = [struct.unpack_from("<2Q", b, off + 16 * i) for i in range(h64[5])]
    else:
        out["image"] = np.frombuffer(b, dtype="<u8", count=h64[1], offset=off)
    return out


def read(driver, path, tmp_path, r=R, smax=SMAX):
    out = tmp_path / "read.bin"
    p = run(driver, "read", path, r, smax, out)
    if p.returncode:
        return None, p
    f = p.stdout.split()
    info = {"d": int(f[1]), "next": int(f[3]), "nbuckets": int(f[5]), "period": float(f[7]),
            "used": f[9], "base": int(f[11])}
    return (info, load(out)), p


def test_reference_full_image_is_read(driver, tmp_path):
    k = keys(1)
    ref_file(tmp_path / "c", 17, 0, 0, period=600, image=k)
    (info, got), _ = read(driver, tmp_path / "c", tmp_path)
    assert (got == k).all()
    assert (info["d"], info["next"], info["period"]) == (17, 0, 600)


@pytest.mark.parametrize("nxt,nb,want", [(3, 8, (30, 3, 8)), (8, 8, (31, 0, 0)),
                                         (0, 0, (30, 0, 0))])
def test_resume_point(driver, tmp_path, nxt, nb, want):
    """A finished bucketed degree resumes at the next degree (ckpt_read_one
    799-804); a part-done one keeps its coordinates."""
    ref_file(tmp_path / "c", 30, nxt, nb, image=keys(2))
    (info, _), _ = read(driver, tmp_path / "c", tmp_path)
    assert (info["d"], info["next"], info["nbuckets"]) == want


def test_delta_against_found_image(driver, tmp_path):
    base = keys(3)
    best = base.copy()
    rng = np.random.default_rng(4)
    idx = np.sort(rng.choice(SMAX, size=50, replace=False))
    best[idx] = (np.uint64(25) << np.uint64(48)) | np.uint64(12345)
    save(tmp_path / "base.found.bin", base)
    save(tmp_path / "best.bin", best)
    bp = str(tmp_path / "base.found.bin")
    p = run(driver, "write", tmp_path / "c", 3, R, SMAX, 26, 300, 26, 0, 0, tmp_path / "best.bin",
            1, bp)
    assert p.returncode == 0 and p.stdout.startswith("delta 1 entries 50"), p.stdout + p.stderr
    f = parse(tmp_path / "c")
    assert (f["version"], f["d"], f["kind"], f["bpath"], f["depth"], f["period"]) == \
        (2, 26, 1, bp, 26, 300)
    assert f["hash"] == fnv1a(base)
    assert f["pairs"] == [(int(i) + 1, int(best[i])) for i in idx]
    assert f["size"] == 80 + len(bp) + 16 * 50
    (info, got), _ = read(driver, tmp_path / "c", tmp_path)
    assert (got == best).all() and info["base"] == 1


def test_reference_delta_against_survivors_list(driver, tmp_path):
    """kind 2: listed s open, every other s the sentinel 0 (coarse_sieve.cu
    689-713); the delta sets keys on listed s."""
    listed = [5, 17, 400, 4999]
    (tmp_path / "surv.txt").write_text("".join(f"{s}\n" for s in listed) + "9999999\n")
    base = np.zeros(SMAX, dtype=np.uint64)
    base[np.array(listed) - 1] = np.uint64(ALL)
    bp = str(tmp_path / "surv.txt").encode()
    pairs = [(17, (27 << 48) | 0x1234567), (4999, (28 << 48) | 0x2345)]
    ref_file(tmp_path / "c", 29, 0, 0, kind=2, bpath=bp, bhash=fnv1a(base), pairs=pairs)
    (info, got), _ = read(driver, tmp_path / "c", tmp_path)
    want = base.copy()
    for s, v in pairs:
        want[s - 1] = v
    assert (got == want).all() and info["base"] == 2 and info["d"] == 29


def test_changed_baseline_falls_back_to_older_generation(driver, tmp_path):
    older, base = keys(5), keys(6)
    save(tmp_path / "older.bin", older)
    save(tmp_path / "base.found.bin", base)
    c = tmp_path / "c"
    assert run(driver, "write", c, 3, R, SMAX, 24, 0, 20, 0, 0, tmp_path / "older.bin").returncode == 0
    best = base.copy()
    best[7] = np.uint64(99)
    save(tmp_path / "best.bin", best)
    assert run(driver, "write", c, 3, R, SMAX, 24, 0, 21, 0, 0, tmp_path / "best.bin", 1,
               tmp_path / "base.found.bin").returncode == 0
    (info, got), _ = read(driver, c, tmp_path)
    assert info["d"] == 21 and (got == best).all()
    base[0] ^= np.uint64(1)                         # the baseline changed since
    save(tmp_path / "base.found.bin", base)
    (info, got), p = read(driver, c, tmp_path)
    assert info["used"].endswith("c.1") and info["d"] == 20 and (got == older).all()
    assert "not the one it was written against" in p.stderr


def test_generations_rotate(driver, tmp_path):
    save(tmp_path / "k.bin", keys(7))
    c = tmp_path / "c"
    for d in (5, 6, 7, 8):
        assert run(driver, "write", c, 3, R, SMAX, 24, 0, d, 0, 0, tmp_path / "k.bin").returncode == 0
    assert [parse(f"{c}{suf}")["d"] for suf in ("", ".1", ".2")] == [8, 7, 6]
    assert not os.path.exists(f"{c}.3") and not os.path.exists(f"{c}.tmp")
    with open(c, "r+b") as f:                       # a newest copy cut short
        f.truncate(100)
    (info, _), p = read(driver, c, tmp_path)
    assert info["d"] == 7 and "truncated" in p.stderr


def test_large_delta_writes_full_image(driver, tmp_path):
    base = keys(8)
    best = keys(9)                                  # differs almost everywhere
    save(tmp_path / "base.found.bin", base)
    save(tmp_path / "best.bin", best)
    p = run(driver, "write", tmp_path / "c", 1, R, SMAX, 24, 0, 22, 0, 0, tmp_path / "best.bin", 1,
            tmp_path / "base.found.bin")
    assert p.stdout.startswith("delta 0")
    f = parse(tmp_path / "c")
    assert f["kind"] == 0 and f["size"] == 80 + 8 * SMAX and (f["image"] == best).all()


def test_other_run_rejected(driver, tmp_path):
    ref_file(tmp_path / "c", 17, 0, 0, image=keys(10))
    assert read(driver, tmp_path / "c", tmp_path, r=R + 2)[0] is None
    ref_file(tmp_path / "c", 17, 0, 0, smax=SMAX - 1, image=keys(10, SMAX - 1))
    assert read(driver, tmp_path / "c", tmp_path)[0] is None
    (tmp_path / "c").write_bytes(b"GF2SVCK1" + bytes(72))
    assert read(driver, tmp_path / "c", tmp_path)[0] is None


def test_damaged_files_never_crash_the_reader(driver, tmp_path):
    """A delta checkpoint cut at every length and with single bytes
    flipped: the reader rejects it (or falls back to the older generation)
    and never crashes."""
    smax = 60
    base = keys(11, smax)
    best = base.copy()
    best[[3, 17, 41]] = np.uint64((9 << 48) | 0x3FF)
    save(tmp_path / "base.found.bin", base)
    save(tmp_path / "best.bin", best)
    save(tmp_path / "older.bin", keys(12, smax))
    c = tmp_path / "c"
    assert run(driver, "write", c, 2, R, smax, 24, 0, 9, 0, 0, tmp_path / "older.bin").returncode == 0
    assert run(driver, "write", c, 2, R, smax, 24, 0, 10, 0, 0, tmp_path / "best.bin", 1,
               tmp_path / "base.found.bin").returncode == 0
    good = open(c, "rb").read()
    rng = np.random.default_rng(5)
    damaged = [good[:n] for n in range(len(good))]
    for _ in range(60):
        b = bytearray(good)
        i = int(rng.integers(0, len(b)))
        b[i] ^= 1 << int(rng.integers(0, 8))
        damaged.append(bytes(b))
    for bit in range(32):                          # every bit of the path length
        b = bytearray(good)
        b[28 + bit // 8] ^= 1 << (bit % 8)
        damaged.append(bytes(b))
    for data in damaged:
        open(c, "wb").write(data)
        # bytes: a damaged baseline path may be echoed in the message
        p = subprocess.run([str(driver), "read", str(c), str(R), str(smax),
                            str(tmp_path / "o.bin")], capture_output=True, timeout=60)
        assert p.returncode in (0, 1), (len(data), p.returncode, p.stderr[-300:])
        if p.returncode == 0 and p.stdout.split()[9].endswith(b"c.1"):
            assert (load(tmp_path / "o.bin") == keys(12, smax)).all()


def test_coarse_sieve_rejects_foreign_checkpoints(tmp_path):
    """The tool reads --resume files before any device call: a checkpoint of
    another r or smax, or not a checkpoint, ends the run with exit 1 and the
    reason, as the reference's ckpt_read does (coarse_sieve.cu:742-760)."""
    tool = os.path.join(ROOT, "mersenne_trinomial_b200", "bin", "coarse_sieve")
    if not os.path.exists(tool):
        pytest.skip("coarse_sieve not built")
    smax = 22343
    ref_file(tmp_path / "other_r", 17, 0, 0, r=R + 2, smax=smax, image=keys(1, smax))
    ref_file(tmp_path / "other_smax", 17, 0, 0, r=R, smax=smax - 1, image=keys(1, smax - 1))
    (tmp_path / "junk").write_bytes(b"not a checkpoint at all" * 4)
    for name, why in [("other_r", "written for r="), ("other_smax", "written for r="),
                      ("junk", "not a version-2 sieve checkpoint")]:
        p = subprocess.run([tool, str(R), "20", str(tmp_path / "out"), "--resume",
                            str(tmp_path / name)], capture_output=True, text=True, timeout=60)
        assert p.returncode == 1, (name, p.stderr)
        assert why in p.stderr and "no usable checkpoint generation" in p.stderr, p.stderr
        assert not os.path.exists(f"{tmp_path / 'out'}.found.cert")
    # a valid one is read and the resume point reported before the first
    # device call (without a GPU the run stops there; with one it finishes)
    ref_file(tmp_path / "ok", 17, 3, 8, r=R, smax=smax, image=keys(1, smax))
    p = subprocess.run([tool, str(R), "20", str(tmp_path / "out"), "--resume", str(tmp_path / "ok")],
                       capture_output=True, text=True, timeout=300)
    assert p.returncode in (0, 1), p.stderr
    assert "degree 17 runs again whole" in p.stderr and "continuing at degree 17" in p.stderr
