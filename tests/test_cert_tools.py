"""Certificate formats: cert2bin / bin2cert / check_ref (the reference's
cert2bin.c, bin2cert.c, check_ref.cpp) against the reference's own tools
built from its sources, on a sieve certificate from the oracle.  Host-only
tools: no GPU."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

BIN = os.path.join(ROOT, "mersenne_trinomial_b200", "bin")
REF = os.path.join(ROOT, "oracle", "_ref")


def _need(*paths):
    for p in paths:
        if not os.path.exists(p):
            pytest.skip(f"{p} not built")


@pytest.fixture(scope="module")
def image(oracle, tmp_path_factory):
    """found.bin of the oracle sieve at r = 44687, d <= 20 (s = 1..22343)."""
    best = oracle.sieve(44687, 20, 22343)
    d = tmp_path_factory.mktemp("certs")
    path = d / "f.found.bin"
    np.ascontiguousarray(best[1:], dtype="<u8").tofile(path)
    return d, path, best


def _run(cmd, **kw):
    return subprocess.run([str(c) for c in cmd], capture_output=True, text=kw.pop("text", True),
                          timeout=120, **kw)


def test_bin2cert_matches_reference(image):
    _need(os.path.join(BIN, "bin2cert"), os.path.join(REF, "bin2cert"))
    _, path, best = image
    ours = _run([os.path.join(BIN, "bin2cert"), path])
    ref = _run([os.path.join(REF, "bin2cert"), path])
    assert ours.returncode == ref.returncode == 0
    assert ours.stdout == ref.stdout
    assert ours.stdout.count("\n") == best.size - 1


@pytest.mark.parametrize("limit", [20, 12, 47, 0])
def test_cert2bin_matches_reference(image, limit):
    _need(os.path.join(BIN, "cert2bin"), os.path.join(REF, "cert2bin"))
    d, path, best = image
    cert = d / "f.cert"
    cert.write_text(_run([os.path.join(REF, "bin2cert"), path]).stdout)
    a, b = d / f"ours{limit}.bin", d / f"ref{limit}.bin"
    ro = _run([os.path.join(BIN, "cert2bin"), cert, a, limit])
    rr = _run([os.path.join(REF, "cert2bin"), cert, b, limit])
    assert ro.returncode == rr.returncode == 0
    assert a.read_bytes() == b.read_bytes()
    if limit >= 20:                             # round trip to the image
        assert a.read_bytes() == path.read_bytes()


@pytest.mark.parametrize("where", ["early", "middle", "last"])
@pytest.mark.parametrize("corrupt", ["order", "bits", "hex", "nop", "nodeg"])
def test_cert2bin_rejects_what_the_reference_rejects(image, corrupt, where):
    """Same exit, message and line number as the reference, for errors in
    the first and in later pieces of the parallel parse."""
    _need(os.path.join(BIN, "cert2bin"), os.path.join(REF, "cert2bin"))
    d, path, _ = image
    lines = _run([os.path.join(REF, "bin2cert"), path]).stdout.splitlines()
    start = {"early": 10, "middle": len(lines) * 3 // 5, "last": 0}[where]
    if where == "last":
        i = max(k for k, l in enumerate(lines) if " p" in l)
    else:
        i = next(k for k, l in enumerate(lines) if " p" in l and k > start)
    s, deg, mask = lines[i].split()
    if corrupt == "order":
        lines[i] = f"{int(s) + 1} {deg} {mask}"
    elif corrupt == "bits":
        lines[i] = f"{s} {int(deg) + 1} {mask}"
    elif corrupt == "hex":
        lines[i] = f"{s} {deg} {mask}z"
    elif corrupt == "nop":
        lines[i] = f"{s} {deg} {mask[1:]}"
    else:
        lines[i] = f"{s} x{deg} {mask}"
    cert = d / f"bad_{corrupt}_{where}.cert"
    cert.write_text("\n".join(lines) + "\n")
    ro = _run([os.path.join(BIN, "cert2bin"), cert, d / "o.bin", 40])
    rr = _run([os.path.join(REF, "cert2bin"), cert, d / "r.bin", 40])
    assert ro.returncode != 0 and rr.returncode != 0
    assert ro.stderr == rr.stderr                  # same message, same line number
    assert str(i + 1) in ro.stderr


def _summary(out):
    return [l for l in out.splitlines() if l.startswith(("  ", "reference lines", "sieve input",
                                                          "ALL CHECKS", "*** DISCREP"))]


@pytest.mark.parametrize("plant", [None, "mask", "survivor", "extra"])
def test_check_ref_matches_reference(image, plant):
    _need(os.path.join(BIN, "check_ref"), os.path.join(REF, "check_ref"))
    d, path, best = image
    cert = _run([os.path.join(REF, "bin2cert"), path]).stdout.splitlines()
    facts = [l for l in cert if " p" in l]
    surv = [l.split()[0] for l in cert if l.endswith(" u")]
    ref_lines = [l for l in facts if 14 <= int(l.split()[1]) <= 20]
    sieve = list(facts)
    if plant == "mask":                          # a wrong polynomial
        k = next(i for i, l in enumerate(sieve) if int(l.split()[1]) == 17)
        s_, d_, m_ = sieve[k].split()
        sieve[k] = f"{s_} {d_} p{int(m_[1:], 16) ^ 2:x}"
    elif plant == "survivor":                    # a factor lost
        k = next(i for i, l in enumerate(sieve) if int(l.split()[1]) == 19)
        surv.append(sieve.pop(k).split()[0])
    elif plant == "extra":                       # a factor the reference lacks
        ref_lines = [l for l in ref_lines if int(l.split()[1]) != 15]
    (d / "ref.txt").write_text("\n".join(ref_lines) + "\n")
    (d / "sieve.cert").write_text("\n".join(sieve) + "\n")
    (d / "surv.txt").write_text("\n".join(surv) + "\n")
    args = ["--ref", d / "ref.txt", "--dmin", 14, "--dmax", 20, "--cert", d / "sieve.cert",
            "--survivors", d / "surv.txt", "--smax", best.size - 1]
    ro = _run([os.path.join(BIN, "check_ref")] + args)
    rr = _run([os.path.join(REF, "check_ref")] + args)
    assert ro.returncode == rr.returncode == (0 if plant is None else 1)
    assert _summary(ro.stdout) == _summary(rr.stdout)


def _random_cert(rng, n):
    """A certificate of n records in the shapes cert2bin.c accepts, then
    (half the time) one random corruption."""
    out = []
    for s in range(1, n + 1):
        sp = rng.choice([" ", "  ", "\t", " \t"])
        if rng.random() < 0.25:
            tail = rng.choice(["", " trailing", "\tx"])
            out.append(f"{s}{sp}u{tail}")
            continue
        d = int(rng.integers(1, 60))
        mask = (int(rng.integers(0, 1 << 62)) & ((1 << d) - 1)) | (1 << d)
        h = format(mask, "x")
        if rng.random() < 0.2:
            h = h.upper()
        out.append(f"{s}{sp}{d}{sp}p{h}")
    if rng.random() < 0.5 and n > 1:
        i = int(rng.integers(0, n))
        kind = rng.choice(["swap", "drop", "letter", "noP", "bits", "dup", "lead", "hexz"])
        if kind == "swap" and i + 1 < n:
            out[i], out[i + 1] = out[i + 1], out[i]
        elif kind == "drop":
            out.pop(i)
        elif kind == "letter":
            out[i] = "x" + out[i]
        elif kind == "noP":
            out[i] = out[i].replace(" p", " q").replace("\tp", "\tq")
        elif kind == "bits":
            out[i] = out[i] + "0"
        elif kind == "dup":
            out.insert(i, out[i])
        elif kind == "lead":
            out[i] = out[i].split(None, 1)[0] + " ?"
        else:
            out[i] = out[i] + "z"
    sep = "\r\n" if rng.random() < 0.3 else "\n"
    blank = sep * int(rng.integers(0, 3))
    text = sep.join(l + (blank if rng.random() < 0.05 else "") for l in out)
    return text + (sep if rng.random() < 0.8 else "")


@pytest.mark.parametrize("seed", range(8))
def test_cert2bin_fuzz_against_reference(tmp_path, seed):
    """Random certificates and corruptions: the same exit code, message and
    output as the reference's cert2bin, for small inputs (cut into as many
    pieces as there are lines) and larger ones."""
    _need(os.path.join(BIN, "cert2bin"), os.path.join(REF, "cert2bin"))
    rng = np.random.default_rng(1000 + seed)
    for case in range(25):
        n = int(rng.choice([1, 2, 3, 7, 40, 3000]))
        cert = tmp_path / f"c{case}.cert"
        cert.write_bytes(_random_cert(rng, n).encode())
        lim = int(rng.choice([47, 30, 10, 0]))
        a, b = tmp_path / f"o{case}.bin", tmp_path / f"r{case}.bin"
        ro = _run([os.path.join(BIN, "cert2bin"), cert, a, lim])
        rr = _run([os.path.join(REF, "cert2bin"), cert, b, lim])
        assert (ro.returncode, ro.stderr) == (rr.returncode, rr.stderr), (seed, case, n, lim)
        if rr.returncode == 0:
            assert a.read_bytes() == b.read_bytes(), (seed, case)


def _odd_factor_line(rng, s):
    """A certificate line in one of the forms sscanf("%llu %d p%127s") and
    strtoull(hex, 16) read, canonical or not."""
    d = int(rng.integers(1, 40))
    mask = (int(rng.integers(0, 1 << 40)) & ((1 << d) - 1)) | (1 << d)
    h = format(mask, "x")
    form = int(rng.integers(0, 12))
    if form == 0:
        return f"{s} {d} p{h.upper()}"
    if form == 1:
        return f"{s} {d} p0x{h}"
    if form == 2:
        return f"  {s}\t{d}   p{h} trailing words"
    if form == 3:
        return f"{s:020d} {d} p{h}"
    if form == 4:
        return f"+{s} {d} p{h}"
    if form == 5:
        return f"{s} {d} p{h}" + "x" * 600           # split by fgets(512)
    if form == 6:
        return f"{s} {d} p{h}\r"
    if form == 7:
        return f"{s} {d} p{h}\0{s + 1} 3 p9"
    if form == 8:
        return f"garbage {s}"
    if form == 9:
        return ""
    return f"{s} {d} p{h}"


@pytest.mark.parametrize("seed", range(6))
def test_check_ref_fuzz_against_reference(tmp_path, seed):
    """Random certificate, survivors and reference files mixing canonical
    lines with other forms the reference's parsing accepts or skips: the
    same report and exit code as the reference's check_ref."""
    _need(os.path.join(BIN, "check_ref"), os.path.join(REF, "check_ref"))
    rng = np.random.default_rng(2000 + seed)
    for case in range(6):
        smax = int(rng.choice([50, 400, 3000]))
        surv = sorted(set(int(x) for x in rng.integers(1, smax + 1, size=smax // 4)))
        cert_s = [s for s in range(1, smax + 1) if s not in set(surv) or rng.random() < 0.02]
        cert = "\n".join(_odd_factor_line(rng, s) if rng.random() < 0.3 else
                         f"{s} {int(rng.integers(2, 36))} p{format((1 << 35) | int(rng.integers(0, 1 << 30)), 'x')}"
                         for s in cert_s)
        surv_txt = "\n".join(str(s) if rng.random() < 0.9 else rng.choice([f" {s}", f"{s}\r", f"+{s}", "x"])
                             for s in surv)
        ref = "\n".join(f"{s} {int(rng.integers(30, 35))} p{format((1 << 34) | s, 'x')}"
                        for s in sorted(rng.choice(np.arange(1, smax + 1), size=smax // 5, replace=False).tolist()))
        (tmp_path / "c.cert").write_bytes(cert.encode() + b"\n")
        (tmp_path / "s.txt").write_bytes(surv_txt.encode() + (b"\n" if rng.random() < 0.7 else b""))
        (tmp_path / "r.txt").write_bytes(ref.encode() + b"\n")
        args = ["--ref", tmp_path / "r.txt", "--cert", tmp_path / "c.cert", "--survivors",
                tmp_path / "s.txt", "--dmin", int(rng.choice([2, 30])), "--dmax", 34]
        if rng.random() < 0.5:
            args += ["--smax", smax]
        ro = _run([os.path.join(BIN, "check_ref")] + args)
        rr = _run([os.path.join(REF, "check_ref")] + args)
        assert (ro.returncode, ro.stdout) == (rr.returncode, rr.stdout), (seed, case)
