"""The drop-in C++ headers (include/gf2e_cantor.hpp, gf2e_trinomial.hpp)
used from a compiled translation unit the way the reference's tools use
gf2_cantor_engine.h / gf2_cantor_cuda.h / gf2_trinomial_cuda.h
(tests/dropin_driver.cpp), every result checked against the oracle and
the reference's golden vectors: CantorFFT fwd/inv and W, CudaFFT::dW,
gf2x_fft_mul_buf (with its FA/FB scratch), gf2x_naive_mul / gf2x_comb_mul,
ModP / find_irreducible_modp residues, TrinGPU's Bb / F / dT1 / dFA / dFB
with k_pack / k_pointwise / k_overlap_add, cpu_square_mod and
cpu_mod_trinomial."""
import hashlib
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, load_json
from mersenne_trinomial_b200 import workloads as W

pytestmark = pytest.mark.gpu

SRC = os.path.join(ROOT, "tests", "dropin_driver.cpp")
PKG = os.path.join(ROOT, "mersenne_trinomial_b200")


@pytest.fixture(scope="module")
def drv(tmp_path_factory, engine):
    d = tmp_path_factory.mktemp("dropin")
    exe = d / "dropin_driver"
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                    "-I/usr/local/cuda/include", "-o", str(exe), SRC, "-L" + PKG, "-lgf2e",
                    "-Wl,-rpath," + PKG, "-L/usr/local/cuda/lib64", "-lcudart"],
                   check=True, timeout=300)

    def run(*args):
        p = subprocess.run([str(exe)] + [str(a) for a in args], capture_output=True, text=True,
                           timeout=600)
        assert p.returncode == 0, p.stderr
        return p.stdout
    run.dir = d
    return run


def save(path, arr):
    np.ascontiguousarray(arr, dtype=np.uint64).tofile(path)
    return path


def load(path):
    return np.fromfile(path, dtype="<u8")


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def test_cantor_fft_against_reference_transforms(drv):
    fx = load_json("fft.json")
    for t in fx["transforms"]:
        m = t["m"]
        f = W.splitmix64(t["seed"], 1 << m)
        out = drv.dir / f"fft{m}"
        drv("fft", m, save(drv.dir / f"in{m}", f), out)
        assert sha(load(out)) == t["fwd_sha256"], m
        assert (load(str(out) + ".inv") == f).all(), m


def test_twiddles_host_and_device(drv, oracle):
    out = drv.dir / "tw"
    drv("twiddles", 10, out)
    fx = load_json("fft.json")
    assert sha(load(out)) == fx["twiddles_m10_sha256"]
    assert (load(str(out) + ".dW") == load(out)).all()


@pytest.mark.parametrize("ab,bb", [(1, 1), (100, 77), (4096, 4096), (100000, 77777),
                                   (1 << 20, 1 << 19)])
def test_products(drv, oracle, ab, bb):
    a, b = W.random_bits(ab, ab + 5), W.random_bits(bb, bb + 9)
    want = oracle.comb_mul(a, ab, b, bb)
    pa, pb = save(drv.dir / "a", a), save(drv.dir / "b", b)
    for kind in ("mulbuf", "naive", "comb"):
        out = drv.dir / f"p_{kind}"
        drv(kind, ab, bb, pa, pb, out)
        assert (load(out) == want).all(), (kind, ab, bb)
    # FA holds the product's chunk coefficients, FB the transform of b
    m = int(np.ceil(np.log2(max(2, (ab + 31) // 32 + (bb + 31) // 32 - 1))))
    FA, FB = load(str(drv.dir / "p_mulbuf") + ".FA"), load(str(drv.dir / "p_mulbuf") + ".FB")
    assert FA.size == FB.size == 1 << m
    nch = (ab + 31) // 32 + (bb + 31) // 32 - 1
    assert (FA[nch:] == 0).all()
    bch = np.zeros(1 << m, dtype=np.uint64)
    b32 = np.concatenate([b, [np.uint64(0)]]).view(np.uint32)[:(bb + 31) // 32]
    bch[:b32.size] = b32
    assert (FB == oracle.fft_fwd(bch, m)).all()


def _irreducible_prime_degree(q, d):
    """x^(2^d) = x mod q for q of prime degree d (then q is irreducible)."""
    def mulmod(a, b):
        r = 0
        while b:
            if b & 1:
                r ^= a
            b >>= 1
            a <<= 1
            if a >> d & 1:
                a ^= q
        return r
    t = 2
    for _ in range(d):
        t = mulmod(t, t)
    return t == 2


def test_modp_residues_of_a_product(drv, oracle):
    ab = bb = 1 << 18
    a, b = W.random_bits(ab, 1), W.random_bits(bb, 2)
    c = oracle.comb_mul(a, ab, b, bb)
    pa, pb, pc = save(drv.dir / "ra", a), save(drv.dir / "rb", b), save(drv.dir / "rc", c)
    for seed in (0x1234567, 0xDEADBEEF, 0xC0FFEE):
        qa, ra = map(int, drv("modp", 61, seed, pa, ab).split())
        qb, rb = map(int, drv("modp", 61, seed, pb, bb).split())
        qc, rc = map(int, drv("modp", 61, seed, pc, ab + bb).split())
        assert qa == qb == qc and qa >> 61 == 1
        assert _irreducible_prime_degree(qa, 61)
        assert (ra, rb, rc) == (oracle.residue(a, ab, qa, 61), oracle.residue(b, bb, qa, 61),
                                oracle.residue(c, ab + bb, qa, 61))
        # residue of the product = product of the residues (mod q)
        assert rc == oracle.modq_mul(ra, rb, qa, 61)


@pytest.mark.parametrize("r,s,k", [(4423, 1200, 9), (4423, 1, 3), (999961, 400000, 5),
                                   (136279841, 474, 3)])
def test_tringpu_members_and_cpu_checks(drv, oracle, r, s, k):
    out = drv.dir / f"t{r}_{s}"
    drv("trin", r, s, k, out)
    fk = oracle.trin_square_k(oracle.x_state(r), r, s, k)
    f1 = oracle.trin_square_k(fk, r, s, 1)
    assert (load(out) == fk).all()
    for ext in (".fft", ".sq", ".cpu", ".mod"):
        assert (load(str(out) + ext) == f1).all(), ext
