"""Host-side mirror of the reference's entry points over libgf2e.so.

Names, argument meaning and error behaviour follow the reference headers:
  gf2_cantor_engine.h   CantorBasis, gf2x_fft_mul, bits_to_words, mul_out_words
  gf2_cantor_cuda.h     CudaFFT (init/fwd/inv/fini)
  gf2_trinomial_cuda.h  TrinGPU (init/set_s/reset_acc/square_A/mul_dev/
                        accumulate/reduce/fini), spread32
  sieve_ref.cpp /
  coarse_sieve.cu       run_sieve / run_gpu -> best[] of packed keys
Every computation runs on the GPU through the C ABI; bad arguments raise
Gf2eError where the reference prints and exits.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np

from ._lib import Gf2eError, MulJob, call, check, lib

U64_MAX = np.uint64(0xFFFFFFFFFFFFFFFF)
MASK48 = 0xFFFFFFFFFFFF


def bits_to_words(bits: int) -> int:
    """gf2_cantor_engine.h:198."""
    return (int(bits) + 63) >> 6


def mul_out_words(abits: int, bbits: int) -> int:
    """gf2_cantor_engine.h:201-203."""
    return int(lib().gf2e_mul_out_words(abits, bbits))


def fft_m_for(abits: int, bbits: int) -> int:
    return int(lib().gf2e_mul_fft_m(abits, bbits))


def _sp(stream) -> Optional[int]:
    """cudaStream_t from None / int / torch.cuda.Stream."""
    if stream is None:
        return None
    if hasattr(stream, "cuda_stream"):
        return int(stream.cuda_stream) or None
    return int(stream) or None


class DeviceBuffer:
    """A device allocation owned by Python (gf2e_device_alloc / _free)."""

    def __init__(self, nbytes: int):
        self.nbytes = int(nbytes)
        p = C.c_void_p()
        call("gf2e_device_alloc", C.byref(p), self.nbytes)
        self.ptr = int(p.value)

    @classmethod
    def from_array(cls, arr: np.ndarray, stream=None) -> "DeviceBuffer":
        a = np.ascontiguousarray(arr)
        b = cls(max(a.nbytes, 8))
        if a.nbytes:
            call("gf2e_copy_to_device", b.ptr, a.ctypes.data, a.nbytes, _sp(stream))
        return b

    def upload(self, arr: np.ndarray, offset_bytes: int = 0, stream=None) -> None:
        a = np.ascontiguousarray(arr)
        if offset_bytes + a.nbytes > self.nbytes:
            raise ValueError("upload beyond buffer")
        call("gf2e_copy_to_device", self.ptr + offset_bytes, a.ctypes.data, a.nbytes, _sp(stream))

    def to_numpy(self, count: Optional[int] = None, dtype=np.uint64, offset_bytes: int = 0,
                 stream=None) -> np.ndarray:
        item = np.dtype(dtype).itemsize
        if count is None:
            count = (self.nbytes - offset_bytes) // item
        out = np.empty(count, dtype=dtype)
        if out.nbytes:
            call("gf2e_copy_to_host", out.ctypes.data, self.ptr + offset_bytes, out.nbytes,
                 _sp(stream))
        return out

    def free(self) -> None:
        if getattr(self, "ptr", 0):
            lib().gf2e_device_free(self.ptr)
            self.ptr = 0

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def _ptr(x) -> int:
    """Device address of a DeviceBuffer, a torch CUDA tensor or an int."""
    if isinstance(x, DeviceBuffer):
        return x.ptr
    if hasattr(x, "data_ptr"):
        if not x.is_cuda:
            raise ValueError("expected a CUDA tensor")
        return int(x.data_ptr())
    return int(x)


def stream_sync(stream=None) -> None:
    call("gf2e_stream_sync", _sp(stream))


# ===================================================================== sieve
def primitive_poly(d: int) -> int:
    """gf2_field_setup.h:49-58 (find_primitive_poly)."""
    return int(lib().gf2e_primitive_poly(d))


class SieveWorkspace:
    def __init__(self, dmax: int):
        n = C.c_size_t()
        call("gf2e_sieve_workspace_size", dmax, C.byref(n))
        self.dmax = dmax
        self.buf = DeviceBuffer(n.value)

    def stats(self, stream=None):
        cls = np.zeros(self.dmax + 1, dtype=np.uint64)
        mk = np.zeros(self.dmax + 1, dtype=np.uint64)
        call("gf2e_sieve_stats", self.buf.ptr, self.dmax, cls.ctypes.data, mk.ctypes.data,
             _sp(stream))
        return cls, mk


def sieve_device(r: int, dmax: int, smax: int, best, dmin: int = 2, fill: bool = True,
                 workspace: Optional[SieveWorkspace] = None, stream=None) -> SieveWorkspace:
    """Sieve into a device best[] of smax+1 u64 (coarse_sieve.cu run_gpu)."""
    ws = workspace if workspace is not None and workspace.dmax >= dmax else SieveWorkspace(dmax)
    if fill:
        call("gf2e_sieve_fill", _ptr(best), smax, _sp(stream))
    call("gf2e_sieve_run", r, dmin, dmax, smax, _ptr(best), ws.buf.ptr, ws.buf.nbytes, _sp(stream))
    return ws


def run_sieve(r: int, depth: int, smax: int, dmin: int = 2, preload: Optional[np.ndarray] = None,
              stream=None) -> np.ndarray:
    """best[s], s = 0..smax, packed (d << 48) | mask or all-ones (sieve_ref.cpp:125-134)."""
    best = DeviceBuffer(8 * (smax + 1))
    if preload is not None:
        best.upload(np.asarray(preload, dtype=np.uint64), stream=stream)
    sieve_device(r, depth, smax, best, dmin=dmin, fill=preload is None, stream=stream)
    return best.to_numpy(smax + 1, stream=stream)


def fmt_line(s: int, key: int) -> str:
    """'s d p<hex>' (sieve_ref.cpp:163-169)."""
    return f"{s} {key >> 48} p{key & MASK48:x}"


def cert_lines(best: np.ndarray, smin: int = 1) -> list:
    b = np.asarray(best, dtype=np.uint64)
    idx = np.nonzero(b != U64_MAX)[0]
    out = []
    for s in idx.tolist():
        if s < smin:
            continue
        k = int(b[s])
        if k == 0:
            continue
        out.append(fmt_line(s, k))
    return out


# ================================================================ Cantor FFT
class CantorBasis:
    """gf2_cantor_engine.h:74-121."""

    def __init__(self):
        self.b = np.zeros(64, dtype=np.uint64)
        self.len = 0

    def build(self) -> None:
        n = C.c_int()
        call("gf2e_cantor_basis", self.b.ctypes.data, C.byref(n))
        self.len = n.value

    def verify(self) -> bool:
        from .gf64 import gf64_mul_host  # host check only, no device work
        if self.len < 1 or int(self.b[0]) != 1:
            return False
        for i in range(1, self.len):
            y = int(self.b[i])
            if gf64_mul_host(y, y) ^ y != int(self.b[i - 1]):
                return False
        return True


class CudaFFT:
    """gf2_cantor_cuda.h:361-521: in-place transforms of n = 2^m device words."""

    def __init__(self):
        self._plan = None
        self.m = 0
        self.n = 0

    def init(self, m: int, basis: Optional[CantorBasis] = None) -> None:
        p = C.c_void_p()
        call("gf2e_fft_plan_create", m, C.byref(p))
        self._plan = p.value
        self.m = m
        self.n = 1 << m

    @property
    def plan(self) -> int:
        if not self._plan:
            raise Gf2eError(-1, "CudaFFT used before init")
        return self._plan

    def fwd(self, buf, stream=None) -> None:
        call("gf2e_fft_fwd", self.plan, _ptr(buf), _sp(stream))

    def inv(self, buf, stream=None) -> None:
        call("gf2e_fft_inv", self.plan, _ptr(buf), _sp(stream))

    def passes(self) -> tuple:
        """(forward, inverse) tile passes of this plan."""
        f, i = C.c_int(), C.c_int()
        call("gf2e_fft_plan_passes", self.plan, C.byref(f), C.byref(i))
        return f.value, i.value

    def twiddles(self) -> np.ndarray:
        W = np.zeros(max(1, self.n >> 1), dtype=np.uint64)
        call("gf2e_fft_twiddles", self.plan, W.ctypes.data)
        return W

    def fini(self) -> None:
        if self._plan:
            lib().gf2e_fft_plan_destroy(self._plan)
            self._plan = None

    def __del__(self):
        try:
            self.fini()
        except Exception:
            pass


def gf2x_fft_mul_dev(fft: CudaFFT, a, abits: int, b, bbits: int, out, fa, fb, stream=None) -> None:
    """gf2x_fft_mul_buf on device buffers (gf2_cantor_engine.h:207-229)."""
    call("gf2e_mul", fft.plan, _ptr(a), abits, _ptr(b), bbits, _ptr(out), _ptr(fa), _ptr(fb),
         _sp(stream))


def gf2x_fft_mul(a: np.ndarray, abits: int, b: np.ndarray, bbits: int, stream=None) -> np.ndarray:
    """c = a * b over GF(2)[x] for host arrays (gf2_cantor_engine.h:232-242), on the GPU."""
    m = fft_m_for(abits, bbits)
    F = CudaFFT()
    F.init(m)
    ow = mul_out_words(abits, bbits)
    da = DeviceBuffer.from_array(_words(a, abits), stream)
    db = DeviceBuffer.from_array(_words(b, bbits), stream)
    dout = DeviceBuffer(8 * ow)
    fa = DeviceBuffer(8 << m)
    fb = DeviceBuffer(8 << m)
    gf2x_fft_mul_dev(F, da, abits, db, bbits, dout, fa, fb, stream)
    out = dout.to_numpy(ow, stream=stream)
    F.fini()
    return out


def _words(a, bits):
    a = np.ascontiguousarray(a, dtype=np.uint64)
    need = bits_to_words(bits)
    if a.size < need:
        a = np.concatenate([a, np.zeros(need - a.size, dtype=np.uint64)])
    return a[:need] if a.size > need else a


def mul_batch_dev(jobs: Sequence[tuple], stream=None, workspace: Optional[DeviceBuffer] = None):
    """Many products in one call; jobs = [(a_dev, abits, b_dev, bbits, out_dev), ...]."""
    arr = (MulJob * len(jobs))()
    for i, (a, ab, b, bb, o) in enumerate(jobs):
        arr[i] = MulJob(_ptr(a), ab, _ptr(b), bb, _ptr(o))
    need = C.c_size_t()
    call("gf2e_mul_batch_workspace_size", arr, len(jobs), C.byref(need))
    ws = workspace
    if ws is None or ws.nbytes < need.value:
        ws = DeviceBuffer(need.value)
    call("gf2e_mul_batch", arr, len(jobs), ws.ptr, ws.nbytes, _sp(stream))
    return ws


def mul_batch_workspace_bytes(sizes: Sequence[tuple]) -> int:
    arr = (MulJob * len(sizes))()
    for i, (ab, bb) in enumerate(sizes):
        arr[i] = MulJob(0, ab, 0, bb, 0)
    need = C.c_size_t()
    call("gf2e_mul_batch_workspace_size", arr, len(sizes), C.byref(need))
    return need.value


# ======================================================================= gcd
def gcd_batch(pairs, g_cap_words: int = 0, stream=None):
    """deg gcd(a, b) for every (a_dev, abits, b_dev, bbits) pair, on the GPU
    (gf2_gcd.h:48-75 contract: 0 means gcd = 1).  With g_cap_words > 0 the
    gcds that fit are returned as host arrays (None where they do not fit)."""
    from ._lib import GcdJob
    n = len(pairs)
    jobs = (GcdJob * n)()
    outs = []
    for i, (a, ab, b, bb) in enumerate(pairs):
        g = DeviceBuffer(8 * g_cap_words) if g_cap_words else None
        outs.append(g)
        jobs[i] = GcdJob(_ptr(a), ab, _ptr(b), bb, g.ptr if g else None, g_cap_words)
    need = C.c_size_t()
    call("gf2e_gcd_workspace_size", jobs, n, C.byref(need))
    ws = DeviceBuffer(need.value)
    degs = np.zeros(n, dtype=np.int64)
    call("gf2e_gcd_batch", jobs, n, degs.ctypes.data, ws.ptr, ws.nbytes, _sp(stream))
    gs = []
    for d, g in zip(degs.tolist(), outs):
        if g is None or d // 64 + 1 > g_cap_words:
            gs.append(None)
        else:
            gs.append(g.to_numpy(g_cap_words, stream=stream))
    return degs, gs


def gcd_large(pairs, g_cap_words: int = 0, max_parallel: int = 1, stream=None):
    """Subquadratic (half-gcd) gcd of every (a_dev, abits, b_dev, bbits) pair,
    same contract as gcd_batch; for operands of millions of bits up to
    r = 136279841 (the reference delegates these to NTL, gf2_gcd_ntl.cpp:32-42).
    max_parallel >= 2 runs the pairs as lockstep batches of up to that many
    (at most 64, and as many as device memory holds): one recursion, one
    launch per step, for the whole batch.  Returns (degrees, gcds or None,
    work counters; in a batch the step counters count batch steps)."""
    from ._lib import GcdJob, HgcdStats
    n = len(pairs)
    jobs = (GcdJob * n)()
    outs = []
    for i, (a, ab, b, bb) in enumerate(pairs):
        g = DeviceBuffer(8 * g_cap_words) if g_cap_words else None
        outs.append(g)
        jobs[i] = GcdJob(_ptr(a), ab, _ptr(b), bb, g.ptr if g else None, g_cap_words)
    degs = np.zeros(n, dtype=np.int64)
    st = HgcdStats()
    call("gf2e_gcd_large", C.cast(jobs, C.c_void_p), n, degs.ctypes.data, max_parallel,
         C.byref(st), _sp(stream))
    gs = []
    for d, g in zip(degs.tolist(), outs):
        if g is None or d // 64 + 1 > g_cap_words:
            gs.append(None)
        else:
            gs.append(g.to_numpy(g_cap_words))
    return degs, gs, st.as_dict()


def _hex(words) -> str:
    x = 0
    for i, w in enumerate(np.asarray(words, dtype=np.uint64).tolist()):
        x |= int(w) << (64 * i)
    return format(x, "x")


def make_sched(sched: str = "doubling", q0: int = 0, G: int = 4000, rho: float = 1.25,
               qcap: int = 0):
    """Interval schedule (include/gf2e.h gf2e_sched): 'doubling' (trinomial_scan
    L0, 2 L0, ... Lmax), 'linear' (tsfactor q0, 2 q0, ... blocks) or 'opt'
    (tsfactor's Euler-optimal widths, gcd cost G degrees, floor rho)."""
    from ._lib import SCHED_MODES, Sched
    if sched not in SCHED_MODES:
        raise ValueError(f"schedule {sched!r}: one of {sorted(SCHED_MODES)}")
    return Sched(SCHED_MODES[sched], q0, G, rho, qcap)


def sched_widths(sched: str, block: int, k_start: int, n: int, L0: int = 64, Lmax: int = 4096,
                 **kw) -> list:
    """The first n interval widths (degrees) of a scan starting at k_start."""
    q = make_sched(sched, **kw)
    out = np.zeros(max(1, n), dtype=np.uint64)
    call("gf2e_sched_widths", C.byref(q), block, k_start, L0, Lmax, n, out.ctypes.data)
    return [int(x) for x in out[:n]]


def scan(r: int, survivors, k0: int, maxd: int, L0: int = 64, Lmax: int = 4096,
         batch: int = 64, mask_cap_words: int = 1024, stream=None, block: int = 1,
         sched: str = "doubling", q0: int = 0, G: int = 4000, rho: float = 1.25,
         qcap: int = 0) -> list:
    """Deep scan (trinomial_scan.cu): one result line per s in the reference's
    format, 's d p<hex>', 's u' or 's rA-B'.  block = m > 1 runs tsfactor's
    blocked DDF (m degrees per step: one modmul and m*m squarings); `sched`
    picks the interval schedule (make_sched)."""
    from ._lib import ScanResult
    q = make_sched(sched, q0=q0, G=G, rho=rho, qcap=qcap)
    s = np.ascontiguousarray(np.asarray(survivors, dtype=np.uint64))
    n = s.size
    res = (ScanResult * n)()
    masks = np.zeros((n, mask_cap_words), dtype=np.uint64)
    call("gf2e_scan_sched", r, s.ctypes.data, n, k0, maxd, C.byref(q), L0, Lmax, batch, block,
         res, masks.ctypes.data, mask_cap_words, _sp(stream))
    out = []
    for i in range(n):
        R = res[i]
        if R.status == 1:
            out.append(f"{R.s} {R.d} p{_hex(masks[i, :R.mask_words])}")
        elif R.status == 2:
            out.append(f"{R.s} u")
        else:
            out.append(f"{R.s} r{R.rlo}-{R.rhi}")
    return out


class Scanner:
    """The steppable deep-scan engine (gf2e_scanner_*): submit s values, step
    degrees, poll finished result lines (the reference's line format)."""

    def __init__(self, r: int, slots: int = 64, block: int = 1, mask_cap_words: int = 1024):
        h = C.c_void_p()
        call("gf2e_scanner_create_blocked", r, slots, block, C.byref(h))
        self.h, self.cap = h.value, mask_cap_words

    def submit(self, s_values, k0: int, maxd: int, L0: int = 64, Lmax: int = 4096, tag0: int = 0):
        s = np.ascontiguousarray(np.asarray(s_values, dtype=np.uint64))
        call("gf2e_scanner_submit", self.h, s.ctypes.data, s.size, k0, maxd, L0, Lmax, tag0)

    def step(self, degrees: int = 256, stream=None):
        call("gf2e_scanner_step", self.h, degrees, _sp(stream))

    def poll(self, n: int = 64) -> list:
        """[(s, line)] of the s values finished since the last poll."""
        from ._lib import ScanResult
        res = (ScanResult * n)()
        tags = np.zeros(n, dtype=np.uint64)
        masks = np.zeros((n, self.cap), dtype=np.uint64)
        out, got = [], C.c_int()
        while True:
            call("gf2e_scanner_poll", self.h, res, tags.ctypes.data, masks.ctypes.data, self.cap,
                 n, C.byref(got))
            for i in range(got.value):
                R = res[i]
                if R.status == 1:
                    line = f"{R.s} {R.d} p{_hex(masks[i, :R.mask_words])}"
                elif R.status == 2:
                    line = f"{R.s} u"
                else:
                    line = f"{R.s} r{R.rlo}-{R.rhi}"
                out.append((int(R.s), line))
            if got.value < n:
                return out

    def gcd_time(self):
        g, t = C.c_uint64(), C.c_double()
        call("gf2e_scanner_gcd_time", self.h, C.byref(g), C.byref(t))
        return g.value, t.value

    def pairs(self) -> int:
        p = C.c_uint64()
        call("gf2e_scanner_status", self.h, None, None, None, C.byref(p))
        return p.value

    def close(self):
        if self.h:
            lib().gf2e_scanner_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def resolve_factor(g_words, kmin: int, kmax: int, cap: int = 1024):
    """(d, mask words) of the least-degree, then least, factor of g with
    degree in [kmin, kmax] (host computation on a small gcd)."""
    g = np.ascontiguousarray(np.asarray(g_words, dtype=np.uint64))
    d = C.c_uint64()
    mw = C.c_size_t()
    mask = np.zeros(cap, dtype=np.uint64)
    call("gf2e_resolve_factor", g.ctypes.data, g.size, kmin, kmax, C.byref(d), mask.ctypes.data,
         cap, C.byref(mw))
    return int(d.value), mask[: mw.value].copy()


# ========================================================== trinomial arithmetic
def spread32(v: int) -> int:
    """Interleave zeros (gf2_trinomial_cuda.h:22-30); host helper."""
    x = v & 0xFFFFFFFF
    out = 0
    for i in range(32):
        out |= ((x >> i) & 1) << (2 * i)
    return out


def trin_square(in_dev, out_dev, r: int, s: int, stream=None) -> None:
    call("gf2e_trin_square", _ptr(in_dev), _ptr(out_dev), r, s, _sp(stream))


def trin_square_batch(states, scratch, stride_words: int, nstates: int, r: int, s_dev, k: int,
                      stream=None) -> None:
    call("gf2e_trin_square_batch", _ptr(states), _ptr(scratch), stride_words, nstates, r,
         _ptr(s_dev), k, _sp(stream))


def squarings_per_pass(r: int, stride_words: int, nstates: int) -> int:
    """Squarings one pass of trin_square_batch performs (2 where the fused
    F -> F^4 pass applies and pays, else 1)."""
    return int(lib().gf2e_trin_squarings_per_pass(r, stride_words, nstates))


def frobenius_host(r: int, s_values, k: int, out: Optional[np.ndarray] = None,
                   stream=None) -> np.ndarray:
    """F_k = x^(2^k) mod x^r + x^s + 1 for every s, host in / host out
    (trinomial_stage2 run's .fk for many s at once).  `out` may be a pinned
    (n, stride) uint64 array; a fresh (n, nw) array is returned otherwise."""
    s = np.ascontiguousarray(np.asarray(s_values, dtype=np.uint64))
    nw = bits_to_words(r)
    if out is None:
        out = np.empty((s.size, nw), dtype=np.uint64)
    call("gf2e_trin_frobenius_host", r, s.ctypes.data, s.size, k, out.ctypes.data,
         out.shape[1] if out.ndim == 2 else nw, _sp(stream))
    return out


def trin_set_x(states, stride_words: int, nstates: int, r: int, stream=None) -> None:
    call("gf2e_trin_set_x", _ptr(states), stride_words, nstates, r, _sp(stream))


def trin_set_one(states, stride_words: int, nstates: int, r: int, stream=None) -> None:
    call("gf2e_trin_set_one", _ptr(states), stride_words, nstates, r, _sp(stream))


def trin_reduce(prod, prod_bits: int, out, r: int, s: int, stream=None) -> None:
    call("gf2e_trin_reduce", _ptr(prod), prod_bits, _ptr(out), r, s, _sp(stream))


class TrinGPU:
    """gf2_trinomial_cuda.h:87-178 over the C ABI."""

    def __init__(self):
        self._h = None

    def init(self, r: int) -> None:
        h = C.c_void_p()
        call("gf2e_trin_create", r, C.byref(h))
        self._h = h.value
        self.r = r
        self.s = 0
        a, acc, t0 = C.c_void_p(), C.c_void_p(), C.c_void_p()
        nw, m = C.c_size_t(), C.c_int()
        call("gf2e_trin_buffers", self._h, C.byref(a), C.byref(acc), C.byref(t0), C.byref(nw),
             C.byref(m))
        self.dA, self.dACC, self.dT0 = a.value, acc.value, t0.value
        self.nw, self.m = nw.value, m.value
        self.nw2 = 2 * self.nw

    def set_s(self, s: int) -> None:
        call("gf2e_trin_set_s", self._h, s)
        self.s = s

    def set_x(self, stream=None) -> None:
        call("gf2e_trin_reset_A", self._h, _sp(stream))

    def reset_acc(self, stream=None) -> None:
        call("gf2e_trin_reset_acc", self._h, _sp(stream))

    def square_A(self, stream=None) -> None:
        call("gf2e_trin_square_A", self._h, _sp(stream))

    def mul_dev(self, x, y, stream=None) -> None:
        call("gf2e_trin_mul_dev", self._h, _ptr(x), _ptr(y), _sp(stream))

    def reduce(self, dst, L: int, stream=None) -> None:
        call("gf2e_trin_reduce_T0", self._h, _ptr(dst), L, _sp(stream))

    def accumulate(self, stream=None) -> None:
        call("gf2e_trin_accumulate", self._h, _sp(stream))

    def read(self, which: str = "A", stream=None) -> np.ndarray:
        ptr = {"A": self.dA, "ACC": self.dACC, "T0": self.dT0}[which]
        n = self.nw if which != "T0" else 2 * self.nw + 2
        out = np.empty(n, dtype=np.uint64)
        call("gf2e_copy_to_host", out.ctypes.data, ptr, out.nbytes, _sp(stream))
        return out

    def write(self, which: str, words: np.ndarray, stream=None) -> None:
        ptr = {"A": self.dA, "ACC": self.dACC}[which]
        w = np.ascontiguousarray(words, dtype=np.uint64)[: self.nw]
        call("gf2e_copy_to_device", ptr, w.ctypes.data, w.nbytes, _sp(stream))

    def fini(self) -> None:
        if self._h:
            lib().gf2e_trin_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.fini()
        except Exception:
            pass
