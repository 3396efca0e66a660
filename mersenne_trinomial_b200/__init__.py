"""B200-native engine for the smallest irreducible factor of x^r + x^s + 1
over GF(2): Zech-log sieve, trinomial squaring/fold, Cantor additive-FFT
multiplication, GPU gcd and the batched deep scan, as sm_100a kernels behind
the C ABI in include/gf2e.h."""
from ._lib import Gf2eError, lib  # noqa: F401
from . import engine  # noqa: F401
from .engine import (  # noqa: F401
    CantorBasis, CudaFFT, DeviceBuffer, TrinGPU, bits_to_words, cert_lines, fmt_line,
    frobenius_host, gcd_batch, gcd_large, gf2x_fft_mul, gf2x_fft_mul_dev, mul_batch_dev, mul_out_words,
    primitive_poly, resolve_factor, run_sieve, scan, sieve_device, spread32, stream_sync,
    trin_reduce, trin_set_one, trin_set_x, trin_square, trin_square_batch,
)

__all__ = [
    "Gf2eError", "lib", "engine", "CantorBasis", "CudaFFT", "DeviceBuffer", "TrinGPU",
    "bits_to_words", "cert_lines", "fmt_line", "frobenius_host", "gcd_batch", "gcd_large", "gf2x_fft_mul",
    "gf2x_fft_mul_dev", "mul_batch_dev", "mul_out_words", "primitive_poly", "resolve_factor",
    "run_sieve", "scan", "sieve_device", "spread32", "stream_sync", "trin_reduce",
    "trin_set_one", "trin_set_x", "trin_square", "trin_square_batch",
]
