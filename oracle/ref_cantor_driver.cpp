// ref_cantor_driver.cpp -- TEST INFRASTRUCTURE ONLY.
//
// A thin C-ABI shim around the reference's own host engine
// (gf2_cantor_engine.h, included from the reference tree at build time by
// oracle/build_ref.sh; nothing of the reference is copied here).  The
// resulting oracle/_ref/libref_cantor.so lets the tests compare the CUDA
// engine and the C restatement with the reference's gf2x_fft_mul
// (gf2_cantor_engine.h:207-242), CantorBasis (:74-121) and CantorFFT
// (:125-188) on identical inputs.
#include "gf2_cantor_engine.h"

extern "C" {

int ref_basis(u64 *out64) {
    CantorBasis B;
    B.build();
    if (!B.verify()) return -1;
    for (int i = 0; i < B.len; i++) out64[i] = B.b[i];
    return B.len;
}

// out: mul_out_words(abits, bbits) words
int ref_fft_mul(const u64 *a, u64 abits, const u64 *b, u64 bbits, u64 *out) {
    CantorBasis B;
    B.build();
    if (!B.verify()) return -1;
    gf2x_fft_mul(a, abits, b, bbits, out, B);
    return 0;
}

int ref_fft_fwd(u64 *f, int m) {
    CantorBasis B;
    B.build();
    CantorFFT F;
    F.init(m, B);
    F.fwd(f);
    return 0;
}

int ref_fft_inv(u64 *f, int m) {
    CantorBasis B;
    B.build();
    CantorFFT F;
    F.init(m, B);
    F.inv(f);
    return 0;
}

int ref_twiddles(int m, u64 *W) {
    CantorBasis B;
    B.build();
    CantorFFT F;
    F.init(m, B);
    for (size_t t = 0; t < F.W.size(); t++) W[t] = F.W[t];
    return (int)F.W.size();
}

u64 ref_gf64_mul(u64 a, u64 b) { return gf64_mul(a, b); }

}  // extern "C"
