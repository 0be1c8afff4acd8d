// Register-level DFT building blocks shared by the ring-FFT kernels (hb_fft.cu, hb_ringpack.cu):
// radix-2/4/8/16 transforms of points held in registers, natural order in and out.
// INV = false: X_q = sum_t x_t exp(-2 pi i t q / R); INV = true: the conjugate kernel.
#pragma once
#include "hb_internal.cuh"

namespace hb {

// multiply by -i (forward) or +i (inverse)
template <bool INV, typename V> __device__ __forceinline__ V rot90(V a) {
    return INV ? mk2(-a.y, a.x) : mk2(a.y, -a.x);
}

template <bool INV, typename V> __device__ __forceinline__ void dft2(V *x) {
    const V a = x[0], b = x[1];
    x[0] = cadd(a, b);
    x[1] = csub(a, b);
}

template <bool INV, typename V> __device__ __forceinline__ void dft4(V &x0, V &x1, V &x2, V &x3) {
    const V a0 = cadd(x0, x2), a1 = csub(x0, x2), a2 = cadd(x1, x3), a3 = rot90<INV>(csub(x1, x3));
    x0 = cadd(a0, a2);
    x2 = csub(a0, a2);
    x1 = cadd(a1, a3);
    x3 = csub(a1, a3);
}

template <bool INV, typename V> __device__ __forceinline__ void dft4(V *x) { dft4<INV>(x[0], x[1], x[2], x[3]); }

template <bool INV, typename V> __device__ __forceinline__ void dft8(V *x) {
    using T = decltype(x[0].x);
    const T r = (T)0.70710678118654752440084436210484903928;
    V e0 = x[0], e1 = x[2], e2 = x[4], e3 = x[6];
    V o0 = x[1], o1 = x[3], o2 = x[5], o3 = x[7];
    dft4<INV>(e0, e1, e2, e3);
    dft4<INV>(o0, o1, o2, o3);
    // o_q *= w8^q, w8 = exp(-+ 2 pi i / 8)
    o1 = INV ? mk2(r * (o1.x - o1.y), r * (o1.x + o1.y)) : mk2(r * (o1.x + o1.y), r * (o1.y - o1.x));
    o2 = rot90<INV>(o2);
    o3 = INV ? mk2(-r * (o3.x + o3.y), r * (o3.x - o3.y)) : mk2(r * (o3.y - o3.x), -r * (o3.x + o3.y));
    x[0] = cadd(e0, o0);
    x[4] = csub(e0, o0);
    x[1] = cadd(e1, o1);
    x[5] = csub(e1, o1);
    x[2] = cadd(e2, o2);
    x[6] = csub(e2, o2);
    x[3] = cadd(e3, o3);
    x[7] = csub(e3, o3);
}

// x *= exp(-+ 2 pi i e / 16) for the constant exponents of the radix-16 butterfly
template <int E, bool INV, typename V> __device__ __forceinline__ V w16(V a) {
    using T = decltype(a.x);
    constexpr double C[10] = {1.0, 0.92387953251128675612818318939678828682, 0.70710678118654752440084436210484903928,
                              0.38268343236508977172845998403039886676, 0.0, -0.38268343236508977172845998403039886676,
                              -0.70710678118654752440084436210484903928, -0.92387953251128675612818318939678828682, -1.0,
                              -0.92387953251128675612818318939678828682};
    constexpr double S[10] = {0.0, 0.38268343236508977172845998403039886676, 0.70710678118654752440084436210484903928,
                              0.92387953251128675612818318939678828682, 1.0, 0.92387953251128675612818318939678828682,
                              0.70710678118654752440084436210484903928, 0.38268343236508977172845998403039886676, 0.0,
                              -0.38268343236508977172845998403039886676};
    if constexpr (E == 0) return a;
    else if constexpr (E == 4) return rot90<INV>(a);
    else {
        const T c = (T)C[E], s = INV ? (T)S[E] : (T)(-S[E]);  // (c, s) = cos - +i sin
        return mk2(a.x * c - a.y * s, a.x * s + a.y * c);
    }
}

// DFT-4 of (x0, x1, 0, 0): the two zero inputs are not added (x + 0 is not x for x = -0, so the
// compiler cannot drop those additions by itself)
template <bool INV, typename V> __device__ __forceinline__ void dft4_h(V &x0, V &x1, V &x2, V &x3) {
    const V a = x0, b = x1, rb = rot90<INV>(x1);
    x0 = cadd(a, b);
    x2 = csub(a, b);
    x1 = cadd(a, rb);
    x3 = csub(a, rb);
}

// 16-point DFT as 4 x 4: inner DFT-4 over n2 (n = n1 + 4 n2), twiddles W16^(n1 k2), outer
// DFT-4 over n1; X[4 k1 + k2] ends in register k1 + 4 k2 and is renamed into place.
// HALF: inputs 8 .. 15 are zero and are not read.
template <bool INV, bool HALF = false, typename V> __device__ __forceinline__ void dft16(V *x) {
#pragma unroll
    for (int n1 = 0; n1 < 4; ++n1) {
        if constexpr (HALF)
            dft4_h<INV>(x[n1], x[n1 + 4], x[n1 + 8], x[n1 + 12]);
        else
            dft4<INV>(x[n1], x[n1 + 4], x[n1 + 8], x[n1 + 12]);
    }
    x[5] = w16<1, INV>(x[5]);
    x[9] = w16<2, INV>(x[9]);
    x[13] = w16<3, INV>(x[13]);
    x[6] = w16<2, INV>(x[6]);
    x[10] = w16<4, INV>(x[10]);
    x[14] = w16<6, INV>(x[14]);
    x[7] = w16<3, INV>(x[7]);
    x[11] = w16<6, INV>(x[11]);
    x[15] = w16<9, INV>(x[15]);
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) dft4<INV>(x[4 * k2], x[4 * k2 + 1], x[4 * k2 + 2], x[4 * k2 + 3]);
    V y[16];
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1)
#pragma unroll
        for (int k2 = 0; k2 < 4; ++k2) y[4 * k1 + k2] = x[k1 + 4 * k2];
#pragma unroll
    for (int i = 0; i < 16; ++i) x[i] = y[i];
}

template <int R, bool INV, typename V> __device__ __forceinline__ void dftR(V *x) {
    if constexpr (R == 16)
        dft16<INV>(x);
    else if constexpr (R == 8)
        dft8<INV>(x);
    else if constexpr (R == 4)
        dft4<INV>(x);
    else
        dft2<INV>(x);
}

template <int R> struct Log2R {
    static constexpr int v = R == 16 ? 4 : (R == 8 ? 3 : (R == 4 ? 2 : 1));
};

}  // namespace hb
