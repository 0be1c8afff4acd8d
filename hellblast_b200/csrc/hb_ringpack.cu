// Pair-packed ring FFTs (FP32) for the ring pairs of HEALPix-type grids.
//
// Replaces, for these pairs, the per-ring cp.fft.fft / cp.fft.ifft loops of the reference
// (sht_raw.py:38-43, sht_fallback.py:51-55, isht.py:16-24, spin.py:46-53,107-108).
//
// Which pairs: both rings (north r_N and its mirror r_S, or an unpaired ring alone) have the
// same even nphi = n and the same phi0 = s pi / n for an integer s, and the transform length
// L (n itself when n is a power of two, else the Bluestein length 2^ceil(log2(2n - 1))) lies in
// [512, 16384].  On a HEALPix grid that is the whole equatorial belt (n = 4 nside, s = 0 or 1
// alternating; with the reference's phi0 convention s = 1 or 2) and every polar ring from
// ring index 64 on (n = 4i, s = 1).  Everything else (the smallest polar rings, generic grids,
// FP64) runs in hb_fft.cu.  Bluestein rings with n = 4q and L = 2^13 or 2^14 (polar rings 513 to
// 2047) run split in four quarter-length transforms (ring_quad_*_kernel, below).
//
// Bluestein (n not a power of two): the length-n DFT X_j = c_j sum_k (x_k c_k) b_{j-k},
// c_t = exp(-i pi t^2 / n), b_t = conj c_t, is a circular convolution of length L >= 2n - 1:
// x c (zero-padded), forward FFT_L, times the chirp spectrum FFT_L(b) / L (natural order), inverse
// FFT_L, times c.  The synthesis runs the inverse DFT as conj(DFT(conj Z)).  One FP32 table per
// distinct n in the geometry holds the chirp spectrum (L entries) followed by c_t (t < L/2,
// FP64-computed from t^2 mod 2n, zero from n on).  n <= L/2 (n is even and 2n - 1 <= L), so the
// forward FFT's input is zero from L/2 on and only the inverse FFT's outputs below L/2 are used:
// its first pass reads 8 of the 16 points of each butterfly and its last pass computes and
// writes 8.  The chirp products ride in the analysis's first pass (ring times c) and in the
// synthesis's last pass (output times c); the chirp-spectrum product is a separate step over
// the shared buffer (fused into a pass, its 16 global loads per thread spill registers).
//
// Grid: (pair, map), so the CTAs in flight work on runs of neighbouring pairs of one map and
// their strided 16-byte coefficient accesses fill whole sectors of the m-major G / F, except for
// the Bluestein pairs of the synthesis and of the m-blocked analysis (fg_off; one CTA fills each
// 128-byte line there): (map, pair), so all maps of a pair run together and read that pair's
// tables once from DRAM.  Measured at nside 2048, 64 maps: the Bluestein synthesis 2.5 ms faster
// per direction this way; the m-major analysis 2.1 ms slower, the m-blocked one 2.5 ms faster.
//
// Packing: the two real rings of a pair form one complex sequence z_j = f_N[j] + i f_S[j],
// j < n, transformed by one complex FFT of length n.  Synthesis builds the spectrum Z of z from
// the two rings' folded Fourier coefficients and writes Re z to the north ring and Im z to the
// south ring; analysis splits the spectrum of z into the two rings' spectra,
// D_N[k] = (Z[k] + conj Z[n-k]) / 2 and D_S[k] = (Z[k] - conj Z[n-k]) / (2i).  No untangling
// step and no per-ring second pass: one FFT per pair and map.
//
// phi0 phase and alias fold (the reference has neither, sht_raw.py:41,51): harmonic m lands on
// bin m mod n and its conjugate on bin -m mod n; with phi0 = s pi / n,
// exp(i m phi0) = exp(i pi s k / n) (-1)^(s j) for m = k + j n, so every residue class k of
// m mod n takes one phase product and alternating signs over its aliases.
//
// FFT: Stockham autosort, compile-time length L = n = 2^LOGL, radix 16 for every pass but the
// second, which takes the remaining 2^(LOGL mod 4).  Pass with radix R after sub-transforms of
// length NS: butterfly b (j = b mod NS) reads points b + t L/R, multiplies point t by
// W_L^(j t L/(NS R)), transforms, and writes point q to (b - j) R + j + q NS.  Every thread
// holds 16 points per pass (one radix-16 butterfly, or 16/R small ones), so the transform runs
// in place in one shared buffer: all loads of a pass, a barrier, then the stores.  Natural order
// in and out: the analysis's first pass reads the two rings straight from global memory and the
// synthesis's last pass writes them (both coalesced, lanes on consecutive pixels).  Twiddles come
// from direct tables of W_L^e and W_L^(4e), the phi0 phases from products of two entries of a
// fine and a coarse table; both are FP64-computed once per geometry and copied into every CTA's
// shared memory (PkTab).
#include <algorithm>
#include <cmath>
#include <type_traits>
#include <vector>

#include "hb_internal.cuh"
#include "hb_fftcore.cuh"
#include "hb_tc.cuh"

namespace hb {

// shared-buffer index of FFT point i: one pad entry per 16 keeps the radix-R strided stores of
// the first passes on distinct banks
__device__ __forceinline__ int pk_pad(int i) { return i + (i >> 4); }

template <int LOGL> struct PkCfg {
    static constexpr int L = 1 << LOGL;
    static constexpr int NT = L / 16;                                // threads: 16 points each
    static constexpr int R1 = (LOGL & 3) ? (1 << (LOGL & 3)) : 16;   // radix of pass 1
    static constexpr int NPASS = (LOGL >> 2) + ((LOGL & 3) ? 1 : 0);
    static constexpr int BUF = L + (L >> 4);
    static constexpr int TW = L / 16;        // twiddle entries W_L^e and W_L^(4e), e < L/16
    static constexpr int TWP = TW + TW / 16; // ... stored at e + e/16 (pk_pad), see PkTab
    static constexpr int TWS = R1 < 16 ? 16 * R1 : 0;  // pass-1 twiddles W_(16 R1)^(j t), j < 16, t < R1
    static constexpr int PHC = 2 * L / 64;   // coarse phase entries exp(i pi 64 c / n), 2n <= 2L
    static constexpr int TWB = 2 * TWP + TWS;  // twiddle part of the table block
    static constexpr int TAB = TWB + 64 + PHC; // table block: twiddles, then phases
    static constexpr int SMEM = (BUF + TAB) * (int)sizeof(float2);
    static constexpr int MINB = 65536 / (NT * 64) > 0 ? 65536 / (NT * 64) : 1;  // <= 64 registers
};

template <int LOGL, int P> struct PkPass {
    static constexpr int R = P == 1 ? PkCfg<LOGL>::R1 : 16;
    static constexpr int NS = P == 0 ? 1 : (P == 1 ? 16 : 16 * PkCfg<LOGL>::R1 * (1 << (4 * (P - 2))));
};

struct PkTab {
    // radix-16 passes: the butterfly exponent e = j L / (16 NS) < L/16 indexes tw1 = W_L^e and
    // tw4 = W_L^(4e) directly (entry e at pk_pad(e): the middle passes' exponents step by 16,
    // which would put a half-warp on one bank); the other powers are their products (at most
    // three products deep)
    const float2 *tw1, *tw4;
    const float2 *tws;        // pass 1 of radix R1 < 16 (NS = 16): W_(16 R1)^(j t) at tws[j R1 + t]
    const float2 *phf, *phc;  // exp(i pi e / n) = phf[e & 63] phc[e >> 6], e < 2n
    __device__ __forceinline__ float2 ph(int e) const { return cmul(phf[e & 63], phc[e >> 6]); }
};

// Entry i of the table block of transform length L = 2^LOGL (FP64-computed, rounded to FP32):
// tw1 and tw4 (entry e at pk_pad(e); slot 16 of every 17, which pk_pad skips, holds zero), the
// pass-1 table, then the phase block for ring length n (pk_phase_entry).  Built once per geometry
// (build_pk_tables); every CTA copies its block into shared memory (pk_tables).
__device__ __forceinline__ float2 pk_phase_entry(int i, int n) {  // exp(i pi e / n): e = i < 64, or 64 (i - 64)
    double sn, cs;
    sincospi((double)(i < 64 ? i : 64 * (i - 64)) / (double)n, &sn, &cs);
    return make_float2((float)cs, (float)sn);
}
template <int LOGL> __device__ __forceinline__ float2 pk_table_entry(int i, int n) {
    using C = PkCfg<LOGL>;
    double sn = 0.0, cs = 0.0;
    if (i < 2 * C::TWP) {  // W_L^e (first block), W_L^(4e) (second)
        const int slot = i % C::TWP, r = slot % 17;
        if (r == 16) return make_float2(0.f, 0.f);
        const int e = 16 * (slot / 17) + r;
        sincospi(-2.0 * (double)(i < C::TWP ? e : 4 * e) / (double)C::L, &sn, &cs);
    } else if (i < C::TWB) {  // W_(16 R1)^(j t)
        const int j = (i - 2 * C::TWP) / C::R1, t = (i - 2 * C::TWP) % C::R1;
        sincospi(-2.0 * (double)(j * t) / (double)(16 * C::R1), &sn, &cs);
    } else {
        return pk_phase_entry(i - C::TWB, n);
    }
    return make_float2((float)cs, (float)sn);
}

// the CTA's table block: the twiddles of length L from gtw (the geometry's block for L), the
// phases exp(i pi e / n) from gph (a Bluestein ring's phase block) or, for n = L, from gtw
__device__ __forceinline__ float2 pk_ld(const float2 *p) { return __ldg(p); }
template <int LOGL>
__device__ __forceinline__ PkTab pk_tables(float2 *base, const float2 *__restrict__ gtw, const float2 *__restrict__ gph) {
    using C = PkCfg<LOGL>;
    float2 *tw1 = base, *tw4 = tw1 + C::TWP, *tws = tw4 + C::TWP, *phf = tws + C::TWS, *phc = phf + 64;
    for (int i = threadIdx.x; i < C::TAB; i += C::NT) base[i] = pk_ld((gph && i >= C::TWB) ? gph + (i - C::TWB) : gtw + i);
    return {tw1, tw4, tws, phf, phc};
}

// points t = 1 .. R-1 of a radix-R butterfly with exponent e (radix 16) or pass-1 row j (R < 16)
// times W_L^(e t) (conjugate for INV)
template <int R, bool INV>
__device__ __forceinline__ void pk_twiddle(float2 *v, int e, int j, const PkTab &T) {
    auto app = [&](int q, float2 w) { v[q] = cmul(v[q], INV ? cconj(w) : w); };
    if constexpr (R == 16) {
        const float2 w1 = T.tw1[pk_pad(e)], w4 = T.tw4[pk_pad(e)];
        const float2 w2 = cmul(w1, w1), w8 = cmul(w4, w4);
        const float2 w3 = cmul(w1, w2), w5 = cmul(w4, w1), w6 = cmul(w4, w2), w7 = cmul(w4, w3);
        app(1, w1); app(2, w2); app(3, w3); app(4, w4); app(5, w5); app(6, w6); app(7, w7); app(8, w8);
        app(9, cmul(w8, w1)); app(10, cmul(w8, w2)); app(11, cmul(w8, w3)); app(12, cmul(w8, w4));
        app(13, cmul(w8, w5)); app(14, cmul(w8, w6)); app(15, cmul(w8, w7));
    } else {
#pragma unroll
        for (int t = 1; t < R; ++t) app(t, T.tws[j * R + t]);
    }
}

// One Stockham pass (see the file comment).  `ld(i, ip)` / `st(i, ip, v)` read and write point i
// of the pass's input and output, ip = pk_pad(i) its shared-buffer slot (base plus compile-time
// offsets: every stride here is a multiple of 16).  The barrier between all loads and all
// stores makes the in-place update over one shared buffer safe.  HIN (first pass only): input
// points from L/2 on are zero and are not read.  HOUT (last pass only): output points from L/2
// on are neither computed nor written.
template <int LOGL, int P, bool INV, bool HIN, bool HOUT, class Ld, class St>
__device__ __forceinline__ void pk_pass(const PkTab &T, int tid, Ld &&ld, St &&st) {
    using C = PkCfg<LOGL>;
    constexpr int L = C::L, NT = C::NT, R = PkPass<LOGL, P>::R, NS = PkPass<LOGL, P>::NS, G = 16 / R;
    static_assert(!HIN || (P == 0 && R == 16), "half input: the first pass, radix 16");
    static_assert(!HOUT || (P == C::NPASS - 1 && R == 16 && NS == L / 16), "half output: the last pass, radix 16");
    static_assert((L / R) % 16 == 0 && NT % 16 == 0 && (NS == 1 || NS % 16 == 0) && (NS > 1 || R == 16),
                  "padded offsets are base plus constants");
    constexpr int LS = L / R + L / R / 16, US = NT + NT / 16, QS = NS == 1 ? 1 : NS + NS / 16;
    const int tp = pk_pad(tid);
    float2 x[16];
#pragma unroll
    for (int u = 0; u < G; ++u) {
        const int b = tid + u * NT, bp = tp + u * US;
#pragma unroll
        for (int t = 0; t < R; ++t)
            if (!HIN || t < R / 2) x[u * R + t] = ld(b + t * (L / R), bp + t * LS);
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < G; ++u) {
        const int b = tid + u * NT;
        const int j = b & (NS - 1);
        float2 *v = x + u * R;
        if constexpr (NS > 1) pk_twiddle<R, INV>(v, j * (L / (NS * R)), j, T);
        if constexpr (HIN)
            dft16<INV, true>(v);
        else
            dftR<R, INV>(v);
        const int base = (b - j) * R + j;
        const int basep = NS == 1 ? 17 * b : pk_pad(base);  // NS == 1: base = 16 b, slot 17 b
#pragma unroll
        for (int q = 0; q < R; ++q)
            if (!HOUT || q < R / 2) st(base + q * NS, basep + q * QS, v[q]);
    }
}

// passes P .. NPASS-1; pass 0 reads through ld0 (HIN: half input), the last pass writes through
// stl (HOUT: half output), the others go through the shared buffer.  tid: the thread's index
// among the L/16 threads of this transform (every thread of the CTA reaches the barriers)
template <int LOGL, bool INV, bool HIN, bool HOUT, int P = 0, class Ld0, class StL>
__device__ __forceinline__ void pk_run(float2 *buf, const PkTab &T, int tid, Ld0 &&ld0, StL &&stl) {
    constexpr int NP = PkCfg<LOGL>::NPASS;
    static_assert(NP >= 3, "pair-packed lengths have at least three passes");
    auto lds = [&](int, int ip) -> float2 { return buf[ip]; };
    auto sts = [&](int, int ip, float2 v) { buf[ip] = v; };
    if constexpr (P == NP - 1) {
        pk_pass<LOGL, P, INV, false, HOUT>(T, tid, lds, stl);
    } else {
        if constexpr (P == 0)
            pk_pass<LOGL, P, INV, HIN, false>(T, tid, ld0, sts);
        else
            pk_pass<LOGL, P, INV, false, false>(T, tid, lds, sts);
        __syncthreads();
        pk_run<LOGL, INV, HIN, HOUT, P + 1>(buf, T, tid, ld0, stl);
    }
}

// phi0 / pi * n as the integer s mod 2n (the host admitted only pairs where it is an integer)
__device__ __forceinline__ int pk_shift(double phi0_pi, int n) {
    long long s = llrint(phi0_pi * (double)n) % (2LL * n);
    return (int)(s < 0 ? s + 2LL * n : s);
}

__device__ __forceinline__ float2 f4lo(float4 v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 f4hi(float4 v) { return make_float2(v.z, v.w); }

// x mod m for 0 <= x < 2^31 and 256 <= m < 2^16: the float quotient estimate is off by at most
// one either way (relative error 2^-23 of a quotient below 2^23 / 256), one correction each way
struct PkMod {
    int m;
    float inv;
    __device__ __forceinline__ int operator()(int x) const {
        const int q = (int)((float)x * inv);
        int r = x - q * m;
        r += r < 0 ? m : 0;
        r -= r >= m ? m : 0;
        return r;
    }
};

// Spectrum points k and n - k of z = f_N + i f_S from the class sums S(k), S(n - k) of the north
// and south rings (ph = exp(i pi s k / n), sg = (-1)^s):
// X(k) = ph (S(k) + sg conj S(n-k)), X(n-k) = conj(ph) (sg S(n-k) + conj S(k)), put as X_N + i X_S
__device__ __forceinline__ void pk_pair_values(float sg, float2 ph, float2 SkN, float2 SkS, float2 SmN, float2 SmS,
                                               float2 &xk, float2 &xnk) {
    const float2 xkN = cmul(ph, make_float2(SkN.x + sg * SmN.x, SkN.y - sg * SmN.y));
    const float2 xkS = cmul(ph, make_float2(SkS.x + sg * SmS.x, SkS.y - sg * SmS.y));
    const float2 xcN = cmul(cconj(ph), make_float2(sg * SmN.x + SkN.x, sg * SmN.y - SkN.y));
    const float2 xcS = cmul(cconj(ph), make_float2(sg * SmS.x + SkS.x, sg * SmS.y - SkS.y));
    xk = make_float2(xkN.x - xkS.y, xkN.y + xkS.x);
    xnk = make_float2(xcN.x - xcS.y, xcN.y + xcS.x);
}
template <class Put>
__device__ __forceinline__ void pk_put_pair(int k, int n, float sg, float2 ph, float2 SkN, float2 SkS, float2 SmN,
                                            float2 SmS, Put &&put) {
    float2 xk, xnk;
    pk_pair_values(sg, ph, SkN, SkS, SmN, SmS, xk, xnk);
    put(k, xk);
    put(n - k, xnk);
}

// class sums S(k) = sum_j (-1)^(s j) chalf G(k + j n) over the orders m = k + j n <= mmax, north (a)
// and south (c)
template <class Ld>
__device__ __forceinline__ void pk_csum(int k, int n, int s, int mmax, float chalf, Ld &&ld, float2 &a, float2 &c) {
    a = make_float2(0.f, 0.f);
    c = a;
    float sj = 1.f;
    for (int m = k; m <= mmax; m += n) {
        const float4 v = ld(m);
        a.x += sj * v.x; a.y += sj * v.y;
        c.x += sj * v.z; c.y += sj * v.w;
        if (s & 1) sj = -sj;
    }
    a = cscale(a, chalf);
    c = cscale(c, chalf);
}

// The spectrum Z of z = f_N + i f_S from the two rings' coefficients G(m) (ld(m): the float4
// (north, south) of order m <= mmax): alias fold by m mod n, the phi0 phase exp(i pi s k / n) and
// (-1)^(s j) over the aliases m = k + j n; put(k, Z_k) for every k < n (CTA-strided loops of NT
// threads).  c_m = 1 for m = 0, dbl for m > 0.  P2: n is a power of two.
template <int NT, bool P2, class Ld, class Put>
__device__ __forceinline__ void pk_fold(int n, int s, int mmax, float dbl, const PkTab &T, Ld &&ld, Put &&put) {
    const float chalf = 0.5f * dbl;
    const float sg = (s & 1) ? -1.f : 1.f;
    const PkMod mod2n{2 * n, 1.f / (float)(2 * n)};
    // phase-table index of exp(i pi s k / n): (s k) mod 2n (s k < 2^31: s < 2n <= 2^15, k <= n)
    auto pidx = [&](int k) -> int { return P2 ? ((s * k) & (2 * n - 1)) : mod2n(s * k); };
    auto csum = [&](int k, float2 &a, float2 &c) { pk_csum(k, n, s, mmax, chalf, ld, a, c); };
    auto put_pair = [&](int k, float2 SkN, float2 SkS, float2 SmN, float2 SmS) {
        pk_put_pair(k, n, sg, T.ph(pidx(k)), SkN, SkS, SmN, SmS, put);
    };
    if (mmax < n) {  // at most one harmonic per residue class (the equatorial belt when mmax < 4 nside)
#pragma unroll 4
        for (int k = threadIdx.x + 1; k < n / 2; k += NT) {
            const float4 a = k <= mmax ? ld(k) : make_float4(0.f, 0.f, 0.f, 0.f);
            const float4 c = n - k <= mmax ? ld(n - k) : make_float4(0.f, 0.f, 0.f, 0.f);
            put_pair(k, cscale(f4lo(a), chalf), cscale(f4hi(a), chalf), cscale(f4lo(c), chalf),
                     cscale(f4hi(c), chalf));
        }
    } else {
        for (int k = threadIdx.x + 1; k < n / 2; k += NT) {
            float2 SkN, SkS, SmN, SmS;
            csum(k, SkN, SkS);
            csum(n - k, SmN, SmS);
            put_pair(k, SkN, SkS, SmN, SmS);
        }
    }
    if (threadIdx.x == 0) {  // bins 0 and n/2: c_m Re(G(m) exp(i m phi0)) of their classes
        float aN = 0.f, aS = 0.f, sj = 1.f;
        for (int m = 0; m <= mmax; m += n) {
            const float4 v = ld(m);
            const float c = m == 0 ? 1.f : dbl;
            aN += sj * c * v.x;
            aS += sj * c * v.z;
            if (s & 1) sj = -sj;
        }
        put(0, make_float2(aN, aS));
        float2 hN, hS;
        csum(n / 2, hN, hS);  // c/2 scaled: times 2 below
        const float2 ph = T.ph(pidx(n / 2));
        put(n / 2, make_float2(2.f * (ph.x * hN.x - ph.y * hN.y), 2.f * (ph.x * hS.x - ph.y * hS.y)));
    }
}

// ------------------------------------------------------------------------------ synthesis
// G[map][m][pair][side] (FP32 complex; one float4 = (north, south) per (m, pair)) -> the two
// rings of each pair.  c_m = 1 for m = 0 and `dbl` (2: real-field synthesis, 1: adjoint of the
// weighted analysis) for m > 0; apply_w multiplies ring r by scale 2 pi w_r / n (no 2 pi with
// HB_F_NO2PI).  BLU: n is not a power of two and L is its Bluestein length.
template <int LOGL, bool BLU>
__global__ void __launch_bounds__(PkCfg<LOGL>::NT, PkCfg<LOGL>::MINB)
    ring_pair_synthesis_kernel(GeomDev g, const int32_t *__restrict__ pairs, const float4 *__restrict__ Gm,
                               int64_t gm_stride4, int mmax, float *__restrict__ maps, int64_t map_stride,
                               const double *__restrict__ w, int apply_w, int mdouble, int flags) {
    using C = PkCfg<LOGL>;
    constexpr int L = C::L, NT = C::NT;
    extern __shared__ __align__(16) float2 pk_smem[];
    float2 *buf = pk_smem;
    const int pair = pairs[BLU ? blockIdx.y : blockIdx.x], bm = BLU ? blockIdx.x : blockIdx.y;
    const int rN = g.pair_ring[2 * pair], rS = g.pair_ring[2 * pair + 1];
    const int n = BLU ? g.nphi[rN] : L;
    // Bluestein tables: chirp spectrum bt[0, L), chirp ch[t] = exp(-i pi t^2 / n) for t < n, then
    // the ring's phase block
    const float2 *bt = BLU ? g.pkb_bt + g.pkb_bt_ofs[pair] : nullptr, *ch = BLU ? bt + L : nullptr;
    const PkTab T = pk_tables<LOGL>(pk_smem + C::BUF, g.pk_tw + g.pk_tw_ofs[LOGL], BLU ? bt + L + L / 2 : nullptr);
    const int s = (flags & HB_F_NOPHASE) ? 0 : pk_shift(g.phi0_pi[rN], n);
    const int64_t np = g.npairs;
    const float4 *gin = Gm + bm * gm_stride4 + pair;  // (m, pair) entry at gin[m * np]
    const float dbl = mdouble ? 2.f : 1.f;
    const bool hasS = rS >= 0;
    __syncthreads();  // tables
    // spectrum point k of z: stored as is (direct) or as conj(Z[k]) c_k (Bluestein)
    auto put = [&](int k, float2 z) { buf[pk_pad(k)] = BLU ? cmul(cconj(z), __ldg(ch + k)) : z; };
    // an unpaired ring's south slot is not read as data: zeros keep the imaginary half finite.
    // ld.global.cg: the 16-byte G reads at the order stride are used once per CTA (the other half
    // of each sector by the neighbouring pair's CTA, from L2); measured 0.26 ms faster per
    // synthesis at nside 2048, 64 maps than the read-only path through L1
    auto ld = [&](int m) -> float4 {
        float4 v = __ldcg(gin + (int64_t)m * np);
        if (!hasS) v.z = v.w = 0.f;
        return v;
    };
    pk_fold<NT, !BLU>(n, s, mmax, dbl, T, ld, put);
    if (BLU)  // zero padding of the convolution (the first pass reads points below L/2 only)
        for (int k = n + threadIdx.x; k < L / 2; k += NT) buf[pk_pad(k)] = make_float2(0.f, 0.f);
    __syncthreads();
    const double sc2 = (flags & HB_F_NO2PI) ? 1.0 : 6.283185307179586476925286766559;
    const float psN = apply_w ? (float)(sc2 * w[rN] / (double)n) : 1.f;
    const float psS = (apply_w && hasS) ? (float)(sc2 * w[rS] / (double)n) : 1.f;
    float *fN = maps + bm * map_stride + g.ofs[rN];
    float *fS = hasS ? maps + bm * map_stride + g.ofs[rS] : nullptr;
    auto lds = [&](int, int ip) -> float2 { return buf[ip]; };
    if constexpr (!BLU) {
        pk_run<LOGL, true, false, false>(buf, T, threadIdx.x, lds, [&](int i, int, float2 v) {
            fN[i] = v.x * psN;
            if (fS) fS[i] = v.y * psS;
        });
    } else {
        // forward FFT_L (input zero from L/2 on), times the chirp spectrum
        pk_run<LOGL, false, true, false>(buf, T, threadIdx.x, lds, [&](int, int ip, float2 v) { buf[ip] = v; });
        __syncthreads();
        for (int i = threadIdx.x; i < L; i += NT) buf[pk_pad(i)] = cmul(buf[pk_pad(i)], __ldg(bt + i));
        __syncthreads();
        // inverse FFT_L, points below L/2 only; times the chirp, conjugated, to the two rings
        pk_run<LOGL, true, false, true>(buf, T, threadIdx.x, lds, [&](int i, int, float2 v) {
            if (i < n) {
                const float2 z = cconj(cmul(__ldg(ch + i), v));
                fN[i] = z.x * psN;
                if (fS) fS[i] = z.y * psS;
            }
        });
    }
}

// The orders of the two rings from the spectrum Z of z = f_N + i f_S (Zf(k), k < n):
// D_N = (Z[k] + conj Z[n-k]) / 2 and D_S = (Z[k] - conj Z[n-k]) / (2 i), times exp(-i pi s k / n)
// and the ring scales scN / scS, stored through at(m) for every m <= mlim of residue class k
// ((-1)^(s j) over the aliases m = k + j n) and, conjugated, of class n - k; c_m = 2 for m > 0
// with mdouble; the orders mlim < m <= mmax are zero.  CTA-strided loops of NT threads; P2: n is
// a power of two.
template <int NT, bool P2, class Zfn, class At>
__device__ __forceinline__ void pk_emit(int n, int s, int mmax, int mlim, bool mdouble, float scN, float scS,
                                        const PkTab &T, Zfn &&Zf, At &&at) {
    const PkMod mod2n{2 * n, 1.f / (float)(2 * n)};
    auto pidx = [&](int k) -> int { return P2 ? ((s * k) & (2 * n - 1)) : mod2n(s * k); };
    // HB_F_NOFOLD: the orders the ring does not resolve (m >= n) are zero, not left unwritten
    for (int m = mlim + 1 + threadIdx.x; m <= mmax; m += NT) at(m) = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int k = threadIdx.x; k <= n / 2; k += NT) {
        const float2 zk = Zf(k), zc = k == 0 ? zk : Zf(n - k);
        // D_N = (Z[k] + conj Z[n-k]) / 2, D_S = (Z[k] - conj Z[n-k]) / (2 i)
        const float2 dN = make_float2(0.5f * (zk.x + zc.x), 0.5f * (zk.y - zc.y));
        const float2 dS = make_float2(0.5f * (zk.y + zc.y), -0.5f * (zk.x - zc.x));
        const float2 ph = cconj(T.ph(pidx(k)));
        const float2 yN = cscale(cmul(ph, dN), scN), yS = cscale(cmul(ph, dS), scS);
        float sj = 1.f;
        for (int m = k; m <= mlim; m += n) {  // class k: (-1)^(s j) Y
            const float c = (mdouble && m > 0) ? 2.f * sj : sj;
            at(m) = make_float4(c * yN.x, c * yN.y, c * yS.x, c * yS.y);
            if (s & 1) sj = -sj;
        }
        if (k > 0 && 2 * k < n) {  // class n - k: (-1)^(s (j + 1)) conj Y
            sj = (s & 1) ? -1.f : 1.f;
            for (int m = n - k; m <= mlim; m += n) {
                const float c = mdouble ? 2.f * sj : sj;
                at(m) = make_float4(c * yN.x, -c * yN.y, c * yS.x, -c * yS.y);
                if (s & 1) sj = -sj;
            }
        }
    }
}

// ------------------------------------------------------------------------------ analysis
// the two rings of each pair -> F[map][m][pair][side] (m-major, or blocked by 8 orders with
// mblk: fg_off), F(m) = c_m scale exp(-i m phi0) D[m mod n] (conjugated above n/2);
// scale = 2 pi w_r / n (1 with unit_w; no 2 pi with HB_F_NO2PI); c_m = 2 for m > 0 with mdouble
// (adjoint of the synthesis), else 1; HB_F_NOFOLD keeps m < n.  Lanes take consecutive orders, so
// in the blocked layout 8 lanes fill one 128-byte line.
template <int LOGL, bool BLU>
__global__ void __launch_bounds__(PkCfg<LOGL>::NT, PkCfg<LOGL>::MINB)
    ring_pair_analysis_kernel(GeomDev g, const int32_t *__restrict__ pairs, const float *__restrict__ maps,
                              int64_t map_stride, const double *__restrict__ w, float4 *__restrict__ Fm,
                              int64_t fm_stride4, int mmax, int flags, int unit_w, int mdouble, int mblk) {
    using C = PkCfg<LOGL>;
    constexpr int L = C::L, NT = C::NT;
    extern __shared__ __align__(16) float2 pk_smem[];
    float2 *buf = pk_smem;
    const bool mf = BLU && mblk;
    const int pair = pairs[mf ? blockIdx.y : blockIdx.x], bm = mf ? blockIdx.x : blockIdx.y;
    const int rN = g.pair_ring[2 * pair], rS = g.pair_ring[2 * pair + 1];
    const int n = BLU ? g.nphi[rN] : L;
    // Bluestein tables: chirp spectrum bt[0, L), chirp ch[t] = exp(-i pi t^2 / n) for t < n, then
    // the ring's phase block
    const float2 *bt = BLU ? g.pkb_bt + g.pkb_bt_ofs[pair] : nullptr, *ch = BLU ? bt + L : nullptr;
    const PkTab T = pk_tables<LOGL>(pk_smem + C::BUF, g.pk_tw + g.pk_tw_ofs[LOGL], BLU ? bt + L + L / 2 : nullptr);
    const int s = (flags & HB_F_NOPHASE) ? 0 : pk_shift(g.phi0_pi[rN], n);
    const int64_t np = g.npairs;
    const float *fN = maps + bm * map_stride + g.ofs[rN];
    const float *fS = rS >= 0 ? maps + bm * map_stride + g.ofs[rS] : nullptr;
    auto sts = [&](int, int ip, float2 v) { buf[ip] = v; };
    auto ring = [&](int i, int = 0) -> float2 { return make_float2(__ldg(fN + i), fS ? __ldg(fS + i) : 0.f); };
    __syncthreads();  // tables
    if constexpr (!BLU) {
        pk_run<LOGL, false, false, false>(buf, T, threadIdx.x, ring, sts);
    } else {
        // forward FFT_L of the chirped ring (zero from n on; read below L/2 only), times the chirp
        // spectrum; inverse FFT_L, points below L/2 only
        auto lds = [&](int, int ip) -> float2 { return buf[ip]; };
        auto ld0 = [&](int i, int) -> float2 { return i < n ? cmul(ring(i), __ldg(ch + i)) : make_float2(0.f, 0.f); };
        pk_run<LOGL, false, true, false>(buf, T, threadIdx.x, ld0, sts);
        __syncthreads();
        for (int i = threadIdx.x; i < L; i += NT) buf[pk_pad(i)] = cmul(buf[pk_pad(i)], __ldg(bt + i));
        __syncthreads();
        pk_run<LOGL, true, false, true>(buf, T, threadIdx.x, lds, sts);
    }
    __syncthreads();
    auto Zf = [&](int k) -> float2 { return BLU ? cmul(__ldg(ch + k), buf[pk_pad(k)]) : buf[pk_pad(k)]; };
    const double sc2 = (flags & HB_F_NO2PI) ? 1.0 : 6.283185307179586476925286766559;
    const float scN = unit_w ? 1.f : (float)(sc2 * w[rN] / (double)n);
    const float scS = rS < 0 ? 0.f : (unit_w ? 1.f : (float)(sc2 * w[rS] / (double)n));
    const int mlim = (flags & HB_F_NOFOLD) ? min(mmax, n - 1) : mmax;
    float4 *out = Fm + bm * fm_stride4;
    auto at = [&](int m) -> float4 & { return out[fg_off(m, pair, np, mblk != 0)]; };
    pk_emit<NT, !BLU>(n, s, mmax, mlim, mdouble != 0, scN, scS, T, Zf, at);
}

// ------------------------------------------------------------------------ quad-split Bluestein
// Ring length n = 4 q (HEALPix polar rings: n = 4 i) that is not a power of two and whose
// Bluestein length for the whole ring would be 2^13 or 2^14: radix-4 Cooley-Tukey turns the
// length-n DFT into four length-q DFTs, and each of those runs as a Bluestein convolution of
// length LQ = 2^LOGQ >= 2q - 1 (a quarter of the whole ring's L), all four side by side in one
// CTA: four groups of LQ/16 threads, one sub-buffer each.  With Y = conj Z (synthesis, the
// inverse DFT as conj(DFT(conj Z))) and W_n = exp(-2 pi i / n):
//   synthesis (decimation of the output): y_{4a+b} = sum_r W_q^(a r) V^b_r,
//     V^b_r = W_n^(b r) sum_t Y_(r+qt) (-i)^(b t);
//   analysis (decimation of the input): U^b = DFT_q(z_(4a+b)),
//     Z_(k+qt) = sum_b (-i)^(b t) W_n^(b k) U^b_k.
// Each length-LQ transform takes 3 passes (LOGQ = 11, 12) where the whole ring's takes 4, and the
// chirp spectrum (LQ entries) fits in shared memory beside the buffers, so its product rides in
// the forward transform's last pass.  The radix-4 steps are one extra exchange through the
// shared buffer each (natural order <-> the four sub-buffers).  Per-ring table (pkb_bt): the
// length-q chirp spectrum (LQ), the length-q chirp c_t = exp(-i pi t^2 / q) (t < LQ/2, zero from
// q on), then the phase block of n with 4 LQ / 64 coarse entries (2n <= 4 LQ).
template <int LOGQ> struct QkCfg {
    using S = PkCfg<LOGQ>;
    static constexpr int LQ = S::L, NTQ = S::NT, NT = 4 * NTQ;
    static constexpr int SBUF = S::BUF, BUF = 4 * SBUF;  // four sub-buffers
    static constexpr int PHC = 4 * LQ / 64;              // coarse phases exp(i pi 64 c / n), 2n <= 4 LQ
    static constexpr int TAB = S::TWB + 64 + PHC;        // twiddles of LQ, then the phases of n
    static constexpr int ALL = TAB + 3 * LQ / 2;         // + the chirp spectrum (LQ) and the chirp (LQ/2)
    static constexpr int SMEM = (BUF + ALL) * (int)sizeof(float2);
    static constexpr int KPT = LQ / NT;                  // spectrum bins k < n/2 < LQ per thread (fold)
    static constexpr int MINB = 65536 / (NT * 64) > 0 ? 65536 / (NT * 64) : 1;  // <= 64 registers
    static constexpr int RPT = (LQ / 2) / NT;            // radix-4 steps: residues r < LQ/2 per thread
    static_assert(NT <= 1024 && RPT * NT == LQ / 2, "one CTA of four sub-transforms");
    static_assert(LQ / 2 + (LQ - 1) / 16 < SBUF, "upper half-buffers hold q <= LQ/2 spectrum points each");
    static_assert(BUF % 2 == 0 && S::TWB % 2 == 0 && TAB % 2 == 0 && KPT * NT == LQ,
                  "16-byte cp.async chunks never straddle two table parts");
};

// the CTA's tables, copied asynchronously (16-byte cp.async, one commit group; the caller waits):
// twiddles of LQ (gtw), the phase block of n (gph), then the chirp spectrum and the chirp (gbt,
// 3 LQ / 2 entries back to back).  Every part has an even entry count and starts 16-byte aligned
// in global memory (even table offsets) and in shared memory (BUF, TWB and TAB are even).
template <int LOGQ>
__device__ __forceinline__ PkTab qk_tables_async(float2 *base, const float2 *__restrict__ gtw,
                                                 const float2 *__restrict__ gph, const float2 *__restrict__ gbt) {
    using C = QkCfg<LOGQ>;
    using S = PkCfg<LOGQ>;
    for (int c = threadIdx.x; c < C::ALL / 2; c += C::NT) {
        const int i = 2 * c;
        tc::cp_async16(base + i, i < S::TWB ? gtw + i : (i < C::TAB ? gph + (i - S::TWB) : gbt + (i - C::TAB)));
    }
    tc::cp_async_commit();
    float2 *tw1 = base, *tw4 = tw1 + S::TWP, *tws = tw4 + S::TWP, *phf = tws + S::TWS, *phc = phf + 64;
    return {tw1, tw4, tws, phf, phc};
}

// Slot of natural-order spectrum point k = j + q t (j < q, t < 4): the upper half of sub-buffer t,
// which the sub-transforms leave free (their inputs and outputs lie below LQ/2), so the radix-4
// steps read one half and write the other without a barrier in between
template <int LOGQ> __device__ __forceinline__ int qk_slot(int k, int q) {
    using C = QkCfg<LOGQ>;
    const int t = (k >= q) + (k >= 2 * q) + (k >= 3 * q);
    return t * C::SBUF + pk_pad(C::LQ / 2 + k - t * q);
}

// W_n^(b r) for b = 1, 2, 3 (b r < 3n/4): w1 = conj exp(i pi 2r / n), w2 = w1^2, w3 = w1 w2
__device__ __forceinline__ void qk_twiddles(const PkTab &T, int r, float2 &w1, float2 &w2, float2 &w3) {
    w1 = cconj(T.ph(2 * r));
    w2 = cmul(w1, w1);
    w3 = cmul(w1, w2);
}

template <int LOGQ>
__global__ void __launch_bounds__(QkCfg<LOGQ>::NT, QkCfg<LOGQ>::MINB)
    ring_quad_synthesis_kernel(GeomDev g, const int32_t *__restrict__ pairs, const float4 *__restrict__ Gm,
                               int64_t gm_stride4, int mmax, float *__restrict__ maps, int64_t map_stride,
                               const double *__restrict__ w, int apply_w, int mdouble, int flags) {
    using C = QkCfg<LOGQ>;
    constexpr int LQ = C::LQ, NTQ = C::NTQ, NT = C::NT, SB = C::SBUF;
    extern __shared__ __align__(16) float2 pk_smem[];
    float2 *buf = pk_smem;
    const float2 *spec = pk_smem + C::BUF + C::TAB, *chs = spec + LQ;  // chirp spectrum, chirp
    const int pair = pairs[blockIdx.y], bm = blockIdx.x;  // (map, pair): the maps of a pair share its tables
    const int rN = g.pair_ring[2 * pair], rS = g.pair_ring[2 * pair + 1];
    const int n = g.nphi[rN], q = n >> 2;
    const float2 *bt = g.pkb_bt + g.pkb_bt_ofs[pair];
    const PkTab T = qk_tables_async<LOGQ>(pk_smem + C::BUF, g.pk_tw + g.pk_tw_ofs[LOGQ], bt + LQ + LQ / 2, bt);
    const int s = (flags & HB_F_NOPHASE) ? 0 : pk_shift(g.phi0_pi[rN], n);
    const int64_t np = g.npairs;
    const float4 *gin = Gm + bm * gm_stride4 + pair;
    const bool hasS = rS >= 0;
    auto ld = [&](int m) -> float4 {  // ld.global.cg as in ring_pair_synthesis_kernel
        float4 v = __ldcg(gin + (int64_t)m * np);
        if (!hasS) v.z = v.w = 0.f;
        return v;
    };
    auto put = [&](int k, float2 z) { buf[qk_slot<LOGQ>(k, q)] = cconj(z); };  // conj Z, point k at qk_slot(k)
    const float dbl = mdouble ? 2.f : 1.f;
    if (mmax < n) {
        // at most one order per residue class: this thread's orders are loaded while the tables
        // arrive.  Bins k = tid + 1 + j NT < n/2 take G(k) and G(n - k); the last thread's last
        // slot (k = LQ > n/2) carries bins 0 and n/2 instead: G(0) and G(n/2).
        const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
        const bool last = threadIdx.x == NT - 1;
        float4 ga[C::KPT], gc[C::KPT];
#pragma unroll
        for (int j = 0; j < C::KPT; ++j) {
            const int k = threadIdx.x + 1 + j * NT;
            const bool in = k < n / 2;
            ga[j] = (in && k <= mmax) ? ld(k) : z4;
            gc[j] = (in && n - k <= mmax) ? ld(n - k) : z4;
        }
        if (last) {
            ga[C::KPT - 1] = ld(0);
            gc[C::KPT - 1] = n / 2 <= mmax ? ld(n / 2) : z4;
        }
        tc::cp_async_wait<0>();
        __syncthreads();  // tables
        const float chalf = 0.5f * dbl, sg = (s & 1) ? -1.f : 1.f;
        const PkMod mod2n{2 * n, 1.f / (float)(2 * n)};
#pragma unroll
        for (int j = 0; j < C::KPT; ++j) {
            const int k = threadIdx.x + 1 + j * NT;
            if (k < n / 2)
                pk_put_pair(k, n, sg, T.ph(mod2n(s * k)), cscale(f4lo(ga[j]), chalf), cscale(f4hi(ga[j]), chalf),
                            cscale(f4lo(gc[j]), chalf), cscale(f4hi(gc[j]), chalf), put);
        }
        if (last) {  // bin 0: Re G(0) (c_0 = 1); bin n/2: c Re(G(n/2) exp(i pi s / 2))
            const float4 v0 = ga[C::KPT - 1], vh = gc[C::KPT - 1];
            put(0, make_float2(v0.x, v0.z));
            const float2 ph = T.ph(mod2n(s * (n / 2)));
            put(n / 2, make_float2(dbl * (ph.x * vh.x - ph.y * vh.y), dbl * (ph.x * vh.z - ph.y * vh.w)));
        }
    } else {
        tc::cp_async_wait<0>();
        __syncthreads();  // tables
        pk_fold<NT, false>(n, s, mmax, dbl, T, ld, put);
    }
    __syncthreads();
    // radix-4 step: V^b_r c_r into sub-buffer b at r (zero for q <= r < LQ/2)
#pragma unroll
    for (int u = 0; u < C::RPT; ++u) {
        const int r = threadIdx.x + u * NT, rp = pk_pad(r);
        if (r < q) {
            const int zp = pk_pad(LQ / 2 + r);
            float2 x0 = buf[zp], x1 = buf[SB + zp], x2 = buf[2 * SB + zp], x3 = buf[3 * SB + zp];
            dft4<false>(x0, x1, x2, x3);
            float2 w1, w2, w3;
            qk_twiddles(T, r, w1, w2, w3);
            const float2 c = chs[r];
            buf[rp] = cmul(x0, c);
            buf[SB + rp] = cmul(x1, cmul(w1, c));
            buf[2 * SB + rp] = cmul(x2, cmul(w2, c));
            buf[3 * SB + rp] = cmul(x3, cmul(w3, c));
        } else {
            buf[rp] = buf[SB + rp] = buf[2 * SB + rp] = buf[3 * SB + rp] = make_float2(0.f, 0.f);
        }
    }
    __syncthreads();
    const int grp = threadIdx.x / NTQ, tq = threadIdx.x % NTQ;
    float2 *sb = buf + grp * SB;
    auto lds = [&](int, int ip) -> float2 { return sb[ip]; };
    // forward FFT_LQ (input zero from LQ/2 on), times the chirp spectrum in its last pass
    pk_run<LOGQ, false, true, false>(sb, T, tq, lds, [&](int k, int ip, float2 v) { sb[ip] = cmul(v, spec[k]); });
    __syncthreads();
    const double sc2 = (flags & HB_F_NO2PI) ? 1.0 : 6.283185307179586476925286766559;
    const float psN = apply_w ? (float)(sc2 * w[rN] / (double)n) : 1.f;
    const float psS = (apply_w && hasS) ? (float)(sc2 * w[rS] / (double)n) : 1.f;
    float *fN = maps + bm * map_stride + g.ofs[rN];
    float *fS = hasS ? maps + bm * map_stride + g.ofs[rS] : nullptr;
    // inverse FFT_LQ, points below LQ/2, into the sub-buffers
    pk_run<LOGQ, true, false, true>(sb, T, tq, lds, [&](int, int ip, float2 v) { sb[ip] = v; });
    __syncthreads();
    // output a of sub-transform b, conj(c_a v), is pixel 4a + b: one thread writes pixels
    // 4a .. 4a+3 of both rings (16-byte stores where the rings start 16-byte aligned)
    const bool vec = ((reinterpret_cast<uintptr_t>(fN) | reinterpret_cast<uintptr_t>(fS)) & 15) == 0;
    for (int a = threadIdx.x; a < q; a += NT) {
        const float2 c = chs[a];
        const int ap = pk_pad(a);
        float2 z[4];
#pragma unroll
        for (int b = 0; b < 4; ++b) z[b] = cconj(cmul(c, buf[b * SB + ap]));
        const float4 oN = make_float4(z[0].x * psN, z[1].x * psN, z[2].x * psN, z[3].x * psN);
        const float4 oS = make_float4(z[0].y * psS, z[1].y * psS, z[2].y * psS, z[3].y * psS);
        if (vec) {
            *reinterpret_cast<float4 *>(fN + 4 * a) = oN;
            if (fS) *reinterpret_cast<float4 *>(fS + 4 * a) = oS;
        } else {
            fN[4 * a] = oN.x; fN[4 * a + 1] = oN.y; fN[4 * a + 2] = oN.z; fN[4 * a + 3] = oN.w;
            if (fS) { fS[4 * a] = oS.x; fS[4 * a + 1] = oS.y; fS[4 * a + 2] = oS.z; fS[4 * a + 3] = oS.w; }
        }
    }
}

template <int LOGQ>
__global__ void __launch_bounds__(QkCfg<LOGQ>::NT, QkCfg<LOGQ>::MINB)
    ring_quad_analysis_kernel(GeomDev g, const int32_t *__restrict__ pairs, const float *__restrict__ maps,
                              int64_t map_stride, const double *__restrict__ w, float4 *__restrict__ Fm,
                              int64_t fm_stride4, int mmax, int flags, int unit_w, int mdouble, int mblk) {
    using C = QkCfg<LOGQ>;
    constexpr int LQ = C::LQ, NTQ = C::NTQ, NT = C::NT, SB = C::SBUF;
    extern __shared__ __align__(16) float2 pk_smem[];
    float2 *buf = pk_smem;
    const float2 *spec = pk_smem + C::BUF + C::TAB, *chs = spec + LQ;  // chirp spectrum, chirp
    const int pair = pairs[mblk ? blockIdx.y : blockIdx.x], bm = mblk ? blockIdx.x : blockIdx.y;
    const int rN = g.pair_ring[2 * pair], rS = g.pair_ring[2 * pair + 1];
    const int n = g.nphi[rN], q = n >> 2;
    const float2 *bt = g.pkb_bt + g.pkb_bt_ofs[pair], *ch = bt + LQ;
    const PkTab T = qk_tables_async<LOGQ>(pk_smem + C::BUF, g.pk_tw + g.pk_tw_ofs[LOGQ], bt + LQ + LQ / 2, bt);
    const int s = (flags & HB_F_NOPHASE) ? 0 : pk_shift(g.phi0_pi[rN], n);
    const int64_t np = g.npairs;
    const int grp = threadIdx.x / NTQ, tq = threadIdx.x % NTQ;
    const float *fN = maps + bm * map_stride + g.ofs[rN];
    const float *fS = rS >= 0 ? maps + bm * map_stride + g.ofs[rS] : nullptr;
    float2 *sb = buf + grp * SB;
    auto lds = [&](int, int ip) -> float2 { return sb[ip]; };
    auto sts = [&](int, int ip, float2 v) { sb[ip] = v; };
    // sub-sequence b: samples 4a + b times the chirp c_a into sub-buffer b at a (a < q; zero from q
    // to LQ/2).  One thread reads pixels 4a .. 4a+3 of both rings (16-byte loads where the rings
    // start 16-byte aligned) and the chirp from global memory, while the tables arrive.
    const bool vec = ((reinterpret_cast<uintptr_t>(fN) | reinterpret_cast<uintptr_t>(fS)) & 15) == 0;
    auto ld4 = [&](const float *f, int a) -> float4 {
        if (!f) return make_float4(0.f, 0.f, 0.f, 0.f);
        if (vec) return __ldg(reinterpret_cast<const float4 *>(f + 4 * a));
        return make_float4(__ldg(f + 4 * a), __ldg(f + 4 * a + 1), __ldg(f + 4 * a + 2), __ldg(f + 4 * a + 3));
    };
#pragma unroll
    for (int u = 0; u < C::RPT; ++u) {
        const int a = threadIdx.x + u * NT, ap = pk_pad(a);
        if (a < q) {
            const float4 xN = ld4(fN, a), xS = ld4(fS, a);
            const float2 c = __ldg(ch + a);
            buf[ap] = cmul(make_float2(xN.x, xS.x), c);
            buf[SB + ap] = cmul(make_float2(xN.y, xS.y), c);
            buf[2 * SB + ap] = cmul(make_float2(xN.z, xS.z), c);
            buf[3 * SB + ap] = cmul(make_float2(xN.w, xS.w), c);
        } else {
            buf[ap] = buf[SB + ap] = buf[2 * SB + ap] = buf[3 * SB + ap] = make_float2(0.f, 0.f);
        }
    }
    tc::cp_async_wait<0>();
    __syncthreads();  // samples and tables
    // forward FFT_LQ times the chirp spectrum, inverse FFT_LQ (points below LQ/2)
    pk_run<LOGQ, false, true, false>(sb, T, tq, lds, [&](int k, int ip, float2 v) { sb[ip] = cmul(v, spec[k]); });
    __syncthreads();
    pk_run<LOGQ, true, false, true>(sb, T, tq, lds, sts);
    __syncthreads();
    // radix-4 step: U^b_k = c_k (sub-buffer b at k); Z_(k+qt) = sum_b (-i)^(b t) W_n^(b k) U^b_k
    // to qk_slot(k + q t)
#pragma unroll
    for (int u = 0; u < C::RPT; ++u) {
        const int k = threadIdx.x + u * NT;
        if (k < q) {
            const int kp = pk_pad(k), zp = pk_pad(LQ / 2 + k);
            float2 w1, w2, w3;
            qk_twiddles(T, k, w1, w2, w3);
            const float2 c = chs[k];
            float2 x0 = cmul(buf[kp], c), x1 = cmul(buf[SB + kp], cmul(w1, c));
            float2 x2 = cmul(buf[2 * SB + kp], cmul(w2, c)), x3 = cmul(buf[3 * SB + kp], cmul(w3, c));
            dft4<false>(x0, x1, x2, x3);
            buf[zp] = x0;
            buf[SB + zp] = x1;
            buf[2 * SB + zp] = x2;
            buf[3 * SB + zp] = x3;
        }
    }
    __syncthreads();
    const double sc2 = (flags & HB_F_NO2PI) ? 1.0 : 6.283185307179586476925286766559;
    const float scN = unit_w ? 1.f : (float)(sc2 * w[rN] / (double)n);
    const float scS = rS < 0 ? 0.f : (unit_w ? 1.f : (float)(sc2 * w[rS] / (double)n));
    const int mlim = (flags & HB_F_NOFOLD) ? min(mmax, n - 1) : mmax;
    float4 *out = Fm + bm * fm_stride4;
    auto at = [&](int m) -> float4 & { return out[fg_off(m, pair, np, mblk != 0)]; };
    pk_emit<NT, false>(n, s, mmax, mlim, mdouble != 0, scN, scS, T, [&](int k) { return buf[qk_slot<LOGQ>(k, q)]; },
                       at);
}

// ------------------------------------------------------------------------------ host side
static int pk_log2(int64_t v) {
    int lg = 0;
    while ((int64_t(1) << lg) < v) ++lg;
    return lg;
}

// The pairs these kernels take (see the file comment).  *logL: log2 of the transform length;
// *blu: whether it is a Bluestein pair.
bool pk_pair_ok(int nphiN, int nphiS, double phi0N, double phi0S, int *logL, bool *blu) {
    if (nphiN <= 0 || (nphiN & 1)) return false;
    if (nphiS >= 0 && (nphiS != nphiN || phi0S != phi0N)) return false;
    const double s = phi0N * (double)nphiN;  // phi0 / pi * n
    if (std::fabs(s - std::nearbyint(s)) > 1e-9) return false;
    const bool p2 = (nphiN & (nphiN - 1)) == 0;
    const int lg = p2 ? pk_log2(nphiN) : pk_log2(2 * (int64_t)nphiN - 1);
    if (lg < PK_MIN_LOG || lg > PK_MAX_LOG) return false;
    *logL = lg;
    *blu = !p2;
    return true;
}

// log2 of the sub-transform length LQ when a Bluestein pair of ring length n (whole-ring length
// 2^logL) runs as four quarter-length convolutions (see the quad-split kernels), else 0: n a
// multiple of 4 and 2^logL = 2^13 or 2^14, where the quarter length saves a pass
int pk_quad_log(int n, int logL) {
    if ((n & 3) || (n & (n - 1)) == 0 || (logL != 13 && logL != 14)) return 0;
    const int lq = pk_log2(2 * (int64_t)(n / 4) - 1);
    return (lq == logL - 2) ? lq : 0;
}

template <int LOGL, bool BLU> static int pk_prepare() {
    static bool done = false;
    if (!done) {
        HB_CUDA_TRY(cudaFuncSetAttribute(ring_pair_synthesis_kernel<LOGL, BLU>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, PkCfg<LOGL>::SMEM));
        HB_CUDA_TRY(cudaFuncSetAttribute(ring_pair_analysis_kernel<LOGL, BLU>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, PkCfg<LOGL>::SMEM));
        done = true;
    }
    return HB_OK;
}

struct PkSynArgs {
    int nmaps;
    const float2 *Gm;
    int mmax;
    float *maps;
    int64_t map_stride;
    const double *w;
    bool apply_w, mdouble;
    int flags;
};
struct PkAnaArgs {
    int nmaps;
    const float *maps;
    int64_t map_stride;
    const double *w;
    float2 *Fm;
    int mmax, flags;
    bool unit_w, mdouble, mblk;
};

// (pair, map) grid, or (map, pair) with MAP_FAST (Bluestein pairs: the synthesis and the m-blocked
// analysis; see the file comment)
template <bool MAP_FAST> static int pk_grid(int64_t cnt, int nmaps, dim3 *grid) {
    const int64_t y = MAP_FAST ? cnt : nmaps;
    if (y > 65535 || cnt > INT32_MAX || nmaps <= 0)
        return fail(HB_ERR_UNSUPPORTED, "pair-packed ring FFT: more than 65535 pairs in a class or maps in a batch");
    *grid = MAP_FAST ? dim3((unsigned)nmaps, (unsigned)cnt) : dim3((unsigned)cnt, (unsigned)nmaps);
    return HB_OK;
}

template <int LOGL, bool BLU>
static int pk_syn_one(const GeomDev &g, const int32_t *pairs, int64_t cnt, const PkSynArgs &a, cudaStream_t st) {
    int rc = pk_prepare<LOGL, BLU>();
    dim3 grid;
    if (!rc) rc = pk_grid<BLU>(cnt, a.nmaps, &grid);
    if (rc) return rc;
    const int64_t gm4 = (int64_t)(a.mmax + 1) * g.npairs;
    ring_pair_synthesis_kernel<LOGL, BLU><<<grid, PkCfg<LOGL>::NT, PkCfg<LOGL>::SMEM, st>>>(
        g, pairs, reinterpret_cast<const float4 *>(a.Gm), gm4, a.mmax, a.maps, a.map_stride, a.w, a.apply_w ? 1 : 0,
        a.mdouble ? 1 : 0, a.flags);
    HB_CHECK_LAUNCH();
    return HB_OK;
}

template <int LOGL, bool BLU>
static int pk_ana_one(const GeomDev &g, const int32_t *pairs, int64_t cnt, const PkAnaArgs &a, cudaStream_t st) {
    int rc = pk_prepare<LOGL, BLU>();
    dim3 grid;
    if (!rc) rc = (BLU && a.mblk) ? pk_grid<true>(cnt, a.nmaps, &grid) : pk_grid<false>(cnt, a.nmaps, &grid);
    if (rc) return rc;
    const int64_t fm4 = fg_rows(a.mmax, a.mblk) * g.npairs;
    ring_pair_analysis_kernel<LOGL, BLU><<<grid, PkCfg<LOGL>::NT, PkCfg<LOGL>::SMEM, st>>>(
        g, pairs, a.maps, a.map_stride, a.w, reinterpret_cast<float4 *>(a.Fm), fm4, a.mmax, a.flags, a.unit_w ? 1 : 0,
        a.mdouble ? 1 : 0, a.mblk ? 1 : 0);
    HB_CHECK_LAUNCH();
    return HB_OK;
}

template <int LOGQ> static int qk_prepare() {
    static bool done = false;
    if (!done) {
        HB_CUDA_TRY(cudaFuncSetAttribute(ring_quad_synthesis_kernel<LOGQ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         QkCfg<LOGQ>::SMEM));
        HB_CUDA_TRY(cudaFuncSetAttribute(ring_quad_analysis_kernel<LOGQ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         QkCfg<LOGQ>::SMEM));
        done = true;
    }
    return HB_OK;
}

// quad-split pairs: (map, pair) grid for the synthesis and the m-blocked analysis, as the
// Bluestein pairs above
template <int LOGQ>
static int qk_syn_one(const GeomDev &g, const int32_t *pairs, int64_t cnt, const PkSynArgs &a, cudaStream_t st) {
    int rc = qk_prepare<LOGQ>();
    dim3 grid;
    if (!rc) rc = pk_grid<true>(cnt, a.nmaps, &grid);
    if (rc) return rc;
    const int64_t gm4 = (int64_t)(a.mmax + 1) * g.npairs;
    ring_quad_synthesis_kernel<LOGQ><<<grid, QkCfg<LOGQ>::NT, QkCfg<LOGQ>::SMEM, st>>>(
        g, pairs, reinterpret_cast<const float4 *>(a.Gm), gm4, a.mmax, a.maps, a.map_stride, a.w, a.apply_w ? 1 : 0,
        a.mdouble ? 1 : 0, a.flags);
    HB_CHECK_LAUNCH();
    return HB_OK;
}

template <int LOGQ>
static int qk_ana_one(const GeomDev &g, const int32_t *pairs, int64_t cnt, const PkAnaArgs &a, cudaStream_t st) {
    int rc = qk_prepare<LOGQ>();
    dim3 grid;
    if (!rc) rc = a.mblk ? pk_grid<true>(cnt, a.nmaps, &grid) : pk_grid<false>(cnt, a.nmaps, &grid);
    if (rc) return rc;
    const int64_t fm4 = fg_rows(a.mmax, a.mblk) * g.npairs;
    ring_quad_analysis_kernel<LOGQ><<<grid, QkCfg<LOGQ>::NT, QkCfg<LOGQ>::SMEM, st>>>(
        g, pairs, a.maps, a.map_stride, a.w, reinterpret_cast<float4 *>(a.Fm), fm4, a.mmax, a.flags, a.unit_w ? 1 : 0,
        a.mdouble ? 1 : 0, a.mblk ? 1 : 0);
    HB_CHECK_LAUNCH();
    return HB_OK;
}

template <class A>
static int qk_dispatch(const GeomDev &g, int logQ, const int32_t *pp, int64_t cnt, const A &a, cudaStream_t st) {
    constexpr bool SYN = std::is_same<A, PkSynArgs>::value;
    switch (logQ) {
#define HB_QK_CASE(LG) \
    case LG:           \
        if constexpr (SYN) return qk_syn_one<LG>(g, pp, cnt, a, st); else return qk_ana_one<LG>(g, pp, cnt, a, st);
        HB_QK_CASE(11) HB_QK_CASE(12)
#undef HB_QK_CASE
        default:
            return fail(HB_ERR_UNSUPPORTED, "pair-packed ring FFT: unsupported quad-split length class");
    }
}

template <bool BLU, class A>
static int pk_dispatch(const GeomDev &g, int logL, const int32_t *pp, int64_t cnt, const A &a, cudaStream_t st) {
    constexpr bool SYN = std::is_same<A, PkSynArgs>::value;
    switch (logL) {
#define HB_PK_CASE(LG) \
    case LG:           \
        if constexpr (SYN) return pk_syn_one<LG, BLU>(g, pp, cnt, a, st); else return pk_ana_one<LG, BLU>(g, pp, cnt, a, st);
        HB_PK_CASE(9) HB_PK_CASE(10) HB_PK_CASE(11) HB_PK_CASE(12) HB_PK_CASE(13) HB_PK_CASE(14)
#undef HB_PK_CASE
        default:
            return fail(HB_ERR_UNSUPPORTED, "pair-packed ring FFT: unsupported length class");
    }
}

template <class A> static int pk_all(const GeomDev &g, const A &a, cudaStream_t st) {
    for (int c = 0; c < g.pk_n_cls; ++c) {
        const int64_t first = g.pk_first[c], cnt = g.pk_first[c + 1] - first;
        if (cnt <= 0) continue;
        const int lg = g.pk_logn[c] & 0xff;
        const bool blu = (g.pk_logn[c] >> 8) & 1, quad = (g.pk_logn[c] >> 9) & 1;
        int rc = quad  ? qk_dispatch(g, lg, g.pk_pairs + first, cnt, a, st)
                 : blu ? pk_dispatch<true>(g, lg, g.pk_pairs + first, cnt, a, st)
                       : pk_dispatch<false>(g, lg, g.pk_pairs + first, cnt, a, st);
        if (rc) return rc;
    }
    return HB_OK;
}

int launch_pk_synthesis(const GeomDev &g, int nmaps, const float2 *Gm, int mmax, float *maps, int64_t map_stride,
                        const double *w, bool apply_w, bool mdouble, int flags, cudaStream_t st) {
    return pk_all(g, PkSynArgs{nmaps, Gm, mmax, maps, map_stride, w, apply_w, mdouble, flags}, st);
}

int launch_pk_analysis(const GeomDev &g, int nmaps, const float *maps, int64_t map_stride, const double *w,
                       float2 *Fm, int mmax, int flags, bool unit_w, bool mdouble, cudaStream_t st, bool mblk) {
    return pk_all(g, PkAnaArgs{nmaps, maps, map_stride, w, Fm, mmax, flags, unit_w, mdouble, mblk}, st);
}


// ------------------------------------------------------------------------------ table blocks
int64_t pk_tab_entries(int logL) {
    switch (logL) {
#define HB_PK_TAB(LG) \
    case LG:          \
        return PkCfg<LG>::TAB;
        HB_PK_TAB(9) HB_PK_TAB(10) HB_PK_TAB(11) HB_PK_TAB(12) HB_PK_TAB(13) HB_PK_TAB(14)
#undef HB_PK_TAB
        default:
            return 0;
    }
}
int64_t pk_phase_entries(int logL) { return 64 + 2 * (int64_t(1) << logL) / 64; }
// entries of a Bluestein pair's table in pkb_bt: chirp spectrum (L), chirp (L/2), phase block;
// even, so that every table starts 16-byte aligned
int64_t pk_bt_entries(int logL, bool quad) {
    const int64_t L = int64_t(1) << logL;
    return (3 * L / 2 + 64 + (quad ? 4 : 2) * L / 64 + 1) & ~int64_t(1);
}

template <int LOGL> __global__ void __launch_bounds__(256) pk_twtab_kernel(float2 *out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < PkCfg<LOGL>::TAB; i += gridDim.x * blockDim.x)
        out[i] = pk_table_entry<LOGL>(i, PkCfg<LOGL>::L);
}
// one CTA per Bluestein table: the phase block of its ring length rn[e] at ofs[e] + 3 L / 2 (L the
// chirp's transform length); 2 L / 64 coarse entries, 4 L / 64 for a quad-split ring
// (rn[e] = 4 ns[e], 2 rn <= 4 L)
__global__ void __launch_bounds__(256) pk_phtab_kernel(const int32_t *__restrict__ ns, const int32_t *__restrict__ rn,
                                                       const int32_t *__restrict__ logLs,
                                                       const int64_t *__restrict__ ofs, float2 *out) {
    const int e = blockIdx.x, n = rn[e], L = 1 << logLs[e];
    const int cnt = 64 + (n != ns[e] ? 4 : 2) * L / 64;
    float2 *dst = out + ofs[e] + 3 * (int64_t)L / 2;
    for (int i = threadIdx.x; i < cnt; i += blockDim.x) dst[i] = pk_phase_entry(i, n);
}

int build_pk_tables(const GeomDev &g, int count, const int32_t *ns, const int32_t *rn, const int32_t *logL,
                    const int64_t *ofs, cudaStream_t st) {
#define HB_PK_TW(LG)                                                                                   \
    pk_twtab_kernel<LG><<<(PkCfg<LG>::TAB + 255) / 256, 256, 0, st>>>(g.pk_tw + g.pk_tw_ofs[LG]); \
    HB_CHECK_LAUNCH();
    HB_PK_TW(9) HB_PK_TW(10) HB_PK_TW(11) HB_PK_TW(12) HB_PK_TW(13) HB_PK_TW(14)
#undef HB_PK_TW
    if (count > 0) {
        pk_phtab_kernel<<<count, 256, 0, st>>>(ns, rn, logL, ofs, g.pkb_bt);
        HB_CHECK_LAUNCH();
    }
    return HB_OK;
}

}  // namespace hb
