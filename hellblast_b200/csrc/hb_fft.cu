// Ragged per-ring FFT kernels (analysis: ring samples -> F[m, pair, side]; synthesis: the
// reverse).
//
// Replaces the per-ring cp.fft.fft / cp.fft.ifft loops of the reference (sht_raw.py:38-43,
// sht_fallback.py:51-55, isht.py:16-24, spin.py:46-53,107-108), which launch one cuFFT per ring
// and sync on nphi per ring.  Ring r has nphi_r = 4i samples (polar caps) or 4*nside
// (equatorial belt).  A real ring of length n is packed into N = n/2 complex points
// z_j = f_2j + i f_2j+1; their DFT is a power-of-two FFT when N is a power of two and a
// Bluestein chirp-z transform (power-of-two convolution of length L >= 2N-1, chirp spectra
// precomputed per distinct N in the geometry) otherwise.
//
// Work decomposition: one CTA per (ring pair, map); it transforms the pair's north ring, then
// its south ring, in one shared-memory buffer, so the two halves of each F(m, pair) entry are
// written close together in time (and adjacent pairs run side by side), which lets L2 merge the
// partial sector writes.  Pairs are launched in classes of equal convolution length, each class
// with its own shared-memory size.
//
// FFT engine: in-place radix-8 stages (radix 4 or 2 for the last one) in shared memory.  The
// forward transform is decimation-in-frequency (natural order in, digit-reversed out), the
// inverse is its exact mirror, decimation-in-time (digit-reversed in, natural out), so no
// reordering pass exists.  Twiddles come from one table per geometry, W^j = exp(-2 pi i j/Lmax)
// for j < Lmax/2 (FP64-computed, rounded for FP32).  The per-m factors of the untangling
// (exp(-2 pi i k/n)), the ring phase (exp(-i m phi0)) and the Bluestein chirp
// (exp(-i pi q/N)) are products of two entries of small per-ring tables (64 fine steps x
// coarse steps), built per CTA with a few hundred FP64 sincospi.
//
// Fused into the m-major write (the reference has none of these, see sht_raw.py:41,51):
//   * the per-pixel quadrature weight 2*pi*w_r/nphi_r,
//   * the ring phase exp(-i m phi0_r),
//   * the aliasing fold: harmonic m lands on DFT bin m mod nphi (conjugated above nphi/2),
//     so every m <= mmax is produced, also on rings with nphi <= 2*mmax.
#include <algorithm>
#include <cmath>

#include "hb_internal.cuh"

namespace hb {

// ------------------------------------------------------------------------------ FFT engine
// Stage plan of a length-2^logL transform: logL / 3 radix-8 stages, then one radix-2^(logL % 3)
// stage.  Stage i works on sub-transforms of size S_i = 2^(logL - 3i).

// Digit reversal between frequency k and its position p in the forward transform's output:
// p holds k's base-8 digits (lowest first) from the top down, then k's top logL % 3 bits.
// Computed as a full bit reversal plus a fix-up that restores the bit order inside each digit.
__device__ __forceinline__ unsigned digit_fix(unsigned x, int logL) {
    const int n8 = logL / 3, rem = logL - 3 * n8;
    const unsigned low = (1u << (3 * n8)) - 1u;
    const unsigned g = x & low, hi = x & ~low;
    const unsigned m0 = 0x49249249u & low;
    const unsigned gf = (g & (m0 << 1)) | ((g & m0) << 2) | ((g & (m0 << 2)) >> 2);
    const unsigned hf = rem == 2 ? (((hi >> 1) & (1u << (3 * n8))) | ((hi << 1) & (2u << (3 * n8)))) : hi;
    return gf | hf;
}
__device__ __forceinline__ unsigned brev_n(unsigned x, int logL) { return logL ? __brev(x) >> (32 - logL) : 0u; }
__device__ __forceinline__ int freq_to_pos(int k, int logL) { return (int)brev_n(digit_fix((unsigned)k, logL), logL); }
__device__ __forceinline__ int pos_to_freq(int p, int logL) { return (int)digit_fix(brev_n((unsigned)p, logL), logL); }

// Shared-memory FFT buffers carry one pad element per 16: the late stages' strided accesses and
// the digit-reversed reads then spread over the banks.
template <bool PAD> __device__ __forceinline__ int ph(int i) { return PAD ? i + (i >> 4) : i; }
__host__ __device__ __forceinline__ int padded_len(int L) { return L + (L >> 4) + 1; }

template <typename T> struct Tw {
    using V = c2_t<T>;
    const V *tab;  // exp(-2 pi i j / 2^log_tw), j < 2^(log_tw - 1)
    int log_tw;
    // exp(-2 pi i e / 2^logS), 0 <= e < 2^logS <= 2^log_tw
    __device__ __forceinline__ V w(int e, int logS) const {
        const int j = e << (log_tw - logS);
        const int half = 1 << (log_tw - 1);
        const V v = tab[j & (half - 1)];
        return (j & half) ? mk2(-v.x, -v.y) : v;
    }
};

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

template <int R, bool INV, typename V> __device__ __forceinline__ void dftR(V *x) {
    if constexpr (R == 8)
        dft8<INV>(x);
    else if constexpr (R == 4)
        dft4<INV>(x);
    else
        dft2<INV>(x);
}

// x[q] *= W_S^(pos q) (conjugated for INV), q = 1 .. R-1; radix 8 loads W^pos, W^2pos, W^4pos
// and forms the other four by products (about two roundings more)
template <int R, bool INV, typename T>
__device__ __forceinline__ void twiddle_apply(c2_t<T> *x, const Tw<T> &tw, int pos, int logS) {
    using V = c2_t<T>;
    if constexpr (R == 8) {
        const V w1 = tw.w(pos, logS), w2 = tw.w(2 * pos, logS), w4 = tw.w(4 * pos, logS);
        const V w3 = cmul(w1, w2);
        V w[8] = {w1, w1, w2, w3, w4, cmul(w4, w1), cmul(w4, w2), cmul(w4, w3)};
#pragma unroll
        for (int q = 1; q < 8; ++q) x[q] = cmul(x[q], INV ? cconj(w[q]) : w[q]);
    } else {
#pragma unroll
        for (int q = 1; q < R; ++q) {
            const V wq = tw.w(pos * q, logS);
            x[q] = cmul(x[q], INV ? cconj(wq) : wq);
        }
    }
}

// one decimation-in-frequency stage of radix R on sub-transforms of size 2^logS
template <int R, bool PAD, typename T>
__device__ __forceinline__ void dif_stage(c2_t<T> *buf, const Tw<T> &tw, int logL, int logS) {
    using V = c2_t<T>;
    constexpr int logR = R == 8 ? 3 : (R == 4 ? 2 : 1);
    const int logh = logS - logR, h = 1 << logh;
    for (int b = threadIdx.x; b < (1 << (logL - logR)); b += blockDim.x) {
        const int pos = b & (h - 1);
        const int base = ((b >> logh) << logS) + pos;
        V x[R];
#pragma unroll
        for (int t = 0; t < R; ++t) x[t] = buf[ph<PAD>(base + (t << logh))];
        dftR<R, false>(x);
        twiddle_apply<R, false>(x, tw, pos, logS);
#pragma unroll
        for (int q = 0; q < R; ++q) buf[ph<PAD>(base + (q << logh))] = x[q];
    }
    __syncthreads();
}

// the exact inverse of dif_stage (times R): conjugate twiddles, then the inverse radix-R DFT
template <int R, bool PAD, typename T>
__device__ __forceinline__ void dit_inv_stage(c2_t<T> *buf, const Tw<T> &tw, int logL, int logS) {
    using V = c2_t<T>;
    constexpr int logR = R == 8 ? 3 : (R == 4 ? 2 : 1);
    const int logh = logS - logR, h = 1 << logh;
    for (int b = threadIdx.x; b < (1 << (logL - logR)); b += blockDim.x) {
        const int pos = b & (h - 1);
        const int base = ((b >> logh) << logS) + pos;
        V x[R];
#pragma unroll
        for (int q = 0; q < R; ++q) x[q] = buf[ph<PAD>(base + (q << logh))];
        twiddle_apply<R, true>(x, tw, pos, logS);
        dftR<R, true>(x);
#pragma unroll
        for (int t = 0; t < R; ++t) buf[ph<PAD>(base + (t << logh))] = x[t];
    }
    __syncthreads();
}

// forward DFT of buf[0 .. 2^logL): natural order in, X_k at freq_to_pos(k) out
template <bool PAD, typename T> __device__ void fft_fwd(c2_t<T> *buf, const Tw<T> &tw, int logL) {
    const int n8 = logL / 3, rem = logL - 3 * n8;
    int logS = logL;
    for (int i = 0; i < n8; ++i, logS -= 3) dif_stage<8, PAD>(buf, tw, logL, logS);
    if (rem == 2) dif_stage<4, PAD>(buf, tw, logL, 2);
    if (rem == 1) dif_stage<2, PAD>(buf, tw, logL, 1);
}

// unnormalised inverse DFT: X_k at freq_to_pos(k) in, natural order out
template <bool PAD, typename T> __device__ void fft_inv(c2_t<T> *buf, const Tw<T> &tw, int logL) {
    const int n8 = logL / 3, rem = logL - 3 * n8;
    if (rem == 2) dit_inv_stage<4, PAD>(buf, tw, logL, 2);
    if (rem == 1) dit_inv_stage<2, PAD>(buf, tw, logL, 1);
    for (int logS = rem + 3; logS <= logL; logS += 3) dit_inv_stage<8, PAD>(buf, tw, logL, logS);
}

__device__ __forceinline__ int ilog2(int L) { return 31 - __clz(L); }

template <typename T> __device__ __forceinline__ Tw<T> twiddles(const GeomDev &g);
template <> __device__ __forceinline__ Tw<float> twiddles<float>(const GeomDev &g) { return {g.tw32, g.log_tw}; }
template <> __device__ __forceinline__ Tw<double> twiddles<double>(const GeomDev &g) { return {g.tw64, g.log_tw}; }

template <typename T> __device__ __forceinline__ const c2_t<T> *blu_table(const GeomDev &g);
template <> __device__ __forceinline__ const float2 *blu_table<float>(const GeomDev &g) { return g.blu_f32; }
template <> __device__ __forceinline__ const double2 *blu_table<double>(const GeomDev &g) { return g.blu_f64; }

// ------------------------------------------------------------------------------ trig tables
// exp(-i pi x) with x = num / den reduced to [0, 2), in FP64, rounded to T
template <typename T> __device__ __forceinline__ c2_t<T> expmipi(int64_t num, int64_t den) {
    int64_t q = num % (2 * den);
    if (q < 0) q += 2 * den;
    double s, c;
    sincospi((double)q / (double)den, &s, &c);
    return mk2((T)c, (T)(-s));
}
template <typename T> __device__ __forceinline__ c2_t<T> expmipi_real(double p) {  // exp(-i pi p)
    p -= 2.0 * floor(0.5 * p);
    double s, c;
    sincospi(p, &s, &c);
    return mk2((T)c, (T)(-s));
}

// e(j) = fine[j & 63] * coarse[j >> 6]
template <typename T> struct Trig2 {
    const c2_t<T> *fine, *coarse;
    __device__ __forceinline__ c2_t<T> operator()(int64_t j) const { return cmul(fine[j & 63], coarse[j >> 6]); }
};

// per-ring tables in shared memory (after the FFT buffer):
//   untangle U(k) = exp(-2 pi i k / n), k <= N;  phase P(m) = exp(-i m phi0), m <= mmax;
//   chirp C(q) = exp(-i pi q / N), q < 2N (Bluestein rings only)
template <typename T> struct RingTrig {
    Trig2<T> U, P, C;
};

template <typename T> __host__ __device__ __forceinline__ int trig_entries(int Nmax, int mmax) {
    return 3 * 64 + (Nmax >> 6) + 2 + (mmax >> 6) + 2 + ((2 * Nmax) >> 6) + 2;
}

template <typename T>
__device__ RingTrig<T> build_trig(c2_t<T> *tab, int n, int N, double phi0_pi, int mmax, bool chirp) {
    using V = c2_t<T>;
    V *u1 = tab, *p1 = u1 + 64, *c1 = p1 + 64;
    V *u2 = c1 + 64;
    const int nu2 = (N >> 6) + 1, np2 = (mmax >> 6) + 1, nc2 = chirp ? ((2 * N) >> 6) + 1 : 0;
    V *p2 = u2 + nu2, *c2 = p2 + np2;
    for (int j = threadIdx.x; j < 64; j += blockDim.x) {
        u1[j] = expmipi<T>(2 * (int64_t)j, n);
        p1[j] = expmipi_real<T>((double)j * phi0_pi);
        if (chirp) c1[j] = expmipi<T>(j, N);
    }
    for (int j = threadIdx.x; j < nu2; j += blockDim.x) u2[j] = expmipi<T>(128 * (int64_t)j, n);
    for (int j = threadIdx.x; j < np2; j += blockDim.x) p2[j] = expmipi_real<T>(64.0 * (double)j * phi0_pi);
    for (int j = threadIdx.x; j < nc2; j += blockDim.x) c2[j] = expmipi<T>(64 * (int64_t)j, N);
    RingTrig<T> R;
    R.U = {u1, u2};
    R.P = {p1, p2};
    R.C = {c1, c2};
    return R;
}

// tables of ring `side` of the pair; the south ring reuses the north ring's when its nphi and
// phi0 match (always on HEALPix grids).  Ends with a barrier.
template <typename T>
__device__ __forceinline__ RingTrig<T> trig_for_ring(const GeomDev &g, c2_t<T> *tab, int pair, int side, int n,
                                                     int N, int mmax, bool chirp) {
    bool rebuild = true;
    if (side == 1) {
        const int rn = g.pair_ring[2 * pair];
        const int rs = g.pair_ring[2 * pair + 1];
        rebuild = g.nphi[rn] != g.nphi[rs] || g.phi0_pi[rn] != g.phi0_pi[rs];
    }
    if (rebuild) {
        const RingTrig<T> R = build_trig<T>(tab, n, N, side ? g.phi0_pi[g.pair_ring[2 * pair + 1]] : g.phi0_pi[g.pair_ring[2 * pair]], mmax, chirp);
        __syncthreads();
        return R;
    }
    // same layout as build_trig produced for the north ring (same n, N, mmax, chirp)
    RingTrig<T> R;
    c2_t<T> *u1 = tab, *p1 = u1 + 64, *c1 = p1 + 64, *u2 = c1 + 64;
    c2_t<T> *p2 = u2 + (N >> 6) + 1, *c2 = p2 + (mmax >> 6) + 1;
    R.U = {u1, u2};
    R.P = {p1, p2};
    R.C = {c1, c2};
    return R;
}

// chirp w_j = exp(-i pi j^2 / N)
template <typename T> __device__ __forceinline__ c2_t<T> chirp(const RingTrig<T> &R, int64_t j, int N) {
    return R.C((j * j) % (2 * (int64_t)N));
}

// ------------------------------------------------------------------------------ analysis
template <typename T>
__global__ void __launch_bounds__(512, 2) ring_analysis_kernel(GeomDev g, const int32_t *__restrict__ pairs,
                                                               const T *__restrict__ maps, int64_t map_stride,
                                                               const double *__restrict__ w, c2_t<T> *__restrict__ Fm,
                                                               int64_t fm_stride, int mmax, int flags, int unit_w,
                                                               int mdouble, int Lcls) {
    using V = c2_t<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *buf = reinterpret_cast<V *>(smem_raw);
    V *tab = buf + padded_len(Lcls);
    const int pair = pairs[blockIdx.y], b = blockIdx.x;  // maps fastest: a pair's tables stay in L2
    const int64_t np = g.npairs;
    V *out = Fm + b * fm_stride;
    const Tw<T> tw = twiddles<T>(g);
    const double twopi = 6.283185307179586476925286766559;
    for (int side = 0; side < 2; ++side) {
        const int r = g.pair_ring[2 * pair + side];
        if (r < 0) {  // unpaired ring: zero south half
            for (int m = threadIdx.x; m <= mmax; m += blockDim.x) out[((int64_t)m * np + pair) * 2 + 1] = mk2((T)0, (T)0);
            continue;
        }
        const int n = g.nphi[r], N = n >> 1, L = g.fft_len[r], logL = ilog2(L);
        const int64_t bo = g.blu_ofs[r];
        const bool direct = bo < 0;
        __syncthreads();  // previous ring done with buf / tables
        const RingTrig<T> R = trig_for_ring<T>(g, tab, pair, side, n, N, mmax, !direct);
        const V *f2 = reinterpret_cast<const V *>(maps + b * map_stride + g.ofs[r]);  // ring offsets: multiples of 4
        if (direct) {
            for (int j = threadIdx.x; j < N; j += blockDim.x) buf[ph<true>(j)] = f2[j];
        } else {
            for (int j = threadIdx.x; j < L; j += blockDim.x)
                buf[ph<true>(j)] = (j < N) ? cmul(f2[j], chirp(R, j, N)) : mk2((T)0, (T)0);
        }
        __syncthreads();
        fft_fwd<true, T>(buf, tw, logL);
        if (!direct) {
            const V *Bt = blu_table<T>(g) + bo;
            for (int i = threadIdx.x; i < L; i += blockDim.x) buf[ph<true>(i)] = cmul(buf[ph<true>(i)], Bt[i]);
            __syncthreads();
            fft_inv<true, T>(buf, tw, logL);
        }
        // Z_k, 0 <= k < N
        auto Z = [&](int k) -> V {
            return direct ? buf[ph<true>(freq_to_pos(k, logL))] : cmul(buf[ph<true>(k)], chirp(R, k, N));
        };
        const T scale = unit_w ? (T)1 : (T)(((flags & HB_F_NO2PI) ? 1.0 : twopi) * w[r] / (double)n);
        const int side_out = g.ring_side[r];
        auto emit = [&](int m, V X) {
            if (!(flags & HB_F_NOPHASE)) X = cmul(X, R.P(m));
            T sc = scale;
            if (mdouble && m > 0) sc *= (T)2;
            if ((flags & HB_F_NOFOLD) && m >= n) sc = (T)0;
            out[((int64_t)m * np + pair) * 2 + side_out] = cscale(X, sc);
        };
        // F_k = (A - i U(k) D) / 2, A = Z_k + conj Z_{N-k}, D = Z_k - conj Z_{N-k}; harmonic m takes
        // bin m mod n (conjugated above N).  Threads walk the buffer in storage order.
        for (int p = threadIdx.x; p < N; p += blockDim.x) {
            const int k = direct ? pos_to_freq(p, logL) : p;
            const V zk = direct ? buf[ph<true>(p)] : cmul(buf[ph<true>(p)], chirp(R, p, N));
            const V zc = cconj(k == 0 ? zk : Z(N - k));
            const V A = cadd(zk, zc), D = csub(zk, zc);
            auto bin = [&](int kk) -> V {
                const V u = R.U(kk);
                const V iuD = mk2(-(u.x * D.y + u.y * D.x), u.x * D.x - u.y * D.y);  // i u D
                return mk2((T)0.5 * (A.x - iuD.x), (T)0.5 * (A.y - iuD.y));
            };
            const V X = bin(k);
            for (int m = k; m <= mmax; m += n) emit(m, X);
            if (k > 0)
                for (int m = n - k; m <= mmax; m += n) emit(m, cconj(X));
            else {
                const V XN = bin(N);
                for (int m = N; m <= mmax; m += n) emit(m, XN);
            }
        }
    }
}

// ------------------------------------------------------------------------------ synthesis
template <typename T>
__global__ void __launch_bounds__(512, 2) ring_synthesis_kernel(GeomDev g, const int32_t *__restrict__ pairs,
                                                                const c2_t<T> *__restrict__ Gm, int64_t gm_stride,
                                                                int mmax, T *__restrict__ maps, int64_t map_stride,
                                                                const double *__restrict__ w, int apply_w, int mdouble,
                                                                int flags, int Lcls, int stage_t) {
    using V = c2_t<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *buf = reinterpret_cast<V *>(smem_raw);
    V *tab = buf + padded_len(Lcls);
    V *ts = tab + trig_entries<T>(Lcls, mmax);  // staged T_m, m <= mmax (when stage_t)
    const int pair = pairs[blockIdx.y], b = blockIdx.x;  // maps fastest: a pair's tables stay in L2
    const int64_t np = g.npairs;
    const V *gin = Gm + b * gm_stride;
    const Tw<T> tw = twiddles<T>(g);
    const double twopi = 6.283185307179586476925286766559;
    for (int side = 0; side < 2; ++side) {
        const int r = g.pair_ring[2 * pair + side];
        if (r < 0) continue;
        const int n = g.nphi[r], N = n >> 1, L = g.fft_len[r], logL = ilog2(L);
        const int64_t bo = g.blu_ofs[r];
        const bool direct = bo < 0;
        const int side_in = g.ring_side[r];
        __syncthreads();
        const RingTrig<T> R = trig_for_ring<T>(g, tab, pair, side, n, N, mmax, !direct);
        // T_m = c_m G(m) exp(+i m phi0)
        auto Tm_global = [&](int m) -> V {
            V v = gin[((int64_t)m * np + pair) * 2 + side_in];
            if (!(flags & HB_F_NOPHASE)) v = cmul(v, cconj(R.P(m)));
            if (mdouble && m > 0) v = cscale(v, (T)2);
            return v;
        };
        if (stage_t) {  // independent loads of every T_m of the ring, then the folds read shared memory
#pragma unroll 4
            for (int m = threadIdx.x; m <= mmax; m += blockDim.x) ts[m] = Tm_global(m);
            __syncthreads();
        }
        auto Tm = [&](int m) -> V { return stage_t ? ts[m] : Tm_global(m); };
        // Hermitian half-spectrum bin X_k (0 <= k <= N) of the real ring, folded over m
        auto Xk = [&](int k) -> V {
            V acc = mk2((T)0, (T)0);
            if (k == 0 || k == N) {
                for (int m = k; m <= mmax; m += n) acc.x += Tm(m).x;
            } else {
                for (int m = k; m <= mmax; m += n) acc = cadd(acc, cscale(Tm(m), (T)0.5));
                for (int m = n - k; m <= mmax; m += n) acc = cadd(acc, cscale(cconj(Tm(m)), (T)0.5));
            }
            return acc;
        };
        // Zv_k = (X_k + conj X_{N-k}) + i conj(U(k)) (X_k - conj X_{N-k}), k < N, written where the
        // inverse transform expects it; threads walk the buffer in storage order.
        if (!direct)
            for (int j = N + threadIdx.x; j < L; j += blockDim.x) buf[ph<true>(j)] = mk2((T)0, (T)0);
        for (int p = threadIdx.x; p < N; p += blockDim.x) {
            const int k = direct ? pos_to_freq(p, logL) : p;
            const V xa = Xk(k), xb = cconj(Xk(N - k));
            const V S = cadd(xa, xb), D = csub(xa, xb);
            const V u = R.U(k);
            const V z = mk2(S.x - u.x * D.y + u.y * D.x, S.y + u.x * D.x + u.y * D.y);  // S + i conj(u) D
            // inverse DFT as conj(DFT(conj Z)) through the chirp-z convolution
            buf[ph<true>(p)] = direct ? z : cmul(cconj(z), chirp(R, k, N));
        }
        __syncthreads();
        if (direct) {
            fft_inv<true, T>(buf, tw, logL);
        } else {
            fft_fwd<true, T>(buf, tw, logL);
            const V *Bt = blu_table<T>(g) + bo;
            for (int i = threadIdx.x; i < L; i += blockDim.x) buf[ph<true>(i)] = cmul(buf[ph<true>(i)], Bt[i]);
            __syncthreads();
            fft_inv<true, T>(buf, tw, logL);
        }
        const T pscale = apply_w ? (T)(((flags & HB_F_NO2PI) ? 1.0 : twopi) * w[r] / (double)n) : (T)1;
        V *out2 = reinterpret_cast<V *>(maps + b * map_stride + g.ofs[r]);
        for (int j = threadIdx.x; j < N; j += blockDim.x) {
            V z = buf[ph<true>(j)];
            if (!direct) z = cconj(cmul(z, chirp(R, j, N)));
            out2[j] = cscale(z, pscale);
        }
    }
}

// ------------------------------------------------------------------------------ tables
// W^j = exp(-2 pi i j / 2^log_tw), j < 2^(log_tw - 1), FP64 and rounded FP32
__global__ void twiddle_table_kernel(GeomDev g) {
    const int half = 1 << (g.log_tw - 1);
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < half; j += gridDim.x * blockDim.x) {
        double s, c;
        sincospi(-2.0 * (double)j / (double)(1 << g.log_tw), &s, &c);
        g.tw64[j] = make_double2(c, s);
        g.tw32[j] = make_float2((float)c, (float)s);
    }
}

// Chirp spectra for Bluestein: Bt = FFT_L(b) / L in the forward transform's output order,
// b_t = exp(+i pi t^2 / N) for |t| < N (circular); one CTA per distinct N, FP64, then rounded
// to FP32 for the single-precision kernels.
__global__ void __launch_bounds__(1024) bluestein_table_kernel(GeomDev g) {
    const int r = g.blu_owner[blockIdx.x];
    const int64_t bo = g.blu_ofs[r];
    const int N = g.nphi[r] >> 1, L = g.fft_len[r];
    double2 *buf = g.blu_f64 + bo;  // global memory work buffer (the table itself)
    for (int t = threadIdx.x; t < L; t += blockDim.x) {
        const int64_t j = (t < N) ? t : ((L - t < N) ? L - t : -1);
        double2 v = make_double2(0.0, 0.0);
        if (j >= 0) {
            const double2 e = expmipi<double>(j * j, N);  // exp(-i pi j^2/N)
            v = make_double2(e.x, -e.y);
        }
        buf[t] = v;
    }
    __syncthreads();
    const Tw<double> tw{g.tw64, g.log_tw};
    fft_fwd<false, double>(buf, tw, ilog2(L));
    const double inv = 1.0 / (double)L;
    for (int t = threadIdx.x; t < L; t += blockDim.x) {
        const double2 v = make_double2(buf[t].x * inv, buf[t].y * inv);
        buf[t] = v;
        g.blu_f32[bo + t] = make_float2((float)v.x, (float)v.y);
    }
}

int build_fft_tables(GeomDev &g, cudaStream_t st) {
    twiddle_table_kernel<<<64, 256, 0, st>>>(g);
    HB_CHECK_LAUNCH();
    if (g.n_blu > 0) {
        bluestein_table_kernel<<<(unsigned)g.n_blu, 1024, 0, st>>>(g);
        HB_CHECK_LAUNCH();
    }
    return HB_OK;
}

// ------------------------------------------------------------------------------ launch
static int max_smem_optin() {
    static int v = -1;
    if (v < 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) v = 48 * 1024;
    }
    return v;
}

template <typename T> static size_t class_smem(int L, int mmax) {
    return sizeof(c2_t<T>) * ((size_t)padded_len(L) + (size_t)trig_entries<T>(L, mmax));
}
// synthesis: plus the staged T_m (mmax + 1 entries) when that fits
template <typename T> static size_t class_smem_syn(int L, int mmax, bool stage_t) {
    return class_smem<T>(L, mmax) + (stage_t ? sizeof(c2_t<T>) * (size_t)(mmax + 1) : 0);
}

static int class_threads(int L) { return L >= 4096 ? 512 : (L >= 512 ? 256 : (L >= 64 ? 128 : 64)); }

template <typename T>
static int check_smem(const GeomDev &g, int mmax) {
    for (int c = 0; c < g.n_cls; ++c) {
        const size_t smem = class_smem<T>(g.cls_L[c], mmax);
        if (smem > (size_t)max_smem_optin())
            return fail(HB_ERR_UNSUPPORTED, "ring FFT: convolution length " + std::to_string(g.cls_L[c]) + " needs " +
                                                std::to_string(smem) + " B of shared memory in this precision");
    }
    return HB_OK;
}

template <typename T>
static int launch_analysis_t(const GeomDev &g, int nmaps, const T *maps, int64_t map_stride, const double *w,
                             c2_t<T> *Fm, int mmax, int flags, bool unit_w, bool mdouble, cudaStream_t st) {
    int rc = check_smem<T>(g, mmax);
    if (rc) return rc;
    const int64_t fm_stride = (int64_t)(mmax + 1) * g.npairs * 2;
    for (int c = 0; c < g.n_cls; ++c) {
        const int L = g.cls_L[c];
        const int64_t first = g.cls_first[c], cnt = g.cls_first[c + 1] - first;
        const int smem = (int)class_smem<T>(L, mmax);
        HB_CUDA_TRY(cudaFuncSetAttribute(ring_analysis_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        HB_CUDA_TRY(cudaFuncSetAttribute(ring_analysis_kernel<T>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                         cudaSharedmemCarveoutMaxShared));
        dim3 grid((unsigned)nmaps, (unsigned)cnt);
        ring_analysis_kernel<T><<<grid, class_threads(L), smem, st>>>(g, g.cls_pairs + first, maps, map_stride,
                                                                       w ? w : g.w, Fm, fm_stride, mmax, flags,
                                                                       unit_w ? 1 : 0, mdouble ? 1 : 0, L);
        HB_CHECK_LAUNCH();
    }
    return HB_OK;
}

template <typename T>
static int launch_synthesis_t(const GeomDev &g, int nmaps, const c2_t<T> *Gm, int mmax, T *maps, int64_t map_stride,
                              const double *w, bool apply_w, bool mdouble, int flags, cudaStream_t st) {
    int rc = check_smem<T>(g, mmax);
    if (rc) return rc;
    const int64_t gm_stride = (int64_t)(mmax + 1) * g.npairs * 2;
    for (int c = 0; c < g.n_cls; ++c) {
        const int L = g.cls_L[c];
        const int64_t first = g.cls_first[c], cnt = g.cls_first[c + 1] - first;
        const bool stage_t = class_smem_syn<T>(L, mmax, true) <= (size_t)max_smem_optin();
        const int smem = (int)class_smem_syn<T>(L, mmax, stage_t);
        HB_CUDA_TRY(cudaFuncSetAttribute(ring_synthesis_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        HB_CUDA_TRY(cudaFuncSetAttribute(ring_synthesis_kernel<T>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                         cudaSharedmemCarveoutMaxShared));
        dim3 grid((unsigned)nmaps, (unsigned)cnt);
        ring_synthesis_kernel<T><<<grid, class_threads(L), smem, st>>>(g, g.cls_pairs + first, Gm, gm_stride, mmax,
                                                                        maps, map_stride, w ? w : g.w,
                                                                        apply_w ? 1 : 0, mdouble ? 1 : 0, flags, L,
                                                                        stage_t ? 1 : 0);
        HB_CHECK_LAUNCH();
    }
    return HB_OK;
}

int launch_ring_analysis(const GeomDev &g, int precision, int nmaps, const void *maps, int64_t map_stride,
                         const double *w, void *Fm, int mmax, int flags, bool unit_weights, bool mdouble,
                         cudaStream_t st) {
    if (precision == 32)
        return launch_analysis_t<float>(g, nmaps, (const float *)maps, map_stride, w, (float2 *)Fm, mmax, flags,
                                        unit_weights, mdouble, st);
    return launch_analysis_t<double>(g, nmaps, (const double *)maps, map_stride, w, (double2 *)Fm, mmax, flags,
                                     unit_weights, mdouble, st);
}

int launch_ring_synthesis(const GeomDev &g, int precision, int nmaps, const void *Gm, int mmax, void *maps,
                          int64_t map_stride, const double *w, bool apply_weights, bool mdouble, int flags,
                          cudaStream_t st) {
    if (precision == 32)
        return launch_synthesis_t<float>(g, nmaps, (const float2 *)Gm, mmax, (float *)maps, map_stride, w,
                                         apply_weights, mdouble, flags, st);
    return launch_synthesis_t<double>(g, nmaps, (const double2 *)Gm, mmax, (double *)maps, map_stride, w,
                                      apply_weights, mdouble, flags, st);
}

}  // namespace hb
