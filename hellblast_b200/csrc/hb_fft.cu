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
// Work decomposition: one CTA per (ring pair, map), pairs fastest in the grid; it transforms
// the pair's north ring, then its south ring, in one shared-memory buffer.  The analysis keeps
// the north ring's F(m) in shared memory and writes each m's (north, south) entry as one vector
// store, so two neighbouring CTAs fill each 32-byte sector of F.  Pairs are launched in classes
// of equal convolution length, each class with its own shared-memory size.
//
// FFT engine: a length L = 2^logL transform runs logL / 4 radix-16 stages and, when logL % 4 = r
// is not zero, one radix-2^r stage.  Every stage is a pass in registers: each thread loads the
// R points of a butterfly, transforms them and stores them back, with one barrier per pass.
// The passes at the ends read from or write to global memory directly where the order allows:
//   * analysis, direct ring: decimation in frequency (DIF) from the ring in global memory; the
//     untangling reads the digit-ordered spectrum;
//   * analysis, Bluestein ring: DIF from global memory times the chirp, then one fused pass
//     (last DIF stage, product with the stored chirp spectrum, first inverse DIT stage), then
//     the inverse decimation-in-time (DIT) stages, which leave natural order;
//   * synthesis, direct ring: the Hermitian spectrum is built from the folded T_m in one pass,
//     then inverse DIF and a digit-order read for the coalesced ring store;
//   * synthesis, Bluestein ring: the same fused middle, and the last inverse DIT pass writes the
//     ring to global memory.
// Twiddles: a radix-16 butterfly takes W^p, W^2p, W^4p, W^8p and forms the others by at most
// three products; FP32 computes the four with sincospif of exact arguments, FP64 reads them
// from one table per geometry, W^j = exp(-2 pi i j/Lmax), j < Lmax/2 (FP64-computed).  The Bluestein chirp exp(-i pi j^2/N) is a stored table
// per distinct N (after its spectrum).  The per-m factors of the untangling (exp(-2 pi i k/n))
// and the ring phase (exp(-i m phi0)) are products of two entries of small per-ring tables
// (64 fine steps x coarse steps), built per CTA with a few hundred FP64 sincospi.
//
// Fused into the m-major write (the reference has none of these, see sht_raw.py:41,51):
//   * the per-pixel quadrature weight 2*pi*w_r/nphi_r,
//   * the ring phase exp(-i m phi0_r),
//   * the aliasing fold: harmonic m lands on DFT bin m mod nphi (conjugated above nphi/2),
//     so every m <= mmax is produced, also on rings with nphi <= 2*mmax.
#include <algorithm>
#include <cmath>

#include "hb_internal.cuh"
#include "hb_fftcore.cuh"

namespace hb {

// ------------------------------------------------------------------------------ FFT plan
// Digit order: DIF takes natural order to the order in which position p of frequency k holds
// k's base-16 digits (lowest first) from the top down, then k's top r bits:
//   p = (nibble_reverse(k mod 16^a) << r) | (k >> 4a),  a = logL / 4, r = logL % 4.
// DIT (the mirror) takes digit order back to natural order.
__device__ __forceinline__ unsigned nibrev(unsigned x, int a) {  // reverse the order of the a low nibbles
    if (a == 0) return 0u;
    x = __byte_perm(x, 0u, 0x0123);
    x = ((x >> 4) & 0x0F0F0F0Fu) | ((x & 0x0F0F0F0Fu) << 4);
    return x >> (32 - 4 * a);
}
__device__ __forceinline__ int pos_of_freq(int k, int logL) {
    const int a = logL >> 2, r = logL & 3;
    const unsigned low = (1u << (4 * a)) - 1u;
    return (int)((nibrev((unsigned)k & low, a) << r) | ((unsigned)k >> (4 * a)));
}

// Shared-memory FFT buffers carry one pad element per 16 and one more per 256: every pass's
// half-warp accesses (stride 1 within a butterfly row, stride 16 in the last radix-16 stage,
// stride 2^r in the remainder stage) and the digit-order reads then spread over the banks.
__device__ __forceinline__ int ph(int i) { return i + (i >> 4) + (i >> 8); }
__host__ __device__ __forceinline__ int padded_len(int L) { return L + (L >> 4) + (L >> 8) + 1; }

template <typename T> struct Tw {
    using V = c2_t<T>;
    const V *tab;  // exp(-2 pi i j / 2^log_tw), j < 2^(log_tw - 1)
    int log_tw;
    // exp(-2 pi i e / 2^logS), 0 <= e < 2^logS <= 2^log_tw.  FP32: sincospif of the exact
    // argument 2e / 2^logS (no memory access on the butterflies' critical path); FP64: the table.
    __device__ __forceinline__ V w(int e, int logS) const {
        if constexpr (sizeof(T) == 4) {
            float sn, cs;
            sincospif(__int2float_rn(e) * __int_as_float((127 - (logS - 1)) << 23), &sn, &cs);
            return mk2(cs, -sn);
        }
        const int j = e << (log_tw - logS);
        const int half = 1 << (log_tw - 1);
        const V v = tab[j & (half - 1)];
        return (j & half) ? mk2(-v.x, -v.y) : v;
    }
};

// x[q] *= W_S^(pos q) (conjugated for INV), q = 1 .. R-1.  Radix 16 and 8 load W^pos, W^2pos,
// W^4pos (and W^8pos) and form the other factors by at most three products.
template <int R, bool INV, typename T>
__device__ __forceinline__ void twiddle_apply(c2_t<T> *x, const Tw<T> &tw, int pos, int logS) {
    using V = c2_t<T>;
    auto app = [&](int q, V wq) { x[q] = cmul(x[q], INV ? cconj(wq) : wq); };
    if constexpr (R == 16) {
        const V w1 = tw.w(pos, logS), w2 = tw.w(2 * pos, logS), w4 = tw.w(4 * pos, logS), w8 = tw.w(8 * pos, logS);
        const V w3 = cmul(w1, w2), w5 = cmul(w4, w1), w6 = cmul(w4, w2), w7 = cmul(w4, w3);
        app(1, w1); app(2, w2); app(3, w3); app(4, w4); app(5, w5); app(6, w6); app(7, w7); app(8, w8);
        app(9, cmul(w8, w1)); app(10, cmul(w8, w2)); app(11, cmul(w8, w3)); app(12, cmul(w8, w4));
        app(13, cmul(w8, w5)); app(14, cmul(w8, w6)); app(15, cmul(w8, w7));
    } else if constexpr (R == 8) {
        const V w1 = tw.w(pos, logS), w2 = tw.w(2 * pos, logS), w4 = tw.w(4 * pos, logS);
        const V w3 = cmul(w1, w2);
        app(1, w1); app(2, w2); app(3, w3); app(4, w4);
        app(5, cmul(w4, w1)); app(6, cmul(w4, w2)); app(7, cmul(w4, w3));
    } else {
#pragma unroll
        for (int q = 1; q < R; ++q) app(q, tw.w(pos * q, logS));
    }
}

// One stage of radix R on the sub-transforms of size 2^logS (butterfly b: pos = b mod h,
// points base + t h, h = 2^logS / R).  DIF: DFT, then twiddles on the outputs; DIT (its
// mirror): twiddles on the inputs, then DFT.  `ld(p)` / `st(p, v)` read and write point p
// (shared or global memory); a thread stores exactly the points it loaded.
template <int R, bool DIT, bool INV, typename T, class Ld, class St>
__device__ __forceinline__ void fft_pass(int logL, int logS, const Tw<T> &tw, Ld &&ld, St &&st) {
    using V = c2_t<T>;
    constexpr int lr = Log2R<R>::v;
    const int logh = logS - lr, h = 1 << logh;
    for (int b = threadIdx.x; b < (1 << (logL - lr)); b += blockDim.x) {
        const int pos = b & (h - 1), base = ((b >> logh) << logS) + pos;
        V x[R];
#pragma unroll
        for (int t = 0; t < R; ++t) x[t] = ld(base + (t << logh));
        if (DIT && logh > 0) twiddle_apply<R, INV>(x, tw, pos, logS);
        dftR<R, INV>(x);
        if (!DIT && logh > 0) twiddle_apply<R, INV>(x, tw, pos, logS);
#pragma unroll
        for (int q = 0; q < R; ++q) st(base + (q << logh), x[q]);
    }
}

// Bluestein middle: the last forward DIF stage (radix R, h = 1), the product with the chirp
// spectrum (stored in digit order), the first inverse DIT stage; all in registers.
template <int R, typename T, class Ld, class St>
__device__ __forceinline__ void mid_pass(int logL, const c2_t<T> *__restrict__ Bt, Ld &&ld, St &&st) {
    using V = c2_t<T>;
    constexpr int lr = Log2R<R>::v;
    for (int b = threadIdx.x; b < (1 << (logL - lr)); b += blockDim.x) {
        const int base = b << lr;
        V x[R];
#pragma unroll
        for (int t = 0; t < R; ++t) x[t] = ld(base + t);
        dftR<R, false>(x);
#pragma unroll
        for (int q = 0; q < R; ++q) x[q] = cmul(x[q], Bt[base + q]);
        dftR<R, true>(x);
#pragma unroll
        for (int t = 0; t < R; ++t) st(base + t, x[t]);
    }
}

// stage i of the plan in DIF order (i < logL / 4: radix 16; then the radix-2^(logL % 4) stage)
template <bool DIT, bool INV, typename T, class Ld, class St>
__device__ __forceinline__ void fft_stage(int i, int logL, const Tw<T> &tw, Ld &&ld, St &&st) {
    const int a = logL >> 2, r = logL & 3;
    if (i < a) {
        fft_pass<16, DIT, INV, T>(logL, logL - 4 * i, tw, ld, st);
    } else if (r == 3) {
        fft_pass<8, DIT, INV, T>(logL, 3, tw, ld, st);
    } else if (r == 2) {
        fft_pass<4, DIT, INV, T>(logL, 2, tw, ld, st);
    } else {
        fft_pass<2, DIT, INV, T>(logL, 1, tw, ld, st);
    }
}
template <typename T, class Ld, class St>
__device__ __forceinline__ void fft_mid(int logL, const c2_t<T> *Bt, Ld &&ld, St &&st) {
    const int r = logL & 3;
    if (r == 0) mid_pass<16, T>(logL, Bt, ld, st);
    else if (r == 3) mid_pass<8, T>(logL, Bt, ld, st);
    else if (r == 2) mid_pass<4, T>(logL, Bt, ld, st);
    else mid_pass<2, T>(logL, Bt, ld, st);
}
__host__ __device__ __forceinline__ int fft_nstages(int logL) { return (logL >> 2) + ((logL & 3) ? 1 : 0); }

// Bluestein convolution of the natural-order input `ld_in` (zero-padded to L by the caller's
// functor): DIF forward, fused middle, inverse DIT; the last inverse stage hands its points
// (natural order, times L) to `st_out`.  Intermediate stages use the shared buffer `buf`.
template <typename T, class LdIn, class StOut>
__device__ __forceinline__ void bluestein(c2_t<T> *buf, int logL, const Tw<T> &tw, const c2_t<T> *Bt, LdIn &&ld_in,
                                          StOut &&st_out) {
    using V = c2_t<T>;
    auto lds = [&](int p) -> V { return buf[ph(p)]; };
    auto sts = [&](int p, V v) { buf[ph(p)] = v; };
    const int P = fft_nstages(logL);
    if (P == 1) {
        fft_mid<T>(logL, Bt, ld_in, st_out);
        return;
    }
    fft_stage<false, false, T>(0, logL, tw, ld_in, sts);
    __syncthreads();
    for (int i = 1; i < P - 1; ++i) {
        fft_stage<false, false, T>(i, logL, tw, lds, sts);
        __syncthreads();
    }
    fft_mid<T>(logL, Bt, lds, sts);
    __syncthreads();
    for (int i = P - 2; i > 0; --i) {
        fft_stage<true, true, T>(i, logL, tw, lds, sts);
        __syncthreads();
    }
    fft_stage<true, true, T>(0, logL, tw, lds, st_out);
}

// DIF transform (forward or inverse) of the natural-order input `ld_in`; the result stays in
// `buf` in digit order.  Ends with a barrier.
template <bool INV, typename T, class LdIn>
__device__ __forceinline__ void dif_to_smem(c2_t<T> *buf, int logL, const Tw<T> &tw, LdIn &&ld_in) {
    using V = c2_t<T>;
    auto lds = [&](int p) -> V { return buf[ph(p)]; };
    auto sts = [&](int p, V v) { buf[ph(p)] = v; };
    const int P = fft_nstages(logL);
    fft_stage<false, INV, T>(0, logL, tw, ld_in, sts);
    __syncthreads();
    for (int i = 1; i < P; ++i) {
        fft_stage<false, INV, T>(i, logL, tw, lds, sts);
        __syncthreads();
    }
}

__device__ __forceinline__ int ilog2(int L) { return 31 - __clz(L); }

// exp(+i n phi0) of a ring of n pixels when it is exactly +1 or -1 (HEALPix rings, where
// n phi0 is 0 or pi), else 0
__device__ __forceinline__ int alias_sign(double phi0_pi, int n) {
    const double t = phi0_pi * (double)n, f = t - 2.0 * floor(0.5 * t);
    if (fabs(f) < 1e-12 || fabs(f - 2.0) < 1e-12) return 1;
    if (fabs(f - 1.0) < 1e-12) return -1;
    return 0;
}

// Lanes per bin pair: a ring of n = 2N pixels has K = N/2 + 1 bin pairs (k, N - k).  When K is
// small against the block, S = 2^j <= 32 neighbouring lanes share one k and each takes every
// S-th alias m0 + q n of its residue classes, so the alias loops of the small polar rings
// (up to mmax / n aliases per class) do not run on one thread each.
__device__ __forceinline__ int lanes_per_bin(int K) {
    int S = 1;
    while (S < 32 && 2 * S * K <= (int)blockDim.x) S *= 2;
    return S;
}

// asynchronous global -> shared copy of one complex value (cp.async), and its group bookkeeping
template <typename V> __device__ __forceinline__ void cp_async_elem(V *dst, const V *src);
template <> __device__ __forceinline__ void cp_async_elem<float2>(float2 *dst, const float2 *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
template <> __device__ __forceinline__ void cp_async_elem<double2>(double2 *dst, const double2 *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit_all() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

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
//   untangle U(k) = exp(-2 pi i k / n), k <= N;  phase P(m) = exp(-i m phi0), m <= mmax
template <typename T> struct RingTrig {
    Trig2<T> U, P;
};

template <typename T> __host__ __device__ __forceinline__ int trig_entries(int Nmax, int mmax) {
    return 2 * 64 + (Nmax >> 6) + 2 + (mmax >> 6) + 2;
}

template <typename T> __device__ __forceinline__ RingTrig<T> trig_layout(c2_t<T> *tab, int N) {
    RingTrig<T> R;
    c2_t<T> *u1 = tab, *p1 = u1 + 64, *u2 = p1 + 64, *p2 = u2 + (N >> 6) + 1;
    R.U = {u1, u2};
    R.P = {p1, p2};
    return R;
}

template <typename T> __device__ RingTrig<T> build_trig(c2_t<T> *tab, int n, int N, double phi0_pi, int mmax) {
    const RingTrig<T> R = trig_layout<T>(tab, N);
    c2_t<T> *u1 = const_cast<c2_t<T> *>(R.U.fine), *u2 = const_cast<c2_t<T> *>(R.U.coarse);
    c2_t<T> *p1 = const_cast<c2_t<T> *>(R.P.fine), *p2 = const_cast<c2_t<T> *>(R.P.coarse);
    const int nu2 = (N >> 6) + 1, np2 = (mmax >> 6) + 1;
    for (int j = threadIdx.x; j < 64; j += blockDim.x) {
        u1[j] = expmipi<T>(2 * (int64_t)j, n);
        p1[j] = expmipi_real<T>((double)j * phi0_pi);
    }
    for (int j = threadIdx.x; j < nu2; j += blockDim.x) u2[j] = expmipi<T>(128 * (int64_t)j, n);
    for (int j = threadIdx.x; j < np2; j += blockDim.x) p2[j] = expmipi_real<T>(64.0 * (double)j * phi0_pi);
    return R;
}

// tables of ring `side` of the pair; the south ring reuses the north ring's when its nphi and
// phi0 match (always on HEALPix grids).  Ends with a barrier.
template <typename T>
__device__ __forceinline__ RingTrig<T> trig_for_ring(const GeomDev &g, c2_t<T> *tab, int pair, int side, int n,
                                                     int N, int mmax) {
    bool rebuild = true;
    if (side == 1) {
        const int rn = g.pair_ring[2 * pair];
        const int rs = g.pair_ring[2 * pair + 1];
        rebuild = g.nphi[rn] != g.nphi[rs] || g.phi0_pi[rn] != g.phi0_pi[rs];
    }
    if (rebuild) {
        const RingTrig<T> R = build_trig<T>(tab, n, N, g.phi0_pi[g.pair_ring[2 * pair + side]], mmax);
        __syncthreads();
        return R;
    }
    return trig_layout<T>(tab, N);
}

// the chirp exp(-i pi j^2 / N), j < N, of a Bluestein ring: stored after its spectrum
template <typename T> __device__ __forceinline__ const c2_t<T> *chirp_table(const GeomDev &g, int64_t bo, int L) {
    return blu_table<T>(g) + bo + L;
}

// ------------------------------------------------------------------------------ analysis
// F(m) of one ring lands in F[map][m][pair][side].  With `stage_n` the north ring's values wait
// in shared memory until the south ring is done and each m is written as one (north, south)
// vector store; otherwise (unpaired rings, or no room) each side is stored on its own.
template <typename V> __device__ __forceinline__ void store_ns(V *dst, V n, V s);
template <> __device__ __forceinline__ void store_ns<float2>(float2 *dst, float2 n, float2 s) {
    *reinterpret_cast<float4 *>(dst) = make_float4(n.x, n.y, s.x, s.y);
}
template <> __device__ __forceinline__ void store_ns<double2>(double2 *dst, double2 n, double2 s) {
    dst[0] = n;
    dst[1] = s;
}

template <typename T>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 3 : 1)
    ring_analysis_kernel(GeomDev g, const int32_t *__restrict__ pairs, const T *__restrict__ maps, int64_t map_stride,
                         const double *__restrict__ w, c2_t<T> *__restrict__ Fm, int64_t fm_stride, int mmax,
                         int flags, int unit_w, int mdouble, int Lcls, int stage_n, int mblk) {
    using V = c2_t<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *buf = reinterpret_cast<V *>(smem_raw);
    V *tab = buf + padded_len(Lcls);
    V *stn = tab + trig_entries<T>(Lcls, mmax);  // north ring's F(m), m <= mmax (stage_n)
    const int pair = pairs[blockIdx.x], b = blockIdx.y;  // pairs fastest: neighbours complete F's sectors
    const int64_t np = g.npairs;
    V *out = Fm + b * fm_stride;
    auto slot = [&](int m) -> int64_t { return fg_off(m, pair, np, mblk != 0) * 2; };  // (north, south) of m
    const Tw<T> tw = twiddles<T>(g);
    const double twopi = 6.283185307179586476925286766559;
    const bool joint = stage_n && g.pair_ring[2 * pair + 1] >= 0;
    auto sts = [&](int p, V v) { buf[ph(p)] = v; };
    for (int side = 0; side < 2; ++side) {
        const int r = g.pair_ring[2 * pair + side];
        if (r < 0) {  // unpaired ring: zero south half
            for (int m = threadIdx.x; m <= mmax; m += blockDim.x) out[slot(m) + 1] = mk2((T)0, (T)0);
            continue;
        }
        const int n = g.nphi[r], N = n >> 1, L = g.fft_len[r], logL = ilog2(L);
        const int64_t bo = g.blu_ofs[r];
        const bool direct = bo < 0;
        __syncthreads();  // previous ring done with buf / tables
        const RingTrig<T> R = trig_for_ring<T>(g, tab, pair, side, n, N, mmax);
        const V *f2 = reinterpret_cast<const V *>(maps + b * map_stride + g.ofs[r]);  // ring offsets: multiples of 4
        const V *ch = direct ? nullptr : chirp_table<T>(g, bo, L);
        if (direct) {  // DIF from the ring itself: the spectrum stays in digit order
            dif_to_smem<false, T>(buf, logL, tw, [&](int p) -> V { return f2[p]; });
        } else {
            bluestein<T>(buf, logL, tw, blu_table<T>(g) + bo,
                         [&](int p) -> V { return p < N ? cmul(f2[p], ch[p]) : mk2((T)0, (T)0); }, sts);
            __syncthreads();
        }
        // Z_k, 0 <= k < N
        auto Z = [&](int k) -> V { return direct ? buf[ph(pos_of_freq(k, logL))] : cmul(buf[ph(k)], ch[k]); };
        const T scale = unit_w ? (T)1 : (T)(((flags & HB_F_NO2PI) ? 1.0 : twopi) * w[r] / (double)n);
        const int side_out = g.ring_side[r];
        // F(m) = c_m scale X exp(-i m phi0), X the bin m mod n (conjugated above N)
        auto put = [&](int m, V X) {  // X already carries scale exp(-i m phi0)
            if (mdouble && m > 0) X = cscale(X, (T)2);
            if ((flags & HB_F_NOFOLD) && m >= n) X = mk2((T)0, (T)0);
            if (!joint)
                out[slot(m) + side_out] = X;
            else if (side == 0)
                stn[m] = X;
            else
                store_ns(out + slot(m), stn[m], X);
        };
        // When exp(-i n phi0) = s = +-1 (HEALPix rings), exp(-i (m0 + j n) phi0) =
        // exp(-i m0 phi0) s^j: one phase product per residue class m0 instead of one per alias.
        const bool nophase = flags & HB_F_NOPHASE;
        const int s = nophase ? 1 : alias_sign(g.phi0_pi[r], n);
        const int K = N / 2 + 1, SL = lanes_per_bin(K), q0 = threadIdx.x & (SL - 1), kstep = blockDim.x / SL;
        auto emit_class = [&](int m0, V X) {  // aliases q = q0, q0 + S, ... of class m0
            const V Y = cscale(nophase ? X : cmul(X, R.P(m0)), scale);
            const V Yn = s > 0 ? Y : mk2(-Y.x, -Y.y);
            for (int q = q0, m = m0 + q0 * n; m <= mmax; q += SL, m += SL * n)
                put(m, s == 0 ? cscale(cmul(X, R.P(m)), scale) : (q & 1) ? Yn : Y);
        };
        // Bins of the real ring: F_k = (A - i U(k) D) / 2 with A = Z_k + conj Z_{N-k},
        // D = Z_k - conj Z_{N-k}, U(k) = exp(-2 pi i k / n); since U(N-k) = -conj U(k), the same
        // A, D give F_{N-k} = conj(A + i U(k) D) / 2, so one thread takes the pair (k, N-k)
        // (k = 0: bins 0 and N).  Harmonic m takes bin m mod n, conjugated above N.
        // The thread of k emits the residue classes k and n - k (bin k, the second conjugated) and
        // N - k and N + k (bin N - k); k = 0: classes 0 and N.  One loop over the four keeps a
        // single copy of the alias loop in the kernel (instruction-cache footprint).
        const int cstep = N > mmax ? 2 : 1;  // classes n - k, N + k (c = 1, 3) exceed mmax
        for (int k = threadIdx.x / SL; k < K; k += kstep) {
            const V zk = Z(k);
            const V zc = cconj(k == 0 ? zk : Z(N - k));
            const V A = cadd(zk, zc), D = csub(zk, zc);
            const V u = R.U(k);
            const V iuD = mk2(-(u.x * D.y + u.y * D.x), u.x * D.x - u.y * D.y);  // i u D
            const V Fk = mk2((T)0.5 * (A.x - iuD.x), (T)0.5 * (A.y - iuD.y));
            const V Fb = k == 0 ? mk2((T)0.5 * (A.x - D.y), (T)0.5 * (A.y + D.x))  // bin N: U(N) = -1
                                : mk2((T)0.5 * (A.x + iuD.x), (T)(-0.5) * (A.y + iuD.y));
            const bool lo = k > 0, hi = k == 0 || 2 * k < N;
#pragma unroll 1
            for (int c = 0; c < 4; c += cstep) {
                const bool on = c == 0 || (c == 1 && lo) || (c == 2 && hi) || (c == 3 && lo && hi);
                if (!on) continue;
                const int m0 = c == 0 ? k : c == 1 ? n - k : c == 2 ? N - k : N + k;
                if (m0 > mmax) continue;
                const V X = c < 2 ? Fk : Fb;
                emit_class(m0, (c & 1) ? cconj(X) : X);
            }
        }
    }
}

// ------------------------------------------------------------------------------ synthesis
template <typename T>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 3 : 1)
    ring_synthesis_kernel(GeomDev g, const int32_t *__restrict__ pairs, const c2_t<T> *__restrict__ Gm,
                          int64_t gm_stride, int mmax, T *__restrict__ maps, int64_t map_stride,
                          const double *__restrict__ w, int apply_w, int mdouble, int flags, int Lcls, int stage_t) {
    using V = c2_t<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *buf = reinterpret_cast<V *>(smem_raw);
    V *tab = buf + padded_len(Lcls);
    V *ts = tab + trig_entries<T>(Lcls, mmax);  // staged G(m) of the current ring, m <= mmax (when stage_t)
    const int pair = pairs[blockIdx.x], b = blockIdx.y;  // pairs fastest: neighbours share G's sectors
    const int64_t np = g.npairs;
    const V *gin = Gm + b * gm_stride;
    const Tw<T> tw = twiddles<T>(g);
    const double twopi = 6.283185307179586476925286766559;
    // stage_t = 1: a ring's G(m), m <= mmax, are loaded into ts when the ring starts.
    // stage_t = 2 (grids too small to hide load latency with other CTAs): they are copied with
    // cp.async, the north ring's before its trig tables are built, the south ring's as soon as
    // the north ring's spectrum pass is done with ts, so that they land during the north FFT.
    auto stage_issue = [&](int side_in) {
        if (stage_t == 2) {
            for (int m = threadIdx.x; m <= mmax; m += blockDim.x)
                cp_async_elem(ts + m, gin + ((int64_t)m * np + pair) * 2 + side_in);
            cp_async_commit_all();
        } else {
#pragma unroll 8
            for (int m = threadIdx.x; m <= mmax; m += blockDim.x) ts[m] = gin[((int64_t)m * np + pair) * 2 + side_in];
        }
    };
    const int rN = g.pair_ring[2 * pair], rS = g.pair_ring[2 * pair + 1];
    if (stage_t == 2 && rN >= 0) stage_issue(g.ring_side[rN]);
    for (int side = 0; side < 2; ++side) {
        const int r = side ? rS : rN;
        if (r < 0) continue;
        const int n = g.nphi[r], N = n >> 1, L = g.fft_len[r], logL = ilog2(L);
        const int64_t bo = g.blu_ofs[r];
        const bool direct = bo < 0;
        const int side_in = g.ring_side[r];
        __syncthreads();
        const RingTrig<T> R = trig_for_ring<T>(g, tab, pair, side, n, N, mmax);
        const V *ch = direct ? nullptr : chirp_table<T>(g, bo, L);
        if (stage_t) {  // this ring's G(m) in ts
            if (stage_t == 1 || (side == 1 && rN < 0)) stage_issue(side_in);
            cp_async_wait_all();
            __syncthreads();
        }
        auto G = [&](int m) -> V { return stage_t ? ts[m] : gin[((int64_t)m * np + pair) * 2 + side_in]; };
        // T_m = c_m G(m) exp(+i m phi0).  The fold needs, per residue class m0 mod n,
        // S(m0) = sum_j G(m0 + j n) exp(+i (m0 + j n) phi0).  When exp(i n phi0) = s = +-1
        // (HEALPix rings) that is exp(i m0 phi0) sum_j s^j G(m0 + j n): one add per alias.
        const bool nophase = flags & HB_F_NOPHASE;
        const int s = nophase ? 1 : alias_sign(g.phi0_pi[r], n);
        const int K = N / 2 + 1, SL = lanes_per_bin(K), q0 = threadIdx.x & (SL - 1), kstep = blockDim.x / SL;
        // this lane's part of S(m0): aliases q = q0, q0 + SL, ..., before the factor exp(i m0 phi0)
        // when s != 0
        auto Ssum = [&](int m0) -> V {
            V a = mk2((T)0, (T)0), c = a;  // even / odd q
            for (int q = q0, m = m0 + q0 * n; m <= mmax; q += SL, m += SL * n) {
                V v = G(m);
                if (s == 0) v = cmul(v, cconj(R.P(m)));
                if (q & 1)
                    c = cadd(c, v);
                else
                    a = cadd(a, v);
            }
            return s < 0 ? csub(a, c) : cadd(a, c);
        };
        const T dbl = mdouble ? (T)2 : (T)1, half = (T)0.5 * dbl;
        // Zv_k = (X_k + conj X_{N-k}) + i conj(U(k)) (X_k - conj X_{N-k}), 0 <= k < N
        auto spec = [&](V xa, V xb, int k) -> V {  // xa = X_k, xb = X_{N-k}
            xb = cconj(xb);
            const V S = cadd(xa, xb), D = csub(xa, xb);
            const V u = R.U(k);
            return mk2(S.x - u.x * D.y + u.y * D.x, S.y + u.x * D.x + u.y * D.y);  // S + i conj(u) D
        };
        const T pscale = apply_w ? (T)(((flags & HB_F_NO2PI) ? 1.0 : twopi) * w[r] / (double)n) : (T)1;
        V *out2 = reinterpret_cast<V *>(maps + b * map_stride + g.ofs[r]);
        // the spectrum in natural order (its folds loop over aliases, so it gets a pass of its own
        // rather than sitting inside the unrolled first FFT pass); Bluestein: conj(Z_k) chirp_k.
        // One thread takes the bins k and N - k of the Hermitian half-spectrum,
        // X_k = c (S(k) + conj S(n - k)) / 2 and X_{N-k} = c (S(N - k) + conj S(N + k)) / 2, so
        // every residue class of m mod n is folded once; k = 0 gives X_0 = c Re S(0) less the
        // surplus weight of m = 0, and X_N = c Re S(N).  One loop over the four classes
        // keeps a single copy of the alias loop in the kernel (instruction-cache footprint).
        auto put = [&](int k, V z) { buf[ph(k)] = direct ? z : cmul(cconj(z), ch[k]); };
        // The SL lanes of one k sum their parts with a butterfly (trip counts are uniform over the
        // block, so every lane reaches each shuffle); lane q0 = 0 writes the bins.
        const int iters = (K + kstep - 1) / kstep;
        const int cstep = N > mmax ? 2 : 1;  // classes n - k, N + k (c = 1, 3) exceed mmax
        for (int it = 0; it < iters; ++it) {
            const int k = it * kstep + (int)threadIdx.x / SL;
            const bool act = k < K;  // 2k <= N
            const int nc = 2 * k == N ? 2 : 4;
            V xa = mk2((T)0, (T)0), xb = xa;
#pragma unroll 1
            for (int c = 0; c < 4; c += cstep) {
                const int m0 = c == 0 ? k : c == 1 ? n - k : c == 2 ? N - k : N + k;
                const bool on = act && c < nc && m0 <= mmax && !(k == 0 && (c & 1));
                V t = on ? Ssum(m0) : mk2((T)0, (T)0);
                for (int o = 1; o < SL; o <<= 1) {
                    t.x += __shfl_xor_sync(0xffffffffu, t.x, o);
                    t.y += __shfl_xor_sync(0xffffffffu, t.y, o);
                }
                if (on && s != 0 && !nophase) t = cmul(t, cconj(R.P(m0)));
                if (c & 1) t = cconj(t);
                if (c < 2)
                    xa = cadd(xa, t);
                else
                    xb = cadd(xb, t);
            }
            if (!act || q0 != 0) continue;
            if (k == 0) {  // X_0 and X_N: S + conj S of the classes 0 and N
                xa = mk2((T)2 * xa.x, (T)0);
                xb = mk2((T)2 * xb.x, (T)0);
            }
            xa = cscale(xa, half);
            xb = nc == 2 ? xa : cscale(xb, half);
            if (k == 0) xa.x -= (dbl - (T)1) * G(0).x;
            put(k, spec(xa, xb, k));
            if (k > 0 && 2 * k < N) put(N - k, spec(xb, xa, N - k));
        }
        if (!direct)
            for (int k = N + threadIdx.x; k < L; k += blockDim.x) buf[ph(k)] = mk2((T)0, (T)0);
        __syncthreads();
        if (stage_t == 2 && side == 0 && rS >= 0) stage_issue(g.ring_side[rS]);  // lands during this ring's FFT
        auto lds = [&](int p) -> V { return buf[ph(p)]; };
        if (direct) {  // inverse DIF, then a digit-order read for the ring store
            dif_to_smem<true, T>(buf, logL, tw, lds);
            for (int j = threadIdx.x; j < N; j += blockDim.x) out2[j] = cscale(buf[ph(pos_of_freq(j, logL))], pscale);
        } else {  // inverse DFT as conj(DFT(conj Z)) through the chirp-z convolution
            bluestein<T>(buf, logL, tw, blu_table<T>(g) + bo, lds, [&](int p, V v) {
                if (p < N) out2[p] = cscale(cconj(cmul(v, ch[p])), pscale);
            });
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

// Chirp spectra for Bluestein: Bt = FFT_L(b) / L in digit order (the order the fused middle
// pass reads), b_t = exp(+i pi t^2 / N) for |t| < N (circular), and after it the chirp
// exp(-i pi j^2 / N), j < N.  One CTA per distinct N; the transform runs in FP64 on the table
// itself in global memory (barriers make each pass's stores visible to the block), then is
// rounded to FP32 for the single-precision kernels.
__global__ void __launch_bounds__(256) bluestein_table_kernel(GeomDev g) {
    const int r = g.blu_owner[blockIdx.x];
    const int64_t bo = g.blu_ofs[r];
    const int N = g.nphi[r] >> 1, L = g.fft_len[r], logL = ilog2(L);
    double2 *buf = g.blu_f64 + bo;
    for (int t = threadIdx.x; t < L; t += blockDim.x) {
        const int64_t j = (t < N) ? t : ((L - t < N) ? L - t : -1);
        double2 v = make_double2(0.0, 0.0);
        if (j >= 0) {
            const double2 e = expmipi<double>(j * j, N);  // exp(-i pi j^2/N)
            v = make_double2(e.x, -e.y);
            if (t < N) {
                g.blu_f64[bo + L + t] = e;
                g.blu_f32[bo + L + t] = make_float2((float)e.x, (float)e.y);
            }
        }
        buf[t] = v;
    }
    __syncthreads();
    const Tw<double> tw{g.tw64, g.log_tw};
    auto ldg = [&](int p) -> double2 { return buf[p]; };
    auto stg = [&](int p, double2 v) { buf[p] = v; };
    for (int i = 0; i < fft_nstages(logL); ++i) {
        fft_stage<false, false, double>(i, logL, tw, ldg, stg);
        __syncthreads();
    }
    const double inv = 1.0 / (double)L;
    for (int t = threadIdx.x; t < L; t += blockDim.x) {
        const double2 v = make_double2(buf[t].x * inv, buf[t].y * inv);
        buf[t] = v;
        g.blu_f32[bo + t] = make_float2((float)v.x, (float)v.y);
    }
}

// FP32 tables of the pair-packed Bluestein kernels (hb_ringpack.cu), 3L/2 entries each: the
// natural-order chirp spectrum FFT_L(b) / L, b_t = exp(+i pi t^2 / n) for |t| < n (circular),
// L = 2^logL >= 2n - 1, n = ns[e], then the chirp c_t = exp(-i pi t^2 / n) for t < L/2 (zero
// from n on).  One CTA per table; the FP64 transform runs in place in a global scratch slot
// (DIF, digit order; barriers make each pass's stores visible to the block), and the result is
// read back in natural order.
__global__ void __launch_bounds__(256) pk_chirp_kernel(GeomDev g, const int32_t *__restrict__ ns,
                                                       const int32_t *__restrict__ logLs,
                                                       const int64_t *__restrict__ ofs, int first, double2 *scratch,
                                                       int64_t slot, float2 *out) {
    const int e = first + blockIdx.x, n = ns[e], logL = logLs[e], L = 1 << logL;
    double2 *buf = scratch + (int64_t)blockIdx.x * slot;
    for (int t = threadIdx.x; t < L; t += blockDim.x) {
        const int64_t j = (t < n) ? t : ((L - t < n) ? L - t : -1);
        double2 v = make_double2(0.0, 0.0);
        if (j >= 0) {
            const double2 c = expmipi<double>(j * j, n);  // exp(-i pi j^2 / n)
            v = make_double2(c.x, -c.y);
        }
        buf[t] = v;
    }
    __syncthreads();
    const Tw<double> tw{g.tw64, g.log_tw};
    auto ldg = [&](int p) -> double2 { return buf[p]; };
    auto stg = [&](int p, double2 v) { buf[p] = v; };
    for (int i = 0; i < fft_nstages(logL); ++i) {
        fft_stage<false, false, double>(i, logL, tw, ldg, stg);
        __syncthreads();
    }
    const double inv = 1.0 / (double)L;
    for (int k = threadIdx.x; k < L; k += blockDim.x) {
        const double2 v = buf[pos_of_freq(k, logL)];
        out[ofs[e] + k] = make_float2((float)(v.x * inv), (float)(v.y * inv));
    }
    for (int t = threadIdx.x; t < L / 2; t += blockDim.x) {
        double2 c = make_double2(0.0, 0.0);
        if (t < n) c = expmipi<double>((int64_t)t * t, n);
        out[ofs[e] + L + t] = make_float2((float)c.x, (float)c.y);
    }
}

int build_pk_chirp_tables(const GeomDev &g, int count, const int32_t *ns, const int32_t *logL, const int64_t *ofs,
                          int max_logL, float2 *out, cudaStream_t st) {
    const int64_t slot = int64_t(1) << max_logL;
    const int chunk = 128;
    double2 *scratch = nullptr;
    if (cudaMalloc(&scratch, sizeof(double2) * slot * chunk) != cudaSuccess) {
        cudaGetLastError();
        return fail(HB_ERR_ALLOC, "hb_geom: chirp-spectrum scratch allocation failed");
    }
    int rc = HB_OK;
    for (int first = 0; first < count && rc == HB_OK; first += chunk) {
        const int cnt = std::min(chunk, count - first);
        pk_chirp_kernel<<<cnt, 256, 0, st>>>(g, ns, logL, ofs, first, scratch, slot, out);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) rc = fail(HB_ERR_CUDA, std::string("pk_chirp_kernel: ") + cudaGetErrorString(e));
    }
    if (cudaStreamSynchronize(st) != cudaSuccess && rc == HB_OK) rc = fail(HB_ERR_CUDA, "pk_chirp_kernel failed");
    cudaFree(scratch);
    return rc;
}

int build_fft_tables(GeomDev &g, cudaStream_t st) {
    twiddle_table_kernel<<<64, 256, 0, st>>>(g);
    HB_CHECK_LAUNCH();
    if (g.n_blu > 0) {
        bluestein_table_kernel<<<(unsigned)g.n_blu, 256, 0, st>>>(g);
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
// synthesis: plus the staged G(m) of one ring (mmax + 1 entries) when that fits
template <typename T> static size_t class_smem_syn(int L, int mmax, bool stage_t) {
    return class_smem<T>(L, mmax) + (stage_t ? sizeof(c2_t<T>) * (size_t)(mmax + 1) : 0);
}

static int smem_per_sm() {
    static int v = -1;
    if (v < 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess) v = 100 * 1024;
    }
    return v;
}
static int sm_count() {
    static int v = -1;
    if (v < 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) v = 148;
    }
    return v;
}
// CTAs of `bytes` dynamic shared memory that fit on one SM (1 KB reserved per CTA)
static int ctas_by_smem(size_t bytes) { return (int)((size_t)smem_per_sm() / (bytes + 1024)); }

// one radix-16 butterfly per thread where the class allows, 64 to 256 threads
static int class_threads(int L) { return std::max(64, std::min(256, L / 16)); }

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
                             c2_t<T> *Fm, int mmax, int flags, bool unit_w, bool mdouble, cudaStream_t st,
                             bool mblk) {
    int rc = check_smem<T>(g, mmax);
    if (rc) return rc;
    if (nmaps > 65535) return fail(HB_ERR_INVALID, "ring FFT: at most 65535 maps per call");
    const int64_t fm_stride = fg_rows(mmax, mblk) * g.npairs * 2;
    // FP32: the pair-packed kernels take the pairs they can (hb_ringpack.cu), this kernel the rest
    const bool f32 = sizeof(T) == 4;
    if (f32 && g.pk_n_cls > 0) {
        rc = launch_pk_analysis(g, nmaps, reinterpret_cast<const float *>(maps), map_stride, w ? w : g.w,
                                reinterpret_cast<float2 *>(Fm), mmax, flags, unit_w, mdouble, st, mblk);
        if (rc) return rc;
    }
    const int ncls = f32 ? g.rest_n_cls : g.n_cls;
    const int *clsL = f32 ? g.rest_L : g.cls_L;
    const int64_t *clsF = f32 ? g.rest_first : g.cls_first;
    const int32_t *clsP = f32 ? g.rest_pairs : g.cls_pairs;
    for (int c = 0; c < ncls; ++c) {
        const int L = clsL[c];
        const int64_t first = clsF[c], cnt = clsF[c + 1] - first;
        // stage the north ring's F(m) for joint (north, south) stores unless that costs CTAs per SM
        const size_t base_smem = class_smem<T>(L, mmax), stage_bytes = sizeof(c2_t<T>) * (size_t)(mmax + 1);
        const int ctas0 = ctas_by_smem(base_smem), ctas1 = ctas_by_smem(base_smem + stage_bytes);
        const bool stage_n = base_smem + stage_bytes <= (size_t)max_smem_optin() && ctas1 >= std::min(2, ctas0);
        const int smem = (int)(base_smem + (stage_n ? stage_bytes : 0));
        HB_CUDA_TRY(cudaFuncSetAttribute(ring_analysis_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        HB_CUDA_TRY(cudaFuncSetAttribute(ring_analysis_kernel<T>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                         cudaSharedmemCarveoutMaxShared));
        dim3 grid((unsigned)cnt, (unsigned)nmaps);
        ring_analysis_kernel<T><<<grid, class_threads(L), smem, st>>>(g, clsP + first, maps, map_stride,
                                                                       w ? w : g.w, Fm, fm_stride, mmax, flags,
                                                                       unit_w ? 1 : 0, mdouble ? 1 : 0, L,
                                                                       stage_n ? 1 : 0, mblk ? 1 : 0);
        HB_CHECK_LAUNCH();
    }
    return HB_OK;
}

template <typename T>
static int launch_synthesis_t(const GeomDev &g, int nmaps, const c2_t<T> *Gm, int mmax, T *maps, int64_t map_stride,
                              const double *w, bool apply_w, bool mdouble, int flags, cudaStream_t st) {
    int rc = check_smem<T>(g, mmax);
    if (rc) return rc;
    if (nmaps > 65535) return fail(HB_ERR_INVALID, "ring FFT: at most 65535 maps per call");
    const int64_t gm_stride = (int64_t)(mmax + 1) * g.npairs * 2;
    // FP32: the pair-packed kernels take the pairs they can (hb_ringpack.cu), this kernel the rest
    const bool f32 = sizeof(T) == 4;
    if (f32 && g.pk_n_cls > 0) {
        rc = launch_pk_synthesis(g, nmaps, reinterpret_cast<const float2 *>(Gm), mmax, reinterpret_cast<float *>(maps),
                                 map_stride, w ? w : g.w, apply_w, mdouble, flags, st);
        if (rc) return rc;
    }
    const int ncls = f32 ? g.rest_n_cls : g.n_cls;
    const int *clsL = f32 ? g.rest_L : g.cls_L;
    const int64_t *clsF = f32 ? g.rest_first : g.cls_first;
    const int32_t *clsP = f32 ? g.rest_pairs : g.cls_pairs;
    for (int c = 0; c < ncls; ++c) {
        const int L = clsL[c];
        const int64_t first = clsF[c], cnt = clsF[c + 1] - first;
        const bool stage_t = class_smem_syn<T>(L, mmax, true) <= (size_t)max_smem_optin();
        const int smem = (int)class_smem_syn<T>(L, mmax, stage_t), nt = class_threads(L);
        HB_CUDA_TRY(cudaFuncSetAttribute(ring_synthesis_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        HB_CUDA_TRY(cudaFuncSetAttribute(ring_synthesis_kernel<T>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                         cudaSharedmemCarveoutMaxShared));
        // asynchronous staging when the grid is under two waves of resident CTAs
        int occ = 1;
        HB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, ring_synthesis_kernel<T>, nt, smem));
        const bool async_t = stage_t && cnt * (int64_t)nmaps < 2 * (int64_t)sm_count() * std::max(occ, 1);
        dim3 grid((unsigned)cnt, (unsigned)nmaps);
        ring_synthesis_kernel<T><<<grid, nt, smem, st>>>(g, clsP + first, Gm, gm_stride, mmax, maps, map_stride,
                                                         w ? w : g.w, apply_w ? 1 : 0, mdouble ? 1 : 0, flags, L,
                                                         stage_t ? (async_t ? 2 : 1) : 0);
        HB_CHECK_LAUNCH();
    }
    return HB_OK;
}

int launch_ring_analysis(const GeomDev &g, int precision, int nmaps, const void *maps, int64_t map_stride,
                         const double *w, void *Fm, int mmax, int flags, bool unit_weights, bool mdouble,
                         cudaStream_t st, bool mblk) {
    HB_NVTX("ring_analysis");
    if (precision == 32)
        return launch_analysis_t<float>(g, nmaps, (const float *)maps, map_stride, w, (float2 *)Fm, mmax, flags,
                                        unit_weights, mdouble, st, mblk);
    return launch_analysis_t<double>(g, nmaps, (const double *)maps, map_stride, w, (double2 *)Fm, mmax, flags,
                                     unit_weights, mdouble, st, mblk);
}

int launch_ring_synthesis(const GeomDev &g, int precision, int nmaps, const void *Gm, int mmax, void *maps,
                          int64_t map_stride, const double *w, bool apply_weights, bool mdouble, int flags,
                          cudaStream_t st) {
    HB_NVTX("ring_synthesis");
    if (precision == 32)
        return launch_synthesis_t<float>(g, nmaps, (const float2 *)Gm, mmax, (float *)maps, map_stride, w,
                                         apply_weights, mdouble, flags, st);
    return launch_synthesis_t<double>(g, nmaps, (const double2 *)Gm, mmax, (double *)maps, map_stride, w,
                                      apply_weights, mdouble, flags, st);
}

}  // namespace hb
