// Ragged per-ring FFT kernels (analysis: ring samples -> F[m, pair, side]; synthesis: the
// reverse), one CTA per (ring, map), everything staged in shared memory.
//
// Replaces the per-ring cp.fft.fft / cp.fft.ifft loops of the reference (sht_raw.py:38-43,
// sht_fallback.py:51-55, isht.py:16-24, spin.py:46-53,107-108), which launch one cuFFT per ring
// and sync on nphi per ring.  Ring r has nphi_r = 4i samples (polar caps) or 4*nside
// (equatorial belt).  A real ring of length n is packed into n/2 complex points
// z_j = f_2j + i f_2j+1; their DFT is a radix-2 FFT when n/2 is a power of two and a
// Bluestein chirp-z transform (power-of-two convolution, chirp spectra precomputed per
// distinct n in the geometry) otherwise.  Both run on one shared-memory buffer: the forward
// pass is decimation-in-frequency (natural in, bit-reversed out) and the inverse is
// decimation-in-time (bit-reversed in, natural out), so no explicit bit-reversal pass exists.
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

template <typename V> __device__ __forceinline__ int bitrev(int k, int logL) {
    return logL ? (int)(__brev((unsigned)k) >> (32 - logL)) : 0;
}

__device__ __forceinline__ int ilog2(int L) { return 31 - __clz(L); }

// tw[t] = exp(-2 pi i t / L), t < L/2 (L a power of two: t/L is exact in float)
template <typename T> __device__ void make_twiddles(c2_t<T> *tw, int L) {
    for (int t = threadIdx.x; t < L / 2; t += blockDim.x) {
        T s, c;
        sincospi_t((T)(-2 * t) / (T)L, &s, &c);
        tw[t] = mk2(c, s);
    }
}

// In-place radix-2 decimation-in-frequency forward FFT: natural order in, bit-reversed out.
template <typename T> __device__ void fft_dif(c2_t<T> *buf, const c2_t<T> *tw, int L) {
    for (int half = L >> 1, ts = 1; half >= 1; half >>= 1, ts <<= 1) {
        for (int b = threadIdx.x; b < L / 2; b += blockDim.x) {
            int pos = b & (half - 1);
            int i = ((b - pos) << 1) + pos, j = i + half;
            c2_t<T> u = buf[i], v = buf[j];
            buf[i] = cadd(u, v);
            buf[j] = cmul(csub(u, v), tw[pos * ts]);
        }
        __syncthreads();
    }
}

// In-place radix-2 decimation-in-time inverse FFT (sign +, unnormalised): bit-reversed in,
// natural order out.
template <typename T> __device__ void fft_dit_inv(c2_t<T> *buf, const c2_t<T> *tw, int L) {
    for (int half = 1, ts = L >> 1; half < L; half <<= 1, ts >>= 1) {
        for (int b = threadIdx.x; b < L / 2; b += blockDim.x) {
            int pos = b & (half - 1);
            int i = ((b - pos) << 1) + pos, j = i + half;
            c2_t<T> u = buf[i], v = cmul(buf[j], cconj(tw[pos * ts]));
            buf[i] = cadd(u, v);
            buf[j] = csub(u, v);
        }
        __syncthreads();
    }
}

// chirp w_j = exp(-i pi j^2 / N), with j^2 reduced mod 2N in integers
template <typename T> __device__ __forceinline__ c2_t<T> chirp(int64_t j, int N) {
    int64_t q = (j * j) % (2 * (int64_t)N);
    T s, c;
    sincospi_t(-(T)q / (T)N, &s, &c);
    return mk2(c, s);
}

template <typename T> __device__ __forceinline__ const c2_t<T> *blu_table(const GeomDev &g);
template <> __device__ __forceinline__ const float2 *blu_table<float>(const GeomDev &g) { return g.blu_f32; }
template <> __device__ __forceinline__ const double2 *blu_table<double>(const GeomDev &g) { return g.blu_f64; }

// Z = DFT_N(buf[0..N)) for the ring; on return Z_k sits at buf[zidx(k)].
// direct (bo < 0): L == N, Z is bit-reversed.  Bluestein: L >= 2N-1, Z natural.
template <typename T>
__device__ void ring_dft(const GeomDev &g, c2_t<T> *buf, const c2_t<T> *tw, int N, int L, int64_t bo) {
    using V = c2_t<T>;
    if (bo >= 0) {
        for (int j = threadIdx.x; j < L; j += blockDim.x) buf[j] = (j < N) ? cmul(buf[j], chirp<T>(j, N)) : mk2((T)0, (T)0);
        __syncthreads();
    }
    fft_dif<T>(buf, tw, L);
    if (bo >= 0) {
        const V *B = blu_table<T>(g) + bo;
        for (int i = threadIdx.x; i < L; i += blockDim.x) buf[i] = cmul(buf[i], B[i]);
        __syncthreads();
        fft_dit_inv<T>(buf, tw, L);
        for (int k = threadIdx.x; k < N; k += blockDim.x) buf[k] = cmul(buf[k], chirp<T>(k, N));
        __syncthreads();
    }
}

template <typename T>
__global__ void __launch_bounds__(256) ring_analysis_kernel(GeomDev g, const T *__restrict__ maps, int64_t map_stride,
                                                            const double *__restrict__ w, c2_t<T> *__restrict__ Fm,
                                                            int64_t fm_stride, int mmax, int flags, int unit_w,
                                                            int mdouble) {
    using V = c2_t<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int r = blockIdx.x, b = blockIdx.y;
    const int n = g.nphi[r], N = n >> 1, L = g.fft_len[r];
    const int64_t bo = g.blu_ofs[r];
    V *buf = reinterpret_cast<V *>(smem_raw);
    V *tw = buf + L;
    const T *f = maps + b * map_stride + g.ofs[r];
    const V *f2 = reinterpret_cast<const V *>(f);  // ring offsets are multiples of 4 samples
    for (int j = threadIdx.x; j < N; j += blockDim.x) buf[j] = f2[j];
    make_twiddles<T>(tw, L);
    __syncthreads();
    ring_dft<T>(g, buf, tw, N, L, bo);
    const int logL = ilog2(L);
    const bool direct = bo < 0;
    auto Z = [&](int k) -> V { return direct ? buf[bitrev<V>(k, logL)] : buf[k]; };

    const double twopi = 6.283185307179586476925286766559;
    const T scale = unit_w ? (T)1 : (T)(((flags & HB_F_NO2PI) ? 1.0 : twopi) * w[r] / (double)n);
    const int pair = g.ring_pair[r], side = g.ring_side[r];
    const bool has_south = g.pair_ring[2 * pair + 1] >= 0;
    const double ph = g.phi0_pi[r];
    const int64_t np = g.npairs;
    V *out = Fm + b * fm_stride;
    for (int m = threadIdx.x; m <= mmax; m += blockDim.x) {
        int k = m % n;
        bool neg = k > N;
        int kk = neg ? n - k : k;
        V zk = Z(kk == N ? 0 : kk);
        V zc = cconj(Z(kk == 0 ? 0 : N - kk));
        V A = cadd(zk, zc), D = csub(zk, zc);
        T s, c;
        sincospi_t((T)(2 * kk) / (T)n, &s, &c);
        V X = mk2((T)0.5 * (A.x - s * D.x + c * D.y), (T)0.5 * (A.y - s * D.y - c * D.x));
        if (neg) X = cconj(X);
        if (!(flags & HB_F_NOPHASE)) {
            double p = (double)m * ph;
            p -= 2.0 * floor(0.5 * p);
            T ps, pc;
            sincospi_t((T)p, &ps, &pc);
            X = cmul(X, mk2(pc, -ps));
        }
        T sc = scale;
        if (mdouble && m > 0) sc *= (T)2;
        if ((flags & HB_F_NOFOLD) && m >= n) sc = (T)0;
        X = cscale(X, sc);
        int64_t o = ((int64_t)m * np + pair) * 2;
        out[o + side] = X;
        if (!has_south) out[o + 1] = mk2((T)0, (T)0);
    }
}

template <typename T>
__global__ void __launch_bounds__(256) ring_synthesis_kernel(GeomDev g, const c2_t<T> *__restrict__ Gm,
                                                             int64_t gm_stride, int mmax, T *__restrict__ maps,
                                                             int64_t map_stride, const double *__restrict__ w,
                                                             int apply_w, int mdouble, int flags) {
    using V = c2_t<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int r = blockIdx.x, b = blockIdx.y;
    const int n = g.nphi[r], N = n >> 1, L = g.fft_len[r];
    const int64_t bo = g.blu_ofs[r];
    const bool direct = bo < 0;
    const int logL = ilog2(L);
    V *buf = reinterpret_cast<V *>(smem_raw);
    V *tw = buf + L;
    const int pair = g.ring_pair[r], side = g.ring_side[r];
    const double ph = g.phi0_pi[r];
    const int64_t np = g.npairs;
    const V *gin = Gm + b * gm_stride;
    make_twiddles<T>(tw, L);

    // T_m = c_m G(m) exp(i m phi0)
    auto Tm = [&](int m) -> V {
        V v = gin[((int64_t)m * np + pair) * 2 + side];
        if (!(flags & HB_F_NOPHASE)) {
            double p = (double)m * ph;
            p -= 2.0 * floor(0.5 * p);
            T ps, pc;
            sincospi_t((T)p, &ps, &pc);
            v = cmul(v, mk2(pc, ps));
        }
        if (mdouble && m > 0) v = cscale(v, (T)2);
        return v;
    };
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
    for (int k = threadIdx.x; k < N; k += blockDim.x) {
        V xa = Xk(k), xb = cconj(Xk(N - k));
        V S = cadd(xa, xb), D = csub(xa, xb);
        T s, c;
        sincospi_t((T)(2 * k) / (T)n, &s, &c);
        V Zv = mk2(S.x - s * D.x - c * D.y, S.y - s * D.y + c * D.x);
        if (direct)
            buf[bitrev<V>(k, logL)] = Zv;
        else
            buf[k] = cconj(Zv);  // inverse DFT as conj(DFT(conj Z))
    }
    __syncthreads();
    if (direct) {
        fft_dit_inv<T>(buf, tw, L);
    } else {
        ring_dft<T>(g, buf, tw, N, L, bo);
    }
    const double twopi = 6.283185307179586476925286766559;
    const T pscale = apply_w ? (T)(((flags & HB_F_NO2PI) ? 1.0 : twopi) * w[r] / (double)n) : (T)1;
    V *out2 = reinterpret_cast<V *>(maps + b * map_stride + g.ofs[r]);
    for (int j = threadIdx.x; j < N; j += blockDim.x) {
        V z = buf[j];
        if (!direct) z = cconj(z);
        out2[j] = cscale(z, pscale);
    }
}

// Chirp spectra for Bluestein: B = FFT_L(b)/L in bit-reversed order, b_t = exp(+i pi t^2/N)
// for |t| < N (circular), one CTA per ring, computed in place in global memory (FP64), then
// rounded to FP32 for the single-precision kernels.
__global__ void __launch_bounds__(1024) bluestein_table_kernel(GeomDev g) {
    // one CTA per distinct convolution table (rings of equal nphi share one)
    const int r = g.blu_owner[blockIdx.x];
    const int64_t bo = g.blu_ofs[r];
    const int N = g.nphi[r] >> 1, L = g.fft_len[r];
    double2 *buf = g.blu_f64 + bo;
    for (int t = threadIdx.x; t < L; t += blockDim.x) {
        int64_t j = (t < N) ? t : ((L - t < N) ? L - t : -1);
        double2 v = make_double2(0.0, 0.0);
        if (j >= 0) {
            int64_t q = (j * j) % (2 * (int64_t)N);
            double s, c;
            sincospi((double)q / (double)N, &s, &c);
            v = make_double2(c, s);
        }
        buf[t] = v;
    }
    __syncthreads();
    for (int half = L >> 1, ts = 1; half >= 1; half >>= 1, ts <<= 1) {
        for (int b = threadIdx.x; b < L / 2; b += blockDim.x) {
            int pos = b & (half - 1);
            int i = ((b - pos) << 1) + pos, j = i + half;
            double s, c;
            sincospi(-2.0 * (double)(pos * ts) / (double)L, &s, &c);
            double2 u = buf[i], v = buf[j];
            buf[i] = cadd(u, v);
            buf[j] = cmul(csub(u, v), make_double2(c, s));
        }
        __syncthreads();
    }
    const double inv = 1.0 / (double)L;
    for (int t = threadIdx.x; t < L; t += blockDim.x) {
        double2 v = make_double2(buf[t].x * inv, buf[t].y * inv);
        buf[t] = v;
        g.blu_f32[bo + t] = make_float2((float)v.x, (float)v.y);
    }
}

int build_bluestein_tables(GeomDev &g, cudaStream_t st) {
    if (g.n_blu == 0) return HB_OK;
    bluestein_table_kernel<<<(unsigned)g.n_blu, 1024, 0, st>>>(g);
    HB_CHECK_LAUNCH();
    return HB_OK;
}

int fft_smem_bytes(int L, int precision) { return (int)(1.5 * L * (precision == 32 ? 8 : 16)); }

static int max_smem_optin() {
    static int v = -1;
    if (v < 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) v = 48 * 1024;
    }
    return v;
}

template <typename T>
static int launch_analysis_t(const GeomDev &g, int nmaps, const T *maps, int64_t map_stride, const double *w,
                             c2_t<T> *Fm, int mmax, int flags, bool unit_w, bool mdouble, cudaStream_t st) {
    int smem = fft_smem_bytes(g.max_fft_len, sizeof(T) == 4 ? 32 : 64);
    if (smem > max_smem_optin())
        return fail(HB_ERR_UNSUPPORTED, "ring FFT: convolution length " + std::to_string(g.max_fft_len) +
                                            " needs " + std::to_string(smem) + " B of shared memory in this precision");
    HB_CUDA_TRY(cudaFuncSetAttribute(ring_analysis_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    dim3 grid((unsigned)g.nr, (unsigned)nmaps);
    int64_t fm_stride = (int64_t)(mmax + 1) * g.npairs * 2;
    ring_analysis_kernel<T><<<grid, 256, smem, st>>>(g, maps, map_stride, w ? w : g.w, Fm, fm_stride, mmax, flags,
                                                     unit_w ? 1 : 0, mdouble ? 1 : 0);
    HB_CHECK_LAUNCH();
    return HB_OK;
}

template <typename T>
static int launch_synthesis_t(const GeomDev &g, int nmaps, const c2_t<T> *Gm, int mmax, T *maps, int64_t map_stride,
                              const double *w, bool apply_w, bool mdouble, int flags, cudaStream_t st) {
    int smem = fft_smem_bytes(g.max_fft_len, sizeof(T) == 4 ? 32 : 64);
    if (smem > max_smem_optin())
        return fail(HB_ERR_UNSUPPORTED, "ring FFT: convolution length " + std::to_string(g.max_fft_len) +
                                            " needs " + std::to_string(smem) + " B of shared memory in this precision");
    HB_CUDA_TRY(cudaFuncSetAttribute(ring_synthesis_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    dim3 grid((unsigned)g.nr, (unsigned)nmaps);
    int64_t gm_stride = (int64_t)(mmax + 1) * g.npairs * 2;
    ring_synthesis_kernel<T><<<grid, 256, smem, st>>>(g, Gm, gm_stride, mmax, maps, map_stride, w ? w : g.w,
                                                      apply_w ? 1 : 0, mdouble ? 1 : 0, flags);
    HB_CHECK_LAUNCH();
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
