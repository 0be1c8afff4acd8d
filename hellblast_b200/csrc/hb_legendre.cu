// Fused Legendre kernels for the scalar transform (plain per-map form, FP32 and FP64).
//
// Replaces the reference's per-m pipeline (sht_raw.py:46-56: one plm_recurrence launch per m
// writing the [Nr, lmax+1] Lambda block to HBM (legendre.cu:2-35), host-side factorial norms
// (sht_raw.py:26-28, which overflow above lmax 85), a per-ring host gather of F_r[m] and a
// per-l scatter) and the synthesis loops of isht.py:11-23.
//
// One CTA per (m, block of ring pairs, map).  Each thread owns K ring pairs (north ring at
// x = cos theta, south ring at -x) and runs the normalised recursion
//     lambda_l = A_l x lambda_{l-1} + B_l lambda_{l-2},
//     A_l = sqrt((4l^2-1)/(l^2-m^2)),  B_l = -A_l sqrt(((l-1)^2-m^2)/(4(l-1)^2-1)),
// in registers, with the coefficients computed in FP64 per CTA and staged in shared memory.
// The sectoral start lambda_mm = (-1)^m sqrt((2m+1)!!/((2m)!! 4pi)) sin^m theta is formed in
// FP64 from log2 tables and carried as mantissa * 2^(S*e): while e < 0 the pair contributes
// nothing (|lambda| < 2^-S/2 relative), and the recursion rescales by 2^-S whenever the
// mantissa passes 2^(S/2), so nothing overflows or underflows up to lmax = 16383.
// Equatorial symmetry lambda_lm(-x) = (-1)^(l+m) lambda_lm(x) folds north and south rings
// into E = F_N + F_S (even l-m) and O = F_N - F_S (odd l-m).
// In FP32, x is carried as a float pair (hi + lo) so that the sample positions keep ~48 bits:
// a rounded cos(theta) shifts a ring by ~1e-7/sin(theta) rad, an l*dtheta phase error that
// reaches 1e-4 at l ~ 4000.
//
// Analysis: a_lm = sum_pairs lambda_lm(x_p) (E or O)_p.  Each thread accumulates its K pairs
// per l; TL consecutive l are staged in shared memory and reduced across the CTA.
// Synthesis: G_N/S(m) = sum_l a_lm lambda_lm (+-1)^(l-m): per-pair register accumulators, a_lm
// broadcast from shared memory, no cross-thread reduction.
#include <cmath>

#include "hb_internal.cuh"

namespace hb {

template <typename T> struct LegCfg;
template <> struct LegCfg<float> {
    static constexpr int SE = 64;  // exponent step of the running scale
    static constexpr int TL = 16;  // l values per reduction group
};
template <> struct LegCfg<double> {
    static constexpr int SE = 512;
    static constexpr int TL = 8;
};

template <typename T> struct XRep;
template <> struct XRep<float> {
    float hi, lo;
    __device__ __forceinline__ void load(const GeomDev &g, int64_t p) {
        hi = g.pair_xhi[p];
        lo = g.pair_xlo[p];
    }
    __device__ __forceinline__ float mul(float v) const { return fmaf(hi, v, lo * v); }
    __device__ __forceinline__ void zero() { hi = lo = 0.f; }
};
template <> struct XRep<double> {
    double x;
    __device__ __forceinline__ void load(const GeomDev &g, int64_t p) { x = g.pair_x[p]; }
    __device__ __forceinline__ double mul(double v) const { return x * v; }
    __device__ __forceinline__ void zero() { x = 0.0; }
};

// (A_l, B_l) of the scalar recursion, l relative to m; l = m gives (0, 1) so that the loop can
// start from the state (lambda_{m-1}, lambda_{m-2}) = (0, lambda_mm); l > lmax gives (0, 0).
__device__ __forceinline__ void scalar_coef(int l, int m, int lmax, double &A, double &B) {
    if (l == m) {
        A = 0.0;
        B = 1.0;
        return;
    }
    if (l > lmax) {
        A = B = 0.0;
        return;
    }
    double ll = l, mm = m;
    A = sqrt((4.0 * ll * ll - 1.0) / ((ll - mm) * (ll + mm)));
    B = (l - 1 > m) ? -A * sqrt(((ll - 1.0 - mm) * (ll - 1.0 + mm)) / (4.0 * (ll - 1.0) * (ll - 1.0) - 1.0)) : 0.0;
}

// start value of the scaled recursion: lambda_mm = mant * 2^(SE*e)
template <typename T>
__device__ __forceinline__ void sectoral_start(const GeomDev &g, int m, int64_t p, T &mant, int &e) {
    constexpr int SE = LegCfg<T>::SE;
    double L = g.log2cm[m] + (double)m * g.pair_log2sin[p];
    int ee = (int)floor((L + 0.5 * SE) / SE);
    double v = exp2(L - (double)SE * ee);
    mant = (T)((m & 1) ? -v : v);
    e = ee;
}

template <typename T> __device__ __forceinline__ T huge_v();
template <> __device__ __forceinline__ float huge_v<float>() { return 4294967296.0f; }        // 2^32
template <> __device__ __forceinline__ double huge_v<double>() { return 0x1p256; }
template <typename T> __device__ __forceinline__ T down_v();
template <> __device__ __forceinline__ float down_v<float>() { return 5.42101086242752217e-20f; }  // 2^-64
template <> __device__ __forceinline__ double down_v<double>() { return 0x1p-512; }

constexpr int COEF_CH = 256;  // l values per shared-memory coefficient chunk

// Evanescent skip of the FP32 synthesis: a thread's K ring pairs are consecutive, so a warp
// covers 32 K consecutive pairs.  Below its turning point a pair's recursion state has a negative
// exponent (its values kept in units 2^-64 lower) and the exponent never decreases with l; if
// every pair of the warp still has e < 0 at the checkpoint that ends the current 256-l block, the
// warp skips the block (the next block re-anchors on its checkpoint anyway), dropping
// contributions below 2^-64 of the result.  (The analysis kernel keeps its strided pair
// mapping: its per-l block reduction runs for every warp, so skipping saved nothing there.)
template <int K>
__device__ __forceinline__ bool warp_block_dead(const float4 *__restrict__ ck, const int64_t *__restrict__ blk_ofs,
                                                int m, int jnext, int64_t np, int64_t p0) {
    if (blk_ofs[m] + jnext >= blk_ofs[m + 1]) return false;  // the block reaches lmax: no end checkpoint
    const float4 *cb = ck + (blk_ofs[m] + jnext) * np;
    bool dead = true;
#pragma unroll
    for (int k = 0; k < K; ++k)
        if (p0 + k < np) dead &= __float_as_int(cb[p0 + k].z) < 0;
    return __all_sync(0xffffffffu, dead);
}

template <typename T, int K, int NT>
__global__ void __launch_bounds__(NT, 2) leg_analysis_kernel(GeomDev g, int lmax, int mmax, const c2_t<T> *__restrict__ Fm,
                                                             int64_t fm_stride, c2_t<T> *__restrict__ alm,
                                                             int64_t alm_stride, int atomic,
                                                             const float4 *__restrict__ ck,
                                                             const int64_t *__restrict__ blk_ofs,
                                                             const int32_t *__restrict__ mlist) {
    using V = c2_t<T>;
    constexpr int TL = LegCfg<T>::TL;
    constexpr int TPS = NT / TL;  // threads reducing one l slot
    static_assert(TPS >= 1 && TPS <= 32 && (32 % TPS) == 0, "bad reduction shape");
    __shared__ V coef[COEF_CH];
    extern __shared__ __align__(16) unsigned char leg_dyn_smem[];
    V(*red)[TL][NT] = reinterpret_cast<V(*)[TL][NT]>(leg_dyn_smem);  // [2][TL][NT]
    // F row blockIdx.x holds order m (all orders, or the orders of mlist in list order)
    const int m = mlist ? mlist[blockIdx.x] : blockIdx.x, chunk = blockIdx.y, b = blockIdx.z, tid = threadIdx.x;
    if (m < 0 || m > mmax) return;  // a listed order outside the plan: nothing read or written
    const int64_t np = g.npairs;
    const V *F = Fm + b * fm_stride + (int64_t)blockIdx.x * np * 2;
    V *out = alm + b * alm_stride;

    T l1[K], l2[K];
    XRep<T> x[K];
    V ge[K], go[K];
    int e[K];
    bool anyneg = false;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const int64_t p = (int64_t)chunk * NT * K + (int64_t)k * NT + tid;
        l1[k] = (T)0;
        if (p < np) {
            x[k].load(g, p);
            T mant;
            sectoral_start<T>(g, m, p, mant, e[k]);
            l2[k] = mant;
            V fn = F[2 * p], fs = F[2 * p + 1];
            ge[k] = cadd(fn, fs);
            go[k] = csub(fn, fs);
            if (e[k] < 0) {
                ge[k] = go[k] = mk2((T)0, (T)0);
                anyneg = true;
            }
        } else {
            x[k].zero();
            l2[k] = (T)0;
            e[k] = 0;
            ge[k] = go[k] = mk2((T)0, (T)0);
        }
    }

    int rb = 0;
    for (int l0 = m; l0 <= lmax; l0 += TL) {
        const int lrel = l0 - m;
        if ((lrel % COEF_CH) == 0) {
            __syncthreads();
            for (int i = tid; i < COEF_CH; i += NT) {
                double A, B;
                scalar_coef(l0 + i, m, lmax, A, B);
                coef[i] = mk2((T)A, (T)B);
            }
            __syncthreads();
            if constexpr (sizeof(T) == 4) {
                if (ck != nullptr && lrel > 0) {  // re-anchor on the FP64-computed state
                    const float4 *cb = ck + (blk_ofs[m] + lrel / COEF_CH) * np;
                    anyneg = false;
#pragma unroll
                    for (int k = 0; k < K; ++k) {
                        const int64_t p = (int64_t)chunk * NT * K + (int64_t)k * NT + tid;
                        if (p < np) {
                            const float4 c = cb[p];
                            l1[k] = c.x;
                            l2[k] = c.y;
                            const int en = __float_as_int(c.z);
                            if (en != e[k]) {
                                e[k] = en;
                                if (en == 0) {
                                    V fn = F[2 * p], fs = F[2 * p + 1];
                                    ge[k] = cadd(fn, fs);
                                    go[k] = csub(fn, fs);
                                } else {
                                    ge[k] = go[k] = mk2((T)0, (T)0);
                                }
                            }
                            anyneg |= e[k] < 0;
                        }
                    }
                }
            }
        }
        const V *cf = coef + (lrel % COEF_CH);
#pragma unroll
        for (int s = 0; s < TL; ++s) {
            const V ab = cf[s];
            T ar = (T)0, ai = (T)0;
#pragma unroll
            for (int k = 0; k < K; ++k) {
                T v = ab.x * x[k].mul(l1[k]) + ab.y * l2[k];
                l2[k] = l1[k];
                l1[k] = v;
                const V gg = (s & 1) ? go[k] : ge[k];
                ar = fma(v, gg.x, ar);
                ai = fma(v, gg.y, ai);
            }
            red[rb][s][tid] = mk2(ar, ai);
            if ((s & 3) == 3 && __any_sync(0xffffffffu, anyneg)) {
                anyneg = false;
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    if (e[k] < 0) {
                        if (fabs(l1[k]) > huge_v<T>()) {
                            l1[k] *= down_v<T>();
                            l2[k] *= down_v<T>();
                            if (++e[k] == 0) {
                                const int64_t p = (int64_t)chunk * NT * K + (int64_t)k * NT + tid;
                                V fn = F[2 * p], fs = F[2 * p + 1];
                                ge[k] = cadd(fn, fs);
                                go[k] = csub(fn, fs);
                            }
                        }
                        anyneg |= e[k] < 0;
                    }
                }
            }
        }
        __syncthreads();
        {
            const int s = tid / TPS, sub = tid % TPS;
            T rr = (T)0, ri = (T)0;
#pragma unroll
            for (int j = 0; j < TL; ++j) {
                const V v = red[rb][s][sub + j * TPS];
                rr += v.x;
                ri += v.y;
            }
#pragma unroll
            for (int off = TPS / 2; off >= 1; off >>= 1) {
                rr += __shfl_xor_sync(0xffffffffu, rr, off);
                ri += __shfl_xor_sync(0xffffffffu, ri, off);
            }
            const int l = l0 + s;
            if (sub == 0 && l <= lmax) {
                V *dst = out + alm_idx(lmax, l, m);
                if (atomic) {
                    atomicAdd(&dst->x, rr);
                    atomicAdd(&dst->y, ri);
                } else {
                    *dst = mk2(rr, ri);
                }
            }
        }
        rb ^= 1;
    }
}

template <typename T, int K, int NT>
__global__ void __launch_bounds__(NT, 2) leg_synthesis_kernel(GeomDev g, int lmax, int mmax, const c2_t<T> *__restrict__ alm,
                                                              int64_t alm_stride, c2_t<T> *__restrict__ Gm,
                                                              int64_t gm_stride, const float4 *__restrict__ ck,
                                                              const int64_t *__restrict__ blk_ofs,
                                                              const int32_t *__restrict__ mlist) {
    using V = c2_t<T>;
    __shared__ V coef[COEF_CH];
    __shared__ V acoef[COEF_CH];
    // G row blockIdx.x holds order m (all orders, or the orders of mlist in list order)
    const int m = mlist ? mlist[blockIdx.x] : blockIdx.x, chunk = blockIdx.y, b = blockIdx.z, tid = threadIdx.x;
    if (m < 0 || m > mmax) return;  // a listed order outside the plan: nothing read or written
    const int64_t np = g.npairs;
    const V *a = alm + b * alm_stride;
    V *G = Gm + b * gm_stride + (int64_t)blockIdx.x * np * 2;

    T l1[K], l2[K];
    XRep<T> x[K];
    V ae[K], ao[K];
    int e[K];
    bool anyneg = false;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const int64_t p = (int64_t)chunk * NT * K + (int64_t)tid * K + k;
        l1[k] = (T)0;
        ae[k] = ao[k] = mk2((T)0, (T)0);
        if (p < np) {
            x[k].load(g, p);
            T mant;
            sectoral_start<T>(g, m, p, mant, e[k]);
            l2[k] = mant;
            anyneg |= e[k] < 0;
        } else {
            x[k].zero();
            l2[k] = (T)0;
            e[k] = 0;
        }
    }
    bool skip = false;  // this warp's rows are all evanescent through the current block
    for (int l0 = m; l0 <= lmax; l0 += 4) {
        const int lrel = l0 - m;
        if ((lrel % COEF_CH) == 0) {
            __syncthreads();
            for (int i = tid; i < COEF_CH; i += NT) {
                double A, B;
                scalar_coef(l0 + i, m, lmax, A, B);
                coef[i] = mk2((T)A, (T)B);
                acoef[i] = (l0 + i <= lmax) ? a[alm_idx(lmax, l0 + i, m)] : mk2((T)0, (T)0);
            }
            __syncthreads();
            if constexpr (sizeof(T) == 4) {
                if (ck != nullptr && lrel > 0) {  // re-anchor on the FP64-computed state
                    const float4 *cb = ck + (blk_ofs[m] + lrel / COEF_CH) * np;
                    anyneg = false;
#pragma unroll
                    for (int k = 0; k < K; ++k) {
                        const int64_t p = (int64_t)chunk * NT * K + (int64_t)tid * K + k;
                        if (p < np) {
                            const float4 c = cb[p];
                            l1[k] = c.x;
                            l2[k] = c.y;
                            const int en = __float_as_int(c.z);
                            if (en != e[k]) {  // accumulators are kept in units of 2^(64 e)
                                const float f = ldexpf(1.0f, 64 * max(-3, e[k] - en));
                                ae[k] = cscale(ae[k], f);
                                ao[k] = cscale(ao[k], f);
                                e[k] = en;
                            }
                            anyneg |= e[k] < 0;
                        }
                    }
                }
                if (ck != nullptr)
                    skip = warp_block_dead<K>(ck, blk_ofs, m, lrel / COEF_CH + 1, np,
                                              (int64_t)chunk * NT * K + (int64_t)tid * K);
            }
        }
        if (skip) continue;
        const int i0 = lrel % COEF_CH;
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            const V ab = coef[i0 + s], av = acoef[i0 + s];
#pragma unroll
            for (int k = 0; k < K; ++k) {
                T v = ab.x * x[k].mul(l1[k]) + ab.y * l2[k];
                l2[k] = l1[k];
                l1[k] = v;
                if (s & 1) {
                    ao[k].x = fma(v, av.x, ao[k].x);
                    ao[k].y = fma(v, av.y, ao[k].y);
                } else {
                    ae[k].x = fma(v, av.x, ae[k].x);
                    ae[k].y = fma(v, av.y, ae[k].y);
                }
            }
        }
        if (__any_sync(0xffffffffu, anyneg)) {
            anyneg = false;
#pragma unroll
            for (int k = 0; k < K; ++k) {
                if (e[k] < 0) {
                    if (fabs(l1[k]) > huge_v<T>()) {
                        l1[k] *= down_v<T>();
                        l2[k] *= down_v<T>();
                        ae[k] = cscale(ae[k], down_v<T>());
                        ao[k] = cscale(ao[k], down_v<T>());
                        ++e[k];
                    }
                    anyneg |= e[k] < 0;
                }
            }
        }
    }
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const int64_t p = (int64_t)chunk * NT * K + (int64_t)tid * K + k;
        if (p < np) {
            T f = (e[k] == 0) ? (T)1 : (T)ldexp(1.0, LegCfg<T>::SE * e[k]);
            V gn = cscale(cadd(ae[k], ao[k]), f), gs = cscale(csub(ae[k], ao[k]), f);
            G[2 * p] = gn;
            G[2 * p + 1] = gs;
        }
    }
}

template <typename T, int K, int NT>
static int run_analysis(const GeomDev &g, int nmaps, int lmax, int mmax, const c2_t<T> *Fm, c2_t<T> *alm,
                        cudaStream_t st, const float4 *ck, const int64_t *bo, int nm, const int32_t *mlist) {
    const int64_t per = (int64_t)K * NT;
    const int nchunks = (int)((g.npairs + per - 1) / per);
    const int rows = mlist ? nm : mmax + 1;
    const int64_t fm_stride = (int64_t)rows * g.npairs * 2;
    const int64_t alm_stride = alm_size(lmax, mmax);
    if (nchunks > 1) HB_CUDA_TRY(cudaMemsetAsync(alm, 0, sizeof(c2_t<T>) * alm_stride * nmaps, st));
    const int smem = 2 * LegCfg<T>::TL * NT * (int)sizeof(c2_t<T>);
    HB_CUDA_TRY(cudaFuncSetAttribute(leg_analysis_kernel<T, K, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    dim3 grid((unsigned)rows, (unsigned)nchunks, (unsigned)nmaps);
    leg_analysis_kernel<T, K, NT><<<grid, NT, smem, st>>>(g, lmax, mmax, Fm, fm_stride, alm, alm_stride, nchunks > 1,
                                                           ck, bo, mlist);
    HB_CHECK_LAUNCH();
    return HB_OK;
}

template <typename T, int K, int NT>
static int run_synthesis(const GeomDev &g, int nmaps, int lmax, int mmax, const c2_t<T> *alm, c2_t<T> *Gm,
                         cudaStream_t st, const float4 *ck, const int64_t *bo, int nm, const int32_t *mlist) {
    const int64_t per = (int64_t)K * NT;
    const int nchunks = (int)((g.npairs + per - 1) / per);
    const int rows = mlist ? nm : mmax + 1;
    const int64_t gm_stride = (int64_t)rows * g.npairs * 2;
    const int64_t alm_stride = alm_size(lmax, mmax);
    dim3 grid((unsigned)rows, (unsigned)nchunks, (unsigned)nmaps);
    leg_synthesis_kernel<T, K, NT><<<grid, NT, 0, st>>>(g, lmax, mmax, alm, alm_stride, Gm, gm_stride, ck, bo, mlist);
    HB_CHECK_LAUNCH();
    return HB_OK;
}

template <typename T>
static int analysis_t(const GeomDev &g, int nmaps, int lmax, int mmax, int nm, const int32_t *mlist, const c2_t<T> *Fm, c2_t<T> *alm,
                      cudaStream_t st, const float4 *ck, const int64_t *bo) {
    if (g.npairs >= 1024) return run_analysis<T, 8, 256>(g, nmaps, lmax, mmax, Fm, alm, st, ck, bo, nm, mlist);
    if (g.npairs >= 256) return run_analysis<T, 4, 128>(g, nmaps, lmax, mmax, Fm, alm, st, ck, bo, nm, mlist);
    if (g.npairs >= 64) return run_analysis<T, 2, 64>(g, nmaps, lmax, mmax, Fm, alm, st, ck, bo, nm, mlist);
    return run_analysis<T, 1, 64>(g, nmaps, lmax, mmax, Fm, alm, st, ck, bo, nm, mlist);
}

template <typename T>
static int synthesis_t(const GeomDev &g, int nmaps, int lmax, int mmax, int nm, const int32_t *mlist, const c2_t<T> *alm, c2_t<T> *Gm,
                       cudaStream_t st, const float4 *ck, const int64_t *bo) {
    if (g.npairs >= 1024) return run_synthesis<T, 8, 256>(g, nmaps, lmax, mmax, alm, Gm, st, ck, bo, nm, mlist);
    if (g.npairs >= 256) return run_synthesis<T, 4, 128>(g, nmaps, lmax, mmax, alm, Gm, st, ck, bo, nm, mlist);
    if (g.npairs >= 64) return run_synthesis<T, 2, 64>(g, nmaps, lmax, mmax, alm, Gm, st, ck, bo, nm, mlist);
    return run_synthesis<T, 1, 64>(g, nmaps, lmax, mmax, alm, Gm, st, ck, bo, nm, mlist);
}

int launch_leg_analysis(const GeomDev &g, int precision, int nmaps, int lmax, int mmax, const void *Fm, void *alm,
                        cudaStream_t st, const float4 *ck, const int64_t *bo, int nm, const int32_t *mlist) {
    HB_NVTX("legendre_analysis");
    if (precision == 32)
        return analysis_t<float>(g, nmaps, lmax, mmax, nm, mlist, (const float2 *)Fm, (float2 *)alm, st, ck, bo);
    return analysis_t<double>(g, nmaps, lmax, mmax, nm, mlist, (const double2 *)Fm, (double2 *)alm, st, nullptr,
                              nullptr);
}

int launch_leg_synthesis(const GeomDev &g, int precision, int nmaps, int lmax, int mmax, const void *alm, void *Gm,
                         cudaStream_t st, const float4 *ck, const int64_t *bo, int nm, const int32_t *mlist) {
    HB_NVTX("legendre_synthesis");
    if (precision == 32)
        return synthesis_t<float>(g, nmaps, lmax, mmax, nm, mlist, (const float2 *)alm, (float2 *)Gm, st, ck, bo);
    return synthesis_t<double>(g, nmaps, lmax, mmax, nm, mlist, (const double2 *)alm, (double2 *)Gm, st, nullptr,
                               nullptr);
}

}  // namespace hb
