// Spin-2 (Q/U <-> E/B) Legendre kernels, FP32 and FP64.
//
// Replaces map2alm_spin_gpu / eb_from_qu_gpu / qu_from_eb_gpu (spin.py:32-115) and the
// closed-form Wigner sum wigner_d_ms_sum (wigner_d_ms.cu:20-50, one launch per (m, s), O(lmax^2)
// per ring, overflowing lgamma/exp terms).  Convention (HEALPix / Zaldarriaga-Seljak, one
// consistent choice; the reference's inverse uses a2 = -(E - iB) (spin.py:84), which contradicts
// its forward):
//     _sY_lm = _s lambda_lm(theta) e^{i m phi},   _s lambda_lm = sqrt((2l+1)/4pi) d^l_{m,-s}(theta)
//     E = -(a2 + a-2)/2,  B = i (a2 - a-2)/2,  a(+-2) = -(E +- i B).
// P = _{+2}lambda and M = _{-2}lambda on the north ring of a pair come from the three-term
// Wigner recursion in l (same a_l, c_l; opposite sign of the m*s term):
//     P_{l+1} = (a_l x + b_l) P_l - c_l P_{l-1},   M_{l+1} = (a_l x - b_l) M_l - c_l M_{l-1},
//     a_l = (N_{l+1}/N_l)(2l+1)(l+1)/R_{l+1},  b_l = (N_{l+1}/N_l)(2l+1) 2m/(l R_{l+1}),
//     c_l = (N_{l+1}/N_{l-1})(l+1) R_l/(l R_{l+1}),  R_l = sqrt((l^2-m^2)(l^2-4)),
// started at l0 = max(m,2) from the closed-form d^{l0}_{m,+-2} (log-scaled; P and M carry
// separate running exponents: their ratio near the poles is cot^4(theta/2)).
// Mirror symmetry: _s lambda(pi - theta) = (-1)^(l+m) _{-s}lambda(theta).
#include <cmath>

#include "hb_internal.cuh"

namespace hb {

template <typename T> struct SpinCfg;
template <> struct SpinCfg<float> {
    static constexpr int SE = 64;
    static constexpr int TL = 16;
};
template <> struct SpinCfg<double> {
    static constexpr int SE = 512;
    static constexpr int TL = 8;
};

template <typename T> struct V4;
template <> struct V4<float> { using type = float4; };
template <> struct V4<double> { using type = double4; };
template <typename T> using v4_t = typename V4<T>::type;
__device__ __forceinline__ float4 mk4(float a, float b, float c, float d) { return make_float4(a, b, c, d); }
__device__ __forceinline__ double4 mk4(double a, double b, double c, double d) { return make_double4(a, b, c, d); }

template <typename T> struct SXRep;
template <> struct SXRep<float> {
    float hi, lo;
    __device__ __forceinline__ void load(const GeomDev &g, int64_t p) { hi = g.pair_xhi[p]; lo = g.pair_xlo[p]; }
    __device__ __forceinline__ float mul(float v) const { return fmaf(hi, v, lo * v); }
    __device__ __forceinline__ void zero() { hi = lo = 0.f; }
};
template <> struct SXRep<double> {
    double x;
    __device__ __forceinline__ void load(const GeomDev &g, int64_t p) { x = g.pair_x[p]; }
    __device__ __forceinline__ double mul(double v) const { return x * v; }
    __device__ __forceinline__ void zero() { x = 0.0; }
};

template <typename T> __device__ __forceinline__ T s_huge();
template <> __device__ __forceinline__ float s_huge<float>() { return 4294967296.0f; }
template <> __device__ __forceinline__ double s_huge<double>() { return 0x1p256; }
template <typename T> __device__ __forceinline__ T s_down();
template <> __device__ __forceinline__ float s_down<float>() { return 5.42101086242752217e-20f; }
template <> __device__ __forceinline__ double s_down<double>() { return 0x1p-512; }

// coefficients that produce lambda_{lp} from lambda_{lp-1}, lambda_{lp-2}:
// (a, b, c) of l = lp-1; lp == l0 injects the start value held in lambda_{l0-2}; lp > lmax -> 0
__device__ __forceinline__ void spin_coef(int lp, int m, int l0, int lmax, double &a, double &b, double &c) {
    if (lp == l0) {
        a = 0.0; b = 0.0; c = -1.0;
        return;
    }
    if (lp > lmax || lp < l0) {
        a = b = c = 0.0;
        return;
    }
    const double l = lp - 1, mm = m;
    const double R1 = sqrt(((l + 1) * (l + 1) - mm * mm) * ((l + 1) * (l + 1) - 4.0));
    const double R0 = sqrt(fmax(0.0, (l * l - mm * mm) * (l * l - 4.0)));
    const double n10 = sqrt((2 * l + 3) / (2 * l + 1)), n1m = sqrt((2 * l + 3) / (2 * l - 1));
    a = n10 * (2 * l + 1) * (l + 1) / R1;
    b = n10 * (2 * l + 1) * 2.0 * mm / (l * R1);
    c = n1m * (l + 1) * R0 / (l * R1);
}

// log-scaled start values of P (s=+2 function, d_{m,-2}) and M (d_{m,+2}) at l0 = max(m,2)
template <typename T>
__device__ __forceinline__ void spin_start(const GeomDev &g, int m, int64_t p, T &mp, int &ep, T &mm, int &em) {
    constexpr int SE = SpinCfg<T>::SE;
    const double lc = g.pair_log2ch[p], ls = g.pair_log2sh[p], k = g.log2spin[m];
    const int u = m + 2, v = m >= 2 ? m - 2 : 2 - m;
    const double LP = k + v * lc + u * ls, LM = k + u * lc + v * ls;
    const double sp = (m & 1) ? -1.0 : 1.0, sm = (m >= 2) ? sp : 1.0;
    ep = (int)floor((LP + 0.5 * SE) / SE);
    em = (int)floor((LM + 0.5 * SE) / SE);
    mp = (T)(sp * exp2(LP - (double)SE * ep));
    mm = (T)(sm * exp2(LM - (double)SE * em));
}

constexpr int SCOEF_CH = 256;  // == the plan's checkpoint block length

// Per pair and parity class (even / odd l-m, slots s&1 after the l0 parity swap), the weights
//   E += P WPE + M WME,   B += P WPB + M WMB
// with, for parity eps = (-1)^(l-m):
//   Qe = QN + eps QS, Qo = QN - eps QS, Ue = UN + eps US, Uo = UN - eps US,
//   WPE = -(Qe + i Uo)/2, WME = -(Qe - i Uo)/2, WPB = -(Ue - i Qo)/2, WMB = -(Ue + i Qo)/2.
template <typename V, typename T>
__device__ __forceinline__ void spin_weights(V qn, V qs, V un, V us, T eps, V &wpe, V &wme, V &wpb, V &wmb) {
    V Qe = mk2(qn.x + eps * qs.x, qn.y + eps * qs.y), Qo = mk2(qn.x - eps * qs.x, qn.y - eps * qs.y);
    V Ue = mk2(un.x + eps * us.x, un.y + eps * us.y), Uo = mk2(un.x - eps * us.x, un.y - eps * us.y);
    const T h = (T)-0.5;
    // i*z = (-z.y, z.x)
    wpe = mk2(h * (Qe.x - Uo.y), h * (Qe.y + Uo.x));
    wme = mk2(h * (Qe.x + Uo.y), h * (Qe.y - Uo.x));
    wpb = mk2(h * (Ue.x + Qo.y), h * (Ue.y - Qo.x));
    wmb = mk2(h * (Ue.x - Qo.y), h * (Ue.y + Qo.x));
}

template <typename T, int K, int NT>
__global__ void __launch_bounds__(NT, sizeof(T) == 4 ? 4 : 1) spin_analysis_kernel(GeomDev g, int lmax, int mmax, const c2_t<T> *__restrict__ QF,
                                                           const c2_t<T> *__restrict__ UF, int64_t fm_stride,
                                                           c2_t<T> *__restrict__ Eo, c2_t<T> *__restrict__ Bo,
                                                           int64_t alm_stride, int atomic,
                                                           const float4 *__restrict__ ckP,
                                                           const float4 *__restrict__ ckM,
                                                           const int64_t *__restrict__ blk_ofs) {
    using V = c2_t<T>;
    using W = v4_t<T>;
    constexpr int TL = SpinCfg<T>::TL;
    constexpr int TPS = NT / TL;
    static_assert(TPS >= 1 && TPS <= 32 && (32 % TPS) == 0, "bad reduction shape");
    __shared__ W coef[SCOEF_CH];
    extern __shared__ __align__(16) unsigned char spin_dyn_smem[];
    W(*red)[TL][NT] = reinterpret_cast<W(*)[TL][NT]>(spin_dyn_smem);
    const int m = blockIdx.x, chunk = blockIdx.y, b = blockIdx.z, tid = threadIdx.x;
    const int l0 = m > 2 ? m : 2;
    const int par0 = (l0 - m) & 1;
    const int64_t np = g.npairs;
    const V *Qf = QF + b * fm_stride + (int64_t)m * np * 2;
    const V *Uf = UF + b * fm_stride + (int64_t)m * np * 2;
    V *Eout = Eo + b * alm_stride, *Bout = Bo + b * alm_stride;

    T P1[K], P2[K], M1[K], M2[K];
    SXRep<T> x[K];
    int ep[K], em[K];
    V wpe[2][K], wme[2][K], wpb[2][K], wmb[2][K];  // [slot parity][k]
    bool anyneg = false;
    auto load_w = [&](int k, int64_t p, bool gp, bool gm) {
        V qn = Qf[2 * p], qs = Qf[2 * p + 1], un = Uf[2 * p], us = Uf[2 * p + 1];
        for (int q = 0; q < 2; ++q) {
            // slot parity q corresponds to l-m parity q ^ par0
            T eps = ((q ^ par0) & 1) ? (T)-1 : (T)1;
            V a1, a2, a3, a4;
            spin_weights<V, T>(qn, qs, un, us, eps, a1, a2, a3, a4);
            const V z = mk2((T)0, (T)0);
            wpe[q][k] = gp ? a1 : z;
            wpb[q][k] = gp ? a3 : z;
            wme[q][k] = gm ? a2 : z;
            wmb[q][k] = gm ? a4 : z;
        }
    };
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const int64_t p = (int64_t)chunk * NT * K + (int64_t)k * NT + tid;
        P1[k] = M1[k] = (T)0;
        if (p < np) {
            x[k].load(g, p);
            spin_start<T>(g, m, p, P2[k], ep[k], M2[k], em[k]);
            load_w(k, p, ep[k] >= 0, em[k] >= 0);
            anyneg |= (ep[k] < 0) || (em[k] < 0);
        } else {
            x[k].zero();
            P2[k] = M2[k] = (T)0;
            ep[k] = em[k] = 0;
            for (int q = 0; q < 2; ++q) wpe[q][k] = wme[q][k] = wpb[q][k] = wmb[q][k] = mk2((T)0, (T)0);
        }
    }
    int rb = 0;
    for (int lb = l0; lb <= lmax; lb += TL) {
        const int lrel = lb - l0;
        if ((lrel % SCOEF_CH) == 0) {
            __syncthreads();
            for (int i = tid; i < SCOEF_CH; i += NT) {
                double a, bb, c;
                spin_coef(lb + i, m, l0, lmax, a, bb, c);
                coef[i] = mk4((T)a, (T)bb, (T)c, (T)0);
            }
            __syncthreads();
            if constexpr (sizeof(T) == 4) {
                if (ckP != nullptr && lrel > 0) {  // re-anchor both recursions on the FP64 states
                    const int64_t row = (blk_ofs[m] + lrel / SCOEF_CH) * np;
                    anyneg = false;
#pragma unroll
                    for (int k = 0; k < K; ++k) {
                        const int64_t p = (int64_t)chunk * NT * K + (int64_t)k * NT + tid;
                        if (p < np) {
                            const float4 cp = ckP[row + p], cm = ckM[row + p];
                            P1[k] = cp.x; P2[k] = cp.y; M1[k] = cm.x; M2[k] = cm.y;
                            const int np_ = __float_as_int(cp.z), nm_ = __float_as_int(cm.z);
                            if (np_ != ep[k] || nm_ != em[k]) {
                                ep[k] = np_;
                                em[k] = nm_;
                                load_w(k, p, ep[k] >= 0, em[k] >= 0);
                            }
                            anyneg |= (ep[k] < 0) || (em[k] < 0);
                        }
                    }
                }
            }
        }
        const W *cf = coef + (lrel % SCOEF_CH);
#pragma unroll
        for (int s = 0; s < TL; ++s) {
            const W cc = cf[s];
            T er = 0, ei = 0, br = 0, bi = 0;
#pragma unroll
            for (int k = 0; k < K; ++k) {
                T tp = cc.z * P2[k], tm = cc.z * M2[k];
                T vp = fma(cc.x, x[k].mul(P1[k]), fma(cc.y, P1[k], -tp));
                T vm = fma(cc.x, x[k].mul(M1[k]), fma(-cc.y, M1[k], -tm));
                P2[k] = P1[k]; P1[k] = vp;
                M2[k] = M1[k]; M1[k] = vm;
                const int q = s & 1;
                er = fma(vp, wpe[q][k].x, fma(vm, wme[q][k].x, er));
                ei = fma(vp, wpe[q][k].y, fma(vm, wme[q][k].y, ei));
                br = fma(vp, wpb[q][k].x, fma(vm, wmb[q][k].x, br));
                bi = fma(vp, wpb[q][k].y, fma(vm, wmb[q][k].y, bi));
            }
            red[rb][s][tid] = mk4(er, ei, br, bi);
            if ((s & 3) == 3 && __any_sync(0xffffffffu, anyneg)) {
                anyneg = false;
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    bool ch = false;
                    if (ep[k] < 0 && fabs(P1[k]) > s_huge<T>()) {
                        P1[k] *= s_down<T>(); P2[k] *= s_down<T>();
                        ch = (++ep[k] == 0);
                    }
                    if (em[k] < 0 && fabs(M1[k]) > s_huge<T>()) {
                        M1[k] *= s_down<T>(); M2[k] *= s_down<T>();
                        ++em[k];
                        if (em[k] == 0) ch = true;
                    }
                    if (ch) load_w(k, (int64_t)chunk * NT * K + (int64_t)k * NT + tid, ep[k] >= 0, em[k] >= 0);
                    anyneg |= (ep[k] < 0) || (em[k] < 0);
                }
            }
        }
        __syncthreads();
        {
            const int s = tid / TPS, sub = tid % TPS;
            T a0 = 0, a1 = 0, a2 = 0, a3 = 0;
#pragma unroll
            for (int j = 0; j < TL; ++j) {
                const W v = red[rb][s][sub + j * TPS];
                a0 += v.x; a1 += v.y; a2 += v.z; a3 += v.w;
            }
#pragma unroll
            for (int off = TPS / 2; off >= 1; off >>= 1) {
                a0 += __shfl_xor_sync(0xffffffffu, a0, off);
                a1 += __shfl_xor_sync(0xffffffffu, a1, off);
                a2 += __shfl_xor_sync(0xffffffffu, a2, off);
                a3 += __shfl_xor_sync(0xffffffffu, a3, off);
            }
            const int l = lb + s;
            if (sub == 0 && l <= lmax) {
                V *de = Eout + alm_idx(lmax, l, m), *db = Bout + alm_idx(lmax, l, m);
                if (atomic) {
                    atomicAdd(&de->x, a0); atomicAdd(&de->y, a1);
                    atomicAdd(&db->x, a2); atomicAdd(&db->y, a3);
                } else {
                    *de = mk2(a0, a1);
                    *db = mk2(a2, a3);
                }
            }
        }
        rb ^= 1;
    }
    // E, B are zero for l < l0 (l < 2 when m < 2)
    if (chunk == 0 && tid < 2 && m + tid < l0 && m + tid <= lmax) {
        const int l = m + tid;
        if (!atomic) {
            Eout[alm_idx(lmax, l, m)] = mk2((T)0, (T)0);
            Bout[alm_idx(lmax, l, m)] = mk2((T)0, (T)0);
        }
    }
}

template <typename T, int K, int NT>
__global__ void __launch_bounds__(NT, sizeof(T) == 4 ? 4 : 1) spin_synthesis_kernel(GeomDev g, int lmax, int mmax, const c2_t<T> *__restrict__ E,
                                                            const c2_t<T> *__restrict__ B, int64_t alm_stride,
                                                            c2_t<T> *__restrict__ QG, c2_t<T> *__restrict__ UG,
                                                            int64_t gm_stride, const float4 *__restrict__ ckP,
                                                            const float4 *__restrict__ ckM,
                                                            const int64_t *__restrict__ blk_ofs) {
    using V = c2_t<T>;
    using W = v4_t<T>;
    __shared__ W coef[SCOEF_CH];
    __shared__ W aco[SCOEF_CH];  // (A+ = E + iB, A- = E - iB)
    const int m = blockIdx.x, chunk = blockIdx.y, b = blockIdx.z, tid = threadIdx.x;
    const int l0 = m > 2 ? m : 2;
    const int par0 = (l0 - m) & 1;
    const int64_t np = g.npairs;
    const V *Eb = E + b * alm_stride, *Bb = B + b * alm_stride;
    V *Qg = QG + b * gm_stride + (int64_t)m * np * 2;
    V *Ug = UG + b * gm_stride + (int64_t)m * np * 2;

    T P1[K], P2[K], M1[K], M2[K];
    SXRep<T> x[K];
    int ep[K], em[K];
    // X1 = sum P A+, X3 = sum P A-, X2 = sum M A-, X4 = sum M A+, per slot parity
    V X1[2][K], X2[2][K], X3[2][K], X4[2][K];
    bool anyneg = false;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const int64_t p = (int64_t)chunk * NT * K + (int64_t)k * NT + tid;
        P1[k] = M1[k] = (T)0;
        for (int q = 0; q < 2; ++q) X1[q][k] = X2[q][k] = X3[q][k] = X4[q][k] = mk2((T)0, (T)0);
        if (p < np) {
            x[k].load(g, p);
            spin_start<T>(g, m, p, P2[k], ep[k], M2[k], em[k]);
            anyneg |= (ep[k] < 0) || (em[k] < 0);
        } else {
            x[k].zero();
            P2[k] = M2[k] = (T)0;
            ep[k] = em[k] = 0;
        }
    }
    for (int lb = l0; lb <= lmax; lb += 4) {
        const int lrel = lb - l0;
        if ((lrel % SCOEF_CH) == 0) {
            __syncthreads();
            for (int i = tid; i < SCOEF_CH; i += NT) {
                double a, bb, c;
                spin_coef(lb + i, m, l0, lmax, a, bb, c);
                coef[i] = mk4((T)a, (T)bb, (T)c, (T)0);
                const int l = lb + i;
                V e = mk2((T)0, (T)0), bv = mk2((T)0, (T)0);
                if (l <= lmax) {
                    e = Eb[alm_idx(lmax, l, m)];
                    bv = Bb[alm_idx(lmax, l, m)];
                }
                // E + iB, E - iB
                aco[i] = mk4(e.x - bv.y, e.y + bv.x, e.x + bv.y, e.y - bv.x);
            }
            __syncthreads();
            if constexpr (sizeof(T) == 4) {
                if (ckP != nullptr && lrel > 0) {  // re-anchor both recursions on the FP64 states
                    const int64_t row = (blk_ofs[m] + lrel / SCOEF_CH) * np;
                    anyneg = false;
#pragma unroll
                    for (int k = 0; k < K; ++k) {
                        const int64_t p = (int64_t)chunk * NT * K + (int64_t)k * NT + tid;
                        if (p < np) {
                            const float4 cp = ckP[row + p], cm = ckM[row + p];
                            P1[k] = cp.x; P2[k] = cp.y; M1[k] = cm.x; M2[k] = cm.y;
                            const int np_ = __float_as_int(cp.z), nm_ = __float_as_int(cm.z);
                            if (np_ != ep[k]) {  // accumulators are kept in units of 2^(64 e)
                                const float f = ldexpf(1.0f, 64 * max(-3, ep[k] - np_));
                                for (int q = 0; q < 2; ++q) { X1[q][k] = cscale(X1[q][k], f); X3[q][k] = cscale(X3[q][k], f); }
                                ep[k] = np_;
                            }
                            if (nm_ != em[k]) {
                                const float f = ldexpf(1.0f, 64 * max(-3, em[k] - nm_));
                                for (int q = 0; q < 2; ++q) { X2[q][k] = cscale(X2[q][k], f); X4[q][k] = cscale(X4[q][k], f); }
                                em[k] = nm_;
                            }
                            anyneg |= (ep[k] < 0) || (em[k] < 0);
                        }
                    }
                }
            }
        }
        const int i0 = lrel % SCOEF_CH;
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            const W cc = coef[i0 + s], av = aco[i0 + s];
            const int q = s & 1;
#pragma unroll
            for (int k = 0; k < K; ++k) {
                T tp = cc.z * P2[k], tm = cc.z * M2[k];
                T vp = fma(cc.x, x[k].mul(P1[k]), fma(cc.y, P1[k], -tp));
                T vm = fma(cc.x, x[k].mul(M1[k]), fma(-cc.y, M1[k], -tm));
                P2[k] = P1[k]; P1[k] = vp;
                M2[k] = M1[k]; M1[k] = vm;
                X1[q][k].x = fma(vp, av.x, X1[q][k].x); X1[q][k].y = fma(vp, av.y, X1[q][k].y);
                X3[q][k].x = fma(vp, av.z, X3[q][k].x); X3[q][k].y = fma(vp, av.w, X3[q][k].y);
                X2[q][k].x = fma(vm, av.z, X2[q][k].x); X2[q][k].y = fma(vm, av.w, X2[q][k].y);
                X4[q][k].x = fma(vm, av.x, X4[q][k].x); X4[q][k].y = fma(vm, av.y, X4[q][k].y);
            }
        }
        if (__any_sync(0xffffffffu, anyneg)) {
            anyneg = false;
#pragma unroll
            for (int k = 0; k < K; ++k) {
                if (ep[k] < 0 && fabs(P1[k]) > s_huge<T>()) {
                    P1[k] *= s_down<T>(); P2[k] *= s_down<T>();
                    for (int q = 0; q < 2; ++q) {
                        X1[q][k] = cscale(X1[q][k], s_down<T>());
                        X3[q][k] = cscale(X3[q][k], s_down<T>());
                    }
                    ++ep[k];
                }
                if (em[k] < 0 && fabs(M1[k]) > s_huge<T>()) {
                    M1[k] *= s_down<T>(); M2[k] *= s_down<T>();
                    for (int q = 0; q < 2; ++q) {
                        X2[q][k] = cscale(X2[q][k], s_down<T>());
                        X4[q][k] = cscale(X4[q][k], s_down<T>());
                    }
                    ++em[k];
                }
                anyneg |= (ep[k] < 0) || (em[k] < 0);
            }
        }
    }
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const int64_t p = (int64_t)chunk * NT * K + (int64_t)k * NT + tid;
        if (p >= np) continue;
        const T fp = ep[k] == 0 ? (T)1 : (T)ldexp(1.0, SpinCfg<T>::SE * ep[k]);
        const T fm = em[k] == 0 ? (T)1 : (T)ldexp(1.0, SpinCfg<T>::SE * em[k]);
        // slot parity q has l-m parity q ^ par0: eps = +1 for even l-m
        const int qe = par0, qo = par0 ^ 1;
        V x1e = cscale(X1[qe][k], fp), x1o = cscale(X1[qo][k], fp), x3e = cscale(X3[qe][k], fp), x3o = cscale(X3[qo][k], fp);
        V x2e = cscale(X2[qe][k], fm), x2o = cscale(X2[qo][k], fm), x4e = cscale(X4[qe][k], fm), x4o = cscale(X4[qo][k], fm);
        const T h = (T)-0.5;
        // Q_N = -1/2 sum (X1 + X2); Q_S = -1/2 sum eps (X3 + X4)
        V qn = cscale(cadd(cadd(x1e, x2e), cadd(x1o, x2o)), h);
        V qs = cscale(csub(cadd(x3e, x4e), cadd(x3o, x4o)), h);
        // U_N = -1/2 i sum (X2 - X1); U_S = -1/2 i sum eps (X3 - X4)
        V dn = cadd(csub(x2e, x1e), csub(x2o, x1o));
        V ds = csub(csub(x3e, x4e), csub(x3o, x4o));
        V un = mk2(-h * dn.y, h * dn.x);
        V us = mk2(-h * ds.y, h * ds.x);
        Qg[2 * p] = qn;
        Qg[2 * p + 1] = qs;
        Ug[2 * p] = un;
        Ug[2 * p + 1] = us;
    }
}

template <typename T, int K, int NT>
static int run_spin_analysis(const GeomDev &g, int nmaps, int lmax, int mmax, const c2_t<T> *QF, const c2_t<T> *UF,
                             c2_t<T> *E, c2_t<T> *B, cudaStream_t st, const float4 *ckP, const float4 *ckM,
                             const int64_t *bo) {
    const int64_t per = (int64_t)K * NT;
    const int nchunks = (int)((g.npairs + per - 1) / per);
    const int64_t fm_stride = (int64_t)(mmax + 1) * g.npairs * 2;
    const int64_t alm_stride = alm_size(lmax, mmax);
    if (nchunks > 1) {
        HB_CUDA_TRY(cudaMemsetAsync(E, 0, sizeof(c2_t<T>) * alm_stride * nmaps, st));
        HB_CUDA_TRY(cudaMemsetAsync(B, 0, sizeof(c2_t<T>) * alm_stride * nmaps, st));
    }
    const int smem = 2 * SpinCfg<T>::TL * NT * (int)sizeof(v4_t<T>);
    HB_CUDA_TRY(cudaFuncSetAttribute(spin_analysis_kernel<T, K, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    dim3 grid((unsigned)(mmax + 1), (unsigned)nchunks, (unsigned)nmaps);
    spin_analysis_kernel<T, K, NT><<<grid, NT, smem, st>>>(g, lmax, mmax, QF, UF, fm_stride, E, B, alm_stride,
                                                            nchunks > 1, ckP, ckM, bo);
    HB_CHECK_LAUNCH();
    return HB_OK;
}

template <typename T, int K, int NT>
static int run_spin_synthesis(const GeomDev &g, int nmaps, int lmax, int mmax, const c2_t<T> *E, const c2_t<T> *B,
                              c2_t<T> *QG, c2_t<T> *UG, cudaStream_t st, const float4 *ckP, const float4 *ckM,
                              const int64_t *bo) {
    const int64_t per = (int64_t)K * NT;
    const int nchunks = (int)((g.npairs + per - 1) / per);
    const int64_t gm_stride = (int64_t)(mmax + 1) * g.npairs * 2;
    const int64_t alm_stride = alm_size(lmax, mmax);
    dim3 grid((unsigned)(mmax + 1), (unsigned)nchunks, (unsigned)nmaps);
    spin_synthesis_kernel<T, K, NT><<<grid, NT, 0, st>>>(g, lmax, mmax, E, B, alm_stride, QG, UG, gm_stride, ckP,
                                                          ckM, bo);
    HB_CHECK_LAUNCH();
    return HB_OK;
}

template <typename T>
static int spin_analysis_t(const GeomDev &g, int nmaps, int lmax, int mmax, const c2_t<T> *QF, const c2_t<T> *UF,
                           c2_t<T> *E, c2_t<T> *B, cudaStream_t st, const float4 *ckP, const float4 *ckM,
                           const int64_t *bo) {
    if (g.npairs >= 256) return run_spin_analysis<T, 2, 128>(g, nmaps, lmax, mmax, QF, UF, E, B, st, ckP, ckM, bo);
    if (g.npairs >= 128) return run_spin_analysis<T, 2, 64>(g, nmaps, lmax, mmax, QF, UF, E, B, st, ckP, ckM, bo);
    return run_spin_analysis<T, 1, 64>(g, nmaps, lmax, mmax, QF, UF, E, B, st, ckP, ckM, bo);
}

template <typename T>
static int spin_synthesis_t(const GeomDev &g, int nmaps, int lmax, int mmax, const c2_t<T> *E, const c2_t<T> *B,
                            c2_t<T> *QG, c2_t<T> *UG, cudaStream_t st, const float4 *ckP, const float4 *ckM,
                            const int64_t *bo) {
    if (g.npairs >= 256) return run_spin_synthesis<T, 2, 128>(g, nmaps, lmax, mmax, E, B, QG, UG, st, ckP, ckM, bo);
    if (g.npairs >= 128) return run_spin_synthesis<T, 2, 64>(g, nmaps, lmax, mmax, E, B, QG, UG, st, ckP, ckM, bo);
    return run_spin_synthesis<T, 1, 64>(g, nmaps, lmax, mmax, E, B, QG, UG, st, ckP, ckM, bo);
}

int launch_spin_analysis(const GeomDev &g, int precision, int nmaps, int lmax, int mmax, const void *QFm,
                         const void *UFm, void *E, void *B, cudaStream_t st, const float4 *ckP, const float4 *ckM,
                         const int64_t *bo) {
    if (precision == 32)
        return spin_analysis_t<float>(g, nmaps, lmax, mmax, (const float2 *)QFm, (const float2 *)UFm, (float2 *)E,
                                      (float2 *)B, st, ckP, ckM, bo);
    return spin_analysis_t<double>(g, nmaps, lmax, mmax, (const double2 *)QFm, (const double2 *)UFm, (double2 *)E,
                                   (double2 *)B, st, nullptr, nullptr, nullptr);
}

int launch_spin_synthesis(const GeomDev &g, int precision, int nmaps, int lmax, int mmax, const void *E,
                          const void *B, void *QGm, void *UGm, cudaStream_t st, const float4 *ckP,
                          const float4 *ckM, const int64_t *bo) {
    if (precision == 32)
        return spin_synthesis_t<float>(g, nmaps, lmax, mmax, (const float2 *)E, (const float2 *)B, (float2 *)QGm,
                                       (float2 *)UGm, st, ckP, ckM, bo);
    return spin_synthesis_t<double>(g, nmaps, lmax, mmax, (const double2 *)E, (const double2 *)B, (double2 *)QGm,
                                    (double2 *)UGm, st, nullptr, nullptr, nullptr);
}

}  // namespace hb
