// Transform plans: a geometry plus (lmax, mmax) plus the FP64-computed recursion checkpoints
// that re-anchor the FP32 Legendre recursions.
//
// Why: in FP32 the three-term recursion lambda_l = A_l x lambda_{l-1} + B_l lambda_{l-2}
// accumulates rounding error linearly in l near the poles (where x -> 1 the recursion's
// characteristic roots merge), reaching ~1e-4 relative at l ~ 4000 for small m.  The plan stores,
// for every m, every block of R = 256 consecutive l and every ring pair, the recursion state
// (lambda_{l0-1}, lambda_{l0-2}) at the block start l0, computed by the same recursion in FP64
// and rounded to the FP32 kernels' scaled format (mantissa pair + power-of-2^64 exponent).  The
// FP32 kernels reload it at each block start, so FP32 error can only accumulate over R steps.
// The same table lets a kernel start the recursion at any block (used by the batched path).
//
// Layout: ck[(blk_ofs[m] + j) * npairs + p] = float4(mu1, mu2, bits(e), 0) for block j of m
// (block j starts at l = m + j*R for the scalar recursion, at l = max(m,2) + j*R for spin-2).
#include <cmath>
#include <vector>

#include "hb_internal.cuh"

namespace hb {

// (A_l, B_l) of the scalar recursion in FP64 (l > m)
__device__ __forceinline__ void ck_scalar_coef(int l, int m, double &A, double &B) {
    double ll = l, mm = m;
    A = sqrt((4.0 * ll * ll - 1.0) / ((ll - mm) * (ll + mm)));
    B = (l - 1 > m) ? -A * sqrt(((ll - 1.0 - mm) * (ll - 1.0 + mm)) / (4.0 * (ll - 1.0) * (ll - 1.0) - 1.0)) : 0.0;
}

// Convert an FP64 scaled state (v1, v2) * 2^(512 e) to the FP32 format (mu1, mu2) * 2^(64 ef).
__device__ __forceinline__ float4 to_f32_state(double v1, double v2, int e) {
    double ref = (v1 != 0.0) ? v1 : v2;
    if (ref == 0.0) return make_float4(0.f, 0.f, __int_as_float(0), 0.f);
    int ex;
    frexp(ref, &ex);  // |ref| in [2^(ex-1), 2^ex)
    double L = (double)ex + 512.0 * (double)e;
    int ef = (int)floor((L + 32.0) / 64.0);
    if (ef > 0) ef = 0;
    long long sh = 512LL * e - 64LL * ef;
    int shi = (int)(sh < -2000 ? -2000 : (sh > 2000 ? 2000 : sh));
    return make_float4((float)ldexp(v1, shi), (float)ldexp(v2, shi), __int_as_float(ef), 0.f);
}

constexpr int CKR = 256;   // checkpoint block length (== COEF_CH of the Legendre kernels)
constexpr int CK_NT = 128;

// ck (may be null): states at the block starts; ck_mid (may be null): states at l0 + R/2 of every
// block that reaches that far, same indexing.
// states at the start of every CKR-l block (ck), and optionally at its quarter points
// l0 + CKR/4 (ck_q1), l0 + CKR/2 (ck_mid) and l0 + 3 CKR/4 (ck_q3), same indexing; a state past
// lmax is not written
__global__ void __launch_bounds__(CK_NT) ck_scalar_kernel(GeomDev g, int lmax, const int64_t *__restrict__ blk_ofs,
                                                          float4 *__restrict__ ck, float4 *__restrict__ ck_mid,
                                                          float4 *__restrict__ ck_q1 = nullptr,
                                                          float4 *__restrict__ ck_q3 = nullptr) {
    const int m = blockIdx.x;
    const int64_t p = (int64_t)blockIdx.y * CK_NT + threadIdx.x;
    __shared__ double2 cf[CKR];
    const int64_t np = g.npairs;
    const bool live = p < np;
    double x = live ? g.pair_x[p] : 0.0;
    double L = g.log2cm[m] + (double)m * (live ? g.pair_log2sin[p] : 0.0);
    int e = (int)floor((L + 256.0) / 512.0);
    double l1 = 0.0, l2 = exp2(L - 512.0 * e);
    if (m & 1) l2 = -l2;
    const int64_t o = blk_ofs[m] * np;
    for (int l0 = m; l0 <= lmax; l0 += CKR) {
        const int64_t oj = o + (int64_t)((l0 - m) / CKR) * np + p;
        // state at the start of this block: (lambda_{l0-1}, lambda_{l0-2}); block 0 holds (0, lambda_mm)
        if (live && ck) ck[oj] = to_f32_state(l1, l2, e);
        __syncthreads();
        for (int i = threadIdx.x; i < CKR; i += CK_NT) {
            int l = l0 + i;
            double A = 0.0, B = 0.0;
            if (l == m) {
                B = 1.0;
            } else if (l <= lmax) {
                ck_scalar_coef(l, m, A, B);
            }
            cf[i] = make_double2(A, B);
        }
        __syncthreads();
        const int n = min(CKR, lmax - l0 + 1);
        for (int i = 0; i < n; ++i) {
            if (i == CKR / 2 && live && ck_mid) ck_mid[oj] = to_f32_state(l1, l2, e);
            if (i == CKR / 4 && live && ck_q1) ck_q1[oj] = to_f32_state(l1, l2, e);
            if (i == 3 * CKR / 4 && live && ck_q3) ck_q3[oj] = to_f32_state(l1, l2, e);
            double v = cf[i].x * x * l1 + cf[i].y * l2;
            l2 = l1;
            l1 = v;
            if (e < 0 && fabs(l1) > 0x1p256) {
                l1 *= 0x1p-512;
                l2 *= 0x1p-512;
                ++e;
            }
        }
    }
}

// spin-2: P (s=+2 function, recursion with +b) and M (-b), blocks from l0 = max(m,2)
__device__ __forceinline__ void ck_spin_coef(int lp, int m, double &a, double &b, double &c) {
    const double l = lp - 1, mm = m;
    const double R1 = sqrt(((l + 1) * (l + 1) - mm * mm) * ((l + 1) * (l + 1) - 4.0));
    const double R0 = sqrt(fmax(0.0, (l * l - mm * mm) * (l * l - 4.0)));
    const double n10 = sqrt((2 * l + 3) / (2 * l + 1)), n1m = sqrt((2 * l + 3) / (2 * l - 1));
    a = n10 * (2 * l + 1) * (l + 1) / R1;
    b = n10 * (2 * l + 1) * 2.0 * mm / (l * R1);
    c = n1m * (l + 1) * R0 / (l * R1);
}

__global__ void __launch_bounds__(CK_NT) ck_spin_kernel(GeomDev g, int lmax, const int64_t *__restrict__ blk_ofs,
                                                        float4 *__restrict__ ckP, float4 *__restrict__ ckM) {
    const int m = blockIdx.x;
    const int64_t p = (int64_t)blockIdx.y * CK_NT + threadIdx.x;
    __shared__ double4 cf[CKR];
    const int64_t np = g.npairs;
    const bool live = p < np;
    const int l0s = m > 2 ? m : 2;
    double x = live ? g.pair_x[p] : 0.0;
    double lc = live ? g.pair_log2ch[p] : 0.0, ls = live ? g.pair_log2sh[p] : 0.0, k = g.log2spin[m];
    const int u = m + 2, v = m >= 2 ? m - 2 : 2 - m;
    double LP = k + v * lc + u * ls, LM = k + u * lc + v * ls;
    int ep = (int)floor((LP + 256.0) / 512.0), em = (int)floor((LM + 256.0) / 512.0);
    double sp = (m & 1) ? -1.0 : 1.0, sm = (m >= 2) ? sp : 1.0;
    double P1 = 0.0, P2 = sp * exp2(LP - 512.0 * ep), M1 = 0.0, M2 = sm * exp2(LM - 512.0 * em);
    float4 *oP = ckP + blk_ofs[m] * np, *oM = ckM + blk_ofs[m] * np;
    for (int lb = l0s; lb <= lmax; lb += CKR) {
        if (live) {
            oP[(int64_t)((lb - l0s) / CKR) * np + p] = to_f32_state(P1, P2, ep);
            oM[(int64_t)((lb - l0s) / CKR) * np + p] = to_f32_state(M1, M2, em);
        }
        __syncthreads();
        for (int i = threadIdx.x; i < CKR; i += CK_NT) {
            int lp = lb + i;
            double a = 0.0, b = 0.0, c = 0.0;
            if (lp == l0s) {
                c = -1.0;
            } else if (lp <= lmax) {
                ck_spin_coef(lp, m, a, b, c);
            }
            cf[i] = make_double4(a, b, c, 0.0);
        }
        __syncthreads();
        const int n = min(CKR, lmax - lb + 1);
        for (int i = 0; i < n; ++i) {
            const double4 q = cf[i];
            double vp = (q.x * x + q.y) * P1 - q.z * P2;
            double vm = (q.x * x - q.y) * M1 - q.z * M2;
            P2 = P1; P1 = vp; M2 = M1; M1 = vm;
            if (ep < 0 && fabs(P1) > 0x1p256) { P1 *= 0x1p-512; P2 *= 0x1p-512; ++ep; }
            if (em < 0 && fabs(M1) > 0x1p256) { M1 *= 0x1p-512; M2 *= 0x1p-512; ++em; }
        }
    }
}

int launch_ck_mid(const hb_plan *p, float4 *ck_mid, float4 *ck_q1, float4 *ck_q3) {
    const int64_t np = p->g->d.npairs;
    dim3 grid((unsigned)(p->mmax + 1), (unsigned)((np + CK_NT - 1) / CK_NT));
    ck_scalar_kernel<<<grid, CK_NT>>>(p->g->d, p->lmax, p->blk_ofs, nullptr, ck_mid, ck_q1, ck_q3);
    HB_CUDA_TRY(cudaGetLastError());
    return HB_OK;
}

}  // namespace hb

using namespace hb;

static int64_t nblk(int lmax, int lstart) { return lstart > lmax ? 0 : (lmax - lstart) / CKR + 1; }

extern "C" {

int hb_plan_create(const hb_geom *g, int lmax, int mmax, int flags, hb_plan **out) {
    if (!g || !out) return fail(HB_ERR_INVALID, "hb_plan_create: null argument");
    if (lmax < 0 || lmax > HB_MAX_L || mmax < 0 || mmax > lmax)
        return fail(HB_ERR_INVALID, "hb_plan_create: need 0 <= mmax <= lmax <= 16383");
    hb_plan *p = new hb_plan();
    p->g = g;
    p->lmax = lmax;
    p->mmax = mmax;
    p->flags = flags;
    const int64_t np = g->d.npairs;
    std::vector<int64_t> ofs(mmax + 2), ofs_s(mmax + 2);
    ofs[0] = ofs_s[0] = 0;
    for (int m = 0; m <= mmax; ++m) {
        ofs[m + 1] = ofs[m] + nblk(lmax, m);
        ofs_s[m + 1] = ofs_s[m] + nblk(lmax, m > 2 ? m : 2);
    }
    const bool scalar = (flags & HB_PLAN_FP32) != 0, spin = (flags & HB_PLAN_SPIN2_FP32) != 0;
    size_t bytes = 0;
    auto carve = [&](size_t b) { size_t o = bytes; bytes += (b + 255) & ~(size_t)255; return o; };
    size_t o_ofs = carve(8 * (mmax + 2)), o_ofss = carve(8 * (mmax + 2));
    size_t o_ck = scalar ? carve(16 * (size_t)ofs[mmax + 1] * np) : 0;
    size_t o_ckp = spin ? carve(16 * (size_t)ofs_s[mmax + 1] * np) : 0;
    size_t o_ckm = spin ? carve(16 * (size_t)ofs_s[mmax + 1] * np) : 0;
    char *base = nullptr;
    if (cudaMalloc(&base, bytes) != cudaSuccess) {
        cudaGetLastError();
        delete p;
        return fail(HB_ERR_ALLOC, "hb_plan_create: cudaMalloc of " + std::to_string(bytes) + " bytes failed");
    }
    p->alloc_base = base;
    p->bytes = bytes;
    p->blk_ofs = (int64_t *)(base + o_ofs);
    p->blk_ofs_spin = (int64_t *)(base + o_ofss);
    p->ck = scalar ? (float4 *)(base + o_ck) : nullptr;
    p->ckP = spin ? (float4 *)(base + o_ckp) : nullptr;
    p->ckM = spin ? (float4 *)(base + o_ckm) : nullptr;
    int rc = HB_OK;
    if (cudaMemcpy(p->blk_ofs, ofs.data(), 8 * (mmax + 2), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(p->blk_ofs_spin, ofs_s.data(), 8 * (mmax + 2), cudaMemcpyHostToDevice) != cudaSuccess)
        rc = fail(HB_ERR_CUDA, "hb_plan_create: upload failed");
    dim3 grid((unsigned)(mmax + 1), (unsigned)((np + CK_NT - 1) / CK_NT));
    if (rc == HB_OK && scalar) {
        ck_scalar_kernel<<<grid, CK_NT>>>(g->d, lmax, p->blk_ofs, p->ck, nullptr);
        if (cudaGetLastError() != cudaSuccess) rc = fail(HB_ERR_CUDA, "hb_plan_create: checkpoint kernel launch");
    }
    if (rc == HB_OK && spin) {
        ck_spin_kernel<<<grid, CK_NT>>>(g->d, lmax, p->blk_ofs_spin, p->ckP, p->ckM);
        if (cudaGetLastError() != cudaSuccess) rc = fail(HB_ERR_CUDA, "hb_plan_create: spin checkpoint kernel launch");
    }
    if (rc == HB_OK && cudaDeviceSynchronize() != cudaSuccess) rc = fail(HB_ERR_CUDA, "hb_plan_create: table build failed");
    if (rc != HB_OK) {
        cudaFree(base);
        delete p;
        return rc;
    }
    *out = p;
    return HB_OK;
}

int hb_plan_destroy(hb_plan *p) {
    if (!p) return HB_OK;
    cudaFree(p->alloc_base);
    delete p;
    return HB_OK;
}

size_t hb_plan_bytes(const hb_plan *p) { return p ? p->bytes : 0; }

}  // extern "C"
