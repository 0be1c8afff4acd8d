// Batched split-precision Legendre transforms on the 5th-generation tensor cores (tcgen05).
//
// Many maps that share a geometry and lmax reuse every Legendre value lambda_lm(x_p): the
// contraction over l (synthesis) or over ring pairs (analysis) becomes a GEMM whose one operand
// is generated on the fly by the FP32 recursion and whose other operand is the batch.  Both
// operands are split into BF16 hi + lo parts and multiplied in three passes (hi*hi + hi*lo +
// lo*hi) with FP32 accumulation in TMEM; lambda is never written to global memory.
//
// Synthesis (alm -> G_N/S(m) per ring pair), work unit = (group, m, block of 128 ring pairs):
//   D_q[pair, n] = sum_{l = m+q mod 2} lambda_l(x_pair) a_l[n],   q = parity of l-m,
//   MMA M = 128 pairs, N = 2 * maps (Re/Im columns), K = l (32 per parity per stage).
//   Four producer warps run the recursion (one pair per thread) and write the A tiles (K-major);
//   a loader warp streams pre-split alm tiles with bulk copies; one thread issues the MMAs.
//   Epilogue: G_N = D_0 + D_1, G_S = D_0 - D_1.
// Analysis (F -> alm), work unit = (group, m, block of 256 consecutive l):
//   D_q[l, n] = sum_pairs lambda_l(x_pair) (E|O)_pair[n],  E = F_N + F_S, O = F_N - F_S,
//   MMA M = 128 l of one parity, N = 2 * maps, K = ring pairs (32 per stage).  The recursion
//   restarts at the block from the plan's FP64-computed checkpoint; three producer warps each
//   own one pipeline stage (one pair per thread, 256 steps) and write MN-major A tiles.
//
// Every mbarrier wait is bounded (ctl.wait_ns, 2 s unless a plan sets it); on expiry the kernel records an error code in
// *err and returns after releasing its tensor memory.
#include <algorithm>
#include <cmath>
#include <vector>

#include "hb_internal.cuh"
#include "hb_tc.cuh"

namespace hb {

constexpr uint64_t HB_TC_WAIT_NS = 2000000000ull;  // 2 s
// one pipeline stage of either tensor-core kernel: one MMA K-step (16 K) per parity
constexpr int TC_A_TILE = 4096;                // 128 rows x 16 K x 16-bit
constexpr int TC_A_STAGE = 4 * TC_A_TILE;      // [parity][hi/lo]
template <int N> constexpr int tc_b_stage() { return 4 * N * 32; }  // [q][h][N x 16] 16-bit

struct TcGroup {
    GeomDev g;
    int lmax, mmax, nmaps;
    int64_t npb;             // blocks of 128 pairs (synthesis)
    int64_t npc;             // chunks of 32 pairs (analysis)
    const float4 *ck;        // plan checkpoints
    const int64_t *blk_ofs;
    const float4 *ckh;       // checkpoints at l0 + 128 of every block (same indexing as ck)
    const float4 *ckq1, *ckq3;  // ... at l0 + 64 and l0 + 192 (analysis l-quarters)
    const float2 *coef;      // recursion coefficients (A_l, B_l): [(blk_ofs[m] + b) * 256 + i], l = m + 256 b + i
    // synthesis
    const uint4 *alm_tiles;  // [chunk][K-step half][4][N x 16] 16-bit, chunk = tile_ofs[m] + c
    const int64_t *alm_tile_ofs;
    float2 *Gm;              // [map][m][pair][2]
    int64_t gm_stride;
    // analysis
    const uint4 *g_tiles;    // [m][16-pair chunk][4][N x 16] 16-bit
    float *dscale;           // [mmax+1][N/2] power-of-two scale of the batch operand per (m, map column)
    int64_t alm_out_ofs;     // this group's first alm in the caller's output buffer (complex elements)
    int64_t alm_stride;
};

__device__ __forceinline__ void set_err(int *err, int code) { atomicCAS(err, 0, code); }

// Per-launch control of the tensor-core kernels: the bound of every mbarrier wait, and the
// failure-detection test switch (inject = 1: the synthesis loader of CTA 0 withholds its first
// batch-tile copy, so the waits on that stage run out and the kernel reports the error).
struct TcCtl {
    uint64_t wait_ns;
    int inject;
};

// lane 0 waits (bounded), the result is broadcast so the whole warp takes the same path
__device__ __forceinline__ bool warp_wait(uint64_t *bar, uint32_t parity, uint64_t ns) {
    bool okw = true;
    if ((threadIdx.x & 31) == 0) okw = tc::mbar_wait(bar, parity, ns);
    return __shfl_sync(0xffffffffu, (int)okw, 0) != 0;
}

// ------------------------------------------------------------------------------------ prep
// Power-of-two scale that brings the largest |value| of one m's batch operand to [2^13, 2^14):
// exact, keeps IEEE-half hi/lo parts normal over ~2^10 of dynamic range (harmless for BF16).
__device__ __forceinline__ float block_pow2_scale(float vmax) {
    __shared__ float red[32];
    for (int o = 16; o >= 1; o >>= 1) vmax = fmaxf(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = vmax;
    __syncthreads();
    float v = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 0.f;
    if (threadIdx.x < 32)
        for (int o = 16; o >= 1; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    __shared__ float res;
    if (threadIdx.x == 0) {
        int e = 0;
        if (v > 0.f) frexpf(v, &e);  // v in [2^(e-1), 2^e)
        res = (v > 0.f) ? ldexpf(1.0f, 14 - e) : 1.0f;
    }
    __syncthreads();
    return res;
}

// The prep kernels (prep_alm_tiles_kernel, prep_f_tiles_kernel) turn runs of 8 consecutive K
// positions into the hi/lo rows of the K-major core matrices (row n = 2 map + re/im; element
// (n, k) of a 16-K tile at (n%8)*8 + (n/8)*128 + (k/8)*64 + k%8), written as 16-byte stores.  Rows 8j .. 8j+7
// (maps 4j .. 4j+3) of one k8 group are one 128-byte segment, so both kernels work on quads of
// maps and let 4 lanes write one segment's interleaved rows in the same instruction (scattered
// 16-byte stores from separate instructions cost one L2 request each and ran at half the rate).
// tile set [qh][hi/lo][N rows x 16 K]; g: the k8 group (0 or 1) within the 16 K
template <bool BF16>
__device__ __forceinline__ void store_rows8(uint4 *chunk, int N, int qh, int n, int g, const float (&v)[8]) {
    constexpr int KC = 16;
    uint4 hi, lo;
    tc::split8<BF16>(v, hi, lo);
    const int64_t e = (int64_t)(2 * qh) * N * KC + (n & 7) * 8 + (n >> 3) * (8 * KC) + g * 64;  // 16-bit elements
    chunk[e / 8] = hi;
    chunk[(e + (int64_t)N * KC) / 8] = lo;
}

// alm [map][nalm] complex64 -> per (m, 64-l chunk) the synthesis B tiles
// [K-step half][q][h][N rows x 16 K] (l = l0 + 32 half + 2k + q), chunks of m covering
// l = m .. lmax (zero past lmax).
// Work item = (m, quad of 4 maps): the 4 maps' rows of one (chunk, k8 group, q, h) are one
// 128-byte segment of the tile.  F16: a first sweep over the item's alm takes the maximum |value|
// per (m, map) (the power-of-two scale, as block_pow2_scale); BF16 uses scale 1 (a power-of-two
// scale would change no bit of the result).  Then the item's l range streams through shared
// memory in stages of PA_L values of its 4 maps (8-byte cp.async, alm rows start on 8-byte
// boundaries; two stages in flight).  Thread (k8 group, parity q, map) turns its 8 values of one
// parity into the hi/lo rows 2 map (re) and 2 map + 1 (im), so the 4 lanes of one (k8 group, q)
// write the interleaved rows of one tile segment in the same instruction.  Shared-memory slot of
// (map, i = l - m - stage start): map * PA_MS + i + 2 (i / 16), which puts the 16 lanes of a
// half-warp (4 maps x 2 parities x 2 k8 groups) on distinct banks.  Map columns past the group's
// maps get zeros.
constexpr int PA_THREADS = 256, PA_L = 512, PA_MAPS = 4;
constexpr int PA_MS = 580;  // >= PA_L + 2 * (PA_L / 16) entries per map, = 4 mod 16
constexpr int PA_STAGE = PA_MAPS * PA_MS;
constexpr int PA_SMEM = 2 * PA_STAGE * (int)sizeof(float2);
__device__ __forceinline__ int pa_slot(int map, int i) { return map * PA_MS + i + 2 * (i >> 4); }
template <int N, bool BF16>
__global__ void __launch_bounds__(PA_THREADS, 4) prep_alm_tiles_kernel(const TcGroup *groups, int gi,
                                                                       const float2 *__restrict__ alm,
                                                                       int64_t alm_stride) {
    static_assert(PA_THREADS == 8 * 32 && PA_L == 32 * 16 && PA_MAPS == 4, "lane = (k8 group, parity, map)");
    static_assert(PA_MS >= PA_L + 2 * (PA_L / 16) && PA_MS % 16 == 4, "map stride");
    static_assert((N / 2) % PA_MAPS == 0, "whole map quads");
    extern __shared__ float2 sa[];
    __shared__ float red[PA_THREADS / 32][PA_MAPS];
    __shared__ float scl[PA_MAPS];
    const TcGroup &G = groups[gi];
    const int lmax = G.lmax, nq = (N / 2) / PA_MAPS, items = (G.mmax + 1) * nq;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int bl = lane & 3, q = (lane >> 2) & 1, gl = 4 * warp + (lane >> 3);  // map, parity, k8 group
    for (int item = blockIdx.x; item < items; item += gridDim.x) {
        const int m = item / nq, b0 = (item % nq) * PA_MAPS, b = b0 + bl;
        const int nl = lmax - m + 1, nch = (lmax - m + 64) / 64, nstage = (nch * 64 + PA_L - 1) / PA_L;
        const float2 *src = alm + (int64_t)b0 * alm_stride + alm_idx(lmax, m, m);  // map bb at + bb alm_stride
        float sc = 1.f;
        if constexpr (!BF16) {
            float vmax[PA_MAPS];
#pragma unroll
            for (int bb = 0; bb < PA_MAPS; ++bb) {
                vmax[bb] = 0.f;
                if (b0 + bb < G.nmaps)
                    for (int i = threadIdx.x; i < nl; i += PA_THREADS) {
                        const float2 v = __ldg(src + (int64_t)bb * alm_stride + i);
                        vmax[bb] = fmaxf(vmax[bb], fmaxf(fabsf(v.x), fabsf(v.y)));
                    }
                for (int o = 16; o >= 1; o >>= 1) vmax[bb] = fmaxf(vmax[bb], __shfl_xor_sync(0xffffffffu, vmax[bb], o));
                if (lane == 0) red[warp][bb] = vmax[bb];
            }
            __syncthreads();
            if (threadIdx.x < PA_MAPS) {
                float v = 0.f;
                for (int w = 0; w < PA_THREADS / 32; ++w) v = fmaxf(v, red[w][threadIdx.x]);
                int e = 0;
                if (v > 0.f) frexpf(v, &e);  // v in [2^(e-1), 2^e): scaled to [2^13, 2^14)
                scl[threadIdx.x] = v > 0.f ? ldexpf(1.0f, 14 - e) : 1.0f;
            }
            __syncthreads();
            sc = scl[bl];
        }
        if (threadIdx.x < PA_MAPS) G.dscale[(int64_t)m * (N / 2) + b0 + threadIdx.x] = BF16 ? 1.f : scl[threadIdx.x];
        uint4 *base = const_cast<uint4 *>(G.alm_tiles) + G.alm_tile_ofs[m] * (16 * N);
        auto issue = [&](int stg, float2 *dst) {  // one commit group: t = (map, i)
            for (int t = threadIdx.x; t < PA_MAPS * PA_L; t += PA_THREADS) {
                const int bb = t / PA_L, il = t % PA_L, i = stg * PA_L + il;
                float2 *d = dst + pa_slot(bb, il);
                if (b0 + bb < G.nmaps && i < nl)
                    tc::cp_async8(d, src + (int64_t)bb * alm_stride + i);
                else
                    *d = make_float2(0.f, 0.f);
            }
        };
        issue(0, sa);
        tc::cp_async_commit();
        for (int stg = 0; stg < nstage; ++stg) {
            const float2 *cur = sa + (stg & 1) * PA_STAGE;
            if (stg + 1 < nstage) issue(stg + 1, sa + ((stg + 1) & 1) * PA_STAGE);
            tc::cp_async_commit();
            tc::cp_async_wait<1>();  // all groups but the one just committed: stage stg is in
            __syncthreads();
            const int i0 = stg * PA_L + 16 * gl;  // l - m of this k8 group's first value
            if (i0 < nch * 64) {
                const int c = i0 >> 6, g = (i0 >> 4) & 3;
                uint4 *chunk = base + (int64_t)c * (16 * N) + (g >> 1) * (8 * N);  // K-step half g / 2
                float re[8], im[8];
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    const float2 v = cur[pa_slot(bl, 16 * gl + 2 * k + q)];
                    re[k] = v.x * sc;
                    im[k] = v.y * sc;
                }
                store_rows8<BF16>(chunk, N, q, 2 * b, g & 1, re);
                store_rows8<BF16>(chunk, N, q, 2 * b + 1, g & 1, im);
            }
            __syncthreads();  // every thread is done with this stage's buffer before it is refilled
        }
    }
    tc::cp_async_wait<0>();
}

// F [map][m/8][pair][m%8][north, south] (the m-blocked F the batched ring analysis writes, see
// fg_off) -> per (m, 16-pair chunk) the analysis B tiles [q][h][N x 16 pairs] (E = F_N + F_S
// for q = 0, O = F_N - F_S for q = 1).  Work item = (block of 8 orders, quad of 4 maps): the 8
// orders of one pair and map are one 128-byte line of F, and the 4 maps' rows of one
// (m, chunk, k8 group, q, h) are one 128-byte segment of the tile.  F16: a first sweep over the
// item's lines takes the maxima of |E|, |O| per (m, map) (the power-of-two scale, as
// block_pow2_scale); BF16 has FP32's exponent range and uses scale 1 (a power-of-two scale
// would change no bit of the result).  Then the item streams through shared memory in stages
// of PF_PAIRS pairs of its 4 maps (cp.async, two stages in flight).  Warp w converts order w;
// lane (k8 group, map) turns its 8 pairs into the hi/lo rows 2 map, 2 map + 1 of E and O, so
// the 4 lanes of one k8 group write the interleaved rows of one tile segment in the same
// instruction.  Shared-memory slot of (map, pair p, order j): map * PF_MS + 9 p + p / 8 + j
// (the 8 lanes of a quarter-warp, 4 maps x 2 k8 groups, land on distinct bank groups).  Map
// columns past the group's maps get zeros.
constexpr int PF_THREADS = 256, PF_PAIRS = 64, PF_MAPS = 4;
constexpr int PF_MS = 586;  // >= 9 * 63 + 7 + 8 entries per map, = 2 mod 8
constexpr int PF_STAGE = PF_MAPS * PF_MS;
constexpr int PF_SMEM = 2 * PF_STAGE * (int)sizeof(float4);
__device__ __forceinline__ int pf_slot(int map, int p, int j) { return map * PF_MS + 9 * p + (p >> 3) + j; }
template <int N, bool BF16>
__global__ void __launch_bounds__(PF_THREADS, 3) prep_f_tiles_kernel(const TcGroup *groups, int gi,
                                                                     const float4 *__restrict__ F, int64_t f_stride4) {
    static_assert(PF_THREADS == 32 * 8 && PF_PAIRS == 8 * 8 && PF_MAPS == 4, "warp = order, lane = (k8 group, map)");
    static_assert(PF_MS >= 9 * (PF_PAIRS - 1) + (PF_PAIRS - 1) / 8 + 8 && PF_MS % 8 == 2, "map stride");
    static_assert((N / 2) % PF_MAPS == 0, "whole map quads");
    extern __shared__ float4 sf[];
    __shared__ float red[PF_THREADS / 32][PF_MAPS * 8];
    __shared__ float scl[PF_MAPS * 8];
    const TcGroup &G = groups[gi];
    const int64_t np = G.g.npairs;
    const int npc = (int)G.npc, npad = npc * 32, nq = (N / 2) / PF_MAPS, items = (G.mmax / 8 + 1) * nq;
    const int nstage = (npad + PF_PAIRS - 1) / PF_PAIRS;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int j = warp, bl = lane & 3, g8 = lane >> 2;  // order, map in the quad, k8 group in the stage
    for (int item = blockIdx.x; item < items; item += gridDim.x) {
        const int mb = item / nq, b0 = (item % nq) * PF_MAPS, m = 8 * mb + j;
        const float4 *src = F + (int64_t)b0 * f_stride4 + (int64_t)mb * np * 8;  // map bb at + bb f_stride4
        float sc = 1.f;
        if constexpr (!BF16) {  // u = 8 p + jj: the stride keeps every thread on order jj = threadIdx.x % 8
            const int jj = threadIdx.x & 7;
            float vmax[PF_MAPS];
#pragma unroll
            for (int bb = 0; bb < PF_MAPS; ++bb) {
                vmax[bb] = 0.f;
                if (b0 + bb < G.nmaps && 8 * mb + jj <= G.mmax) {
                    const float4 *s4 = src + (int64_t)bb * f_stride4;
#pragma unroll 8
                    for (int64_t u = threadIdx.x; u < np * 8; u += PF_THREADS) {
                        const float4 f = __ldg(s4 + u);
                        vmax[bb] = fmaxf(vmax[bb], fmaxf(fmaxf(fabsf(f.x + f.z), fabsf(f.y + f.w)),
                                                         fmaxf(fabsf(f.x - f.z), fabsf(f.y - f.w))));
                    }
                }
                vmax[bb] = fmaxf(vmax[bb], __shfl_xor_sync(0xffffffffu, vmax[bb], 8));
                vmax[bb] = fmaxf(vmax[bb], __shfl_xor_sync(0xffffffffu, vmax[bb], 16));
                if (lane < 8) red[warp][bb * 8 + lane] = vmax[bb];
            }
            __syncthreads();
            if (threadIdx.x < PF_MAPS * 8) {
                float v = 0.f;
                for (int w = 0; w < PF_THREADS / 32; ++w) v = fmaxf(v, red[w][threadIdx.x]);
                int e = 0;
                if (v > 0.f) frexpf(v, &e);  // v in [2^(e-1), 2^e): scaled to [2^13, 2^14)
                scl[threadIdx.x] = v > 0.f ? ldexpf(1.0f, 14 - e) : 1.0f;
            }
            __syncthreads();
            sc = scl[bl * 8 + j];
        }
        if (threadIdx.x < PF_MAPS * 8) {  // (map b0 + t / 8, order t % 8)
            const int mm = 8 * mb + (threadIdx.x & 7);
            if (mm <= G.mmax) G.dscale[(int64_t)mm * (N / 2) + b0 + (threadIdx.x >> 3)] = BF16 ? 1.f : scl[threadIdx.x];
        }
        auto issue = [&](int stg, float4 *dst) {  // one commit group: t = (map, pair, order)
            for (int t = threadIdx.x; t < PF_MAPS * PF_PAIRS * 8; t += PF_THREADS) {
                const int jj = t & 7, pl = (t >> 3) % PF_PAIRS, bb = t / (8 * PF_PAIRS);
                const int64_t p = (int64_t)stg * PF_PAIRS + pl;
                float4 *d = dst + pf_slot(bb, pl, jj);
                if (b0 + bb < G.nmaps && p < np && 8 * mb + jj <= G.mmax)
                    tc::cp_async16(d, src + (int64_t)bb * f_stride4 + p * 8 + jj);
                else
                    *d = make_float4(0.f, 0.f, 0.f, 0.f);
            }
        };
        issue(0, sf);
        tc::cp_async_commit();
        for (int stg = 0; stg < nstage; ++stg) {
            const float4 *cur = sf + (stg & 1) * PF_STAGE;
            if (stg + 1 < nstage) issue(stg + 1, sf + ((stg + 1) & 1) * PF_STAGE);
            tc::cp_async_commit();
            tc::cp_async_wait<1>();  // all groups but the one just committed: stage stg is in
            __syncthreads();
            const int p0 = stg * PF_PAIRS + 8 * g8;
            if (m <= G.mmax && p0 < npad) {  // 16-pair chunks (the analysis kernel's stages)
                const int c = p0 >> 4, g = (p0 >> 3) & 1, b = b0 + bl;
                uint4 *chunk = const_cast<uint4 *>(G.g_tiles) + ((int64_t)m * 2 * npc + c) * (8 * N);
                float er[8], ei[8], orr[8], oi[8];
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const float4 f = cur[pf_slot(bl, 8 * g8 + i, j)];
                    er[i] = (f.x + f.z) * sc;
                    ei[i] = (f.y + f.w) * sc;
                    orr[i] = (f.x - f.z) * sc;
                    oi[i] = (f.y - f.w) * sc;
                }
                store_rows8<BF16>(chunk, N, 0, 2 * b, g, er);
                store_rows8<BF16>(chunk, N, 0, 2 * b + 1, g, ei);
                store_rows8<BF16>(chunk, N, 1, 2 * b, g, orr);
                store_rows8<BF16>(chunk, N, 1, 2 * b + 1, g, oi);
            }
            __syncthreads();  // every thread is done with this stage's buffer before it is refilled
        }
    }
    tc::cp_async_wait<0>();
}

// ------------------------------------------------------------------------------------ recursion
// One recursion step in the scaled FP32 form used by the plain kernels: lambda = mu * 2^(64 e),
// contributions only while e == 0; rescale by 2^-64 when |mu| passes 2^32 with e < 0.
struct Rec {
    float l1, l2, xh, xl;
    int e;
    // lambda_l = A (x lambda_{l-1}) + B lambda_{l-2}, four FP32 operations.  x lambda_{l-1} is
    // formed first from x = xh + xl (its rounding changes with lambda, so it does not accumulate);
    // a rounded A x would carry nearly the same relative error at every l (A_l -> 2 slowly), i.e.
    // a systematic shift of x, which the hi + lo x exists to avoid.
    __device__ __forceinline__ float step(float A, float B) {
        const float t = fmaf(xh, l1, xl * l1);
        const float v = fmaf(A, t, B * l2);
        l2 = l1;
        l1 = v;
        return v;
    }
    __device__ __forceinline__ void check() {
        if (e < 0 && fabsf(l1) > 4294967296.0f) {
            l1 *= 5.42101086242752217e-20f;
            l2 *= 5.42101086242752217e-20f;
            ++e;
        }
    }
    __device__ __forceinline__ float val(float v) const { return e == 0 ? v : 0.f; }
    // checkpoint state, values multiplied by the operand scale ls (a power of two)
    __device__ __forceinline__ void load(float4 c, float ls) {
        l1 = c.x * ls;
        l2 = c.y * ls;
        e = __float_as_int(c.z);
    }
};

// 8 even-parity and 8 odd-parity values l0+2t, l0+2t+1 (t < 8) from the coefficients cf[0..15].
// CHECKED: some row of the warp still carries a negative exponent, so values are gated and the
// state rescaled; otherwise (all rows at e == 0, the common case) neither is needed.
template <bool CHECKED>
__device__ __forceinline__ void gen16(Rec &R, const float2 *cf, float (&ev)[8], float (&od)[8]) {
    const float4 *c4 = reinterpret_cast<const float4 *>(cf);
#pragma unroll
    for (int t = 0; t < 8; ++t) {
        const float4 c = c4[t];
        ev[t] = R.step(c.x, c.y);
        if (CHECKED) ev[t] = R.val(ev[t]);
        od[t] = R.step(c.z, c.w);
        if (CHECKED) {
            od[t] = R.val(od[t]);
            if (t & 1) R.check();
        }
    }
}

__device__ __forceinline__ void coef_scalar(int l, int m, int lmax, float2 &out) {
    double A = 0.0, B = 0.0;
    if (l == m) {
        B = 1.0;
    } else if (l <= lmax) {
        const double ll = l, mm = m;
        A = sqrt((4.0 * ll * ll - 1.0) / ((ll - mm) * (ll + mm)));
        B = (l - 1 > m) ? -A * sqrt(((ll - 1.0 - mm) * (ll - 1.0 + mm)) / (4.0 * (ll - 1.0) * (ll - 1.0) - 1.0)) : 0.0;
    }
    out = make_float2((float)A, (float)B);
}

// (A_l, B_l) of every (m, l), in the plan's 256-l block layout, zero past lmax; one CTA per m.
__global__ void coef_table_kernel(int lmax, const int64_t *__restrict__ blk_ofs, float2 *__restrict__ tab) {
    const int m = blockIdx.x;
    const int64_t b0 = blk_ofs[m], nb = blk_ofs[m + 1] - b0;
    for (int64_t i = threadIdx.x; i < nb * 256; i += blockDim.x) coef_scalar(m + (int)i, m, lmax, tab[b0 * 256 + i]);
}

// Evanescent skip ranges.  Below its turning point the plan's checkpoint state of a ring pair
// carries an exponent e < 0 (|lambda| < 2^-32) and e never decreases with l, so every value before
// a checkpoint at which all rows have e < 0 is below 2^-32 (the tensor-core kernels' recursion,
// scaled by LS = 256, gates the values below 2^-40 to zeros and keeps the rest):
//   syn[m * npb + pb] = leading 128-l half-blocks of (m, pair block pb) that end at such a
//     checkpoint (checkpoint h at l = m + 128 h: h even ck, h odd the mid-block table; the
//     half-block that reaches past lmax is never skipped);
//   ana[blk_ofs[m] + jb] = leading 32-pair chunks whose rows all have e < 0 at the end of the
//     256-l block jb (none when the block reaches past lmax; at least one chunk stays).
// The kernels skip those chunks entirely (no recursion, no tile, no MMA): the values they drop are
// below 2^-32 of the normalised lambda, far under the 1e-5 error bar.
__global__ void __launch_bounds__(128) skip_table_kernel(GeomDev g, int lmax, const int64_t *__restrict__ blk_ofs,
                                                         const float4 *__restrict__ ck, const float4 *__restrict__ ckh,
                                                         int *__restrict__ syn, int *__restrict__ ana) {
    const int m = blockIdx.x;
    const int64_t np = g.npairs, b0 = blk_ofs[m], nb = blk_ofs[m + 1] - b0;
    const int npb = (int)((np + 127) / 128), npc = (int)((np + 31) / 32);
    auto dead_at = [&](const float4 *tab, int64_t blk, int64_t p) {
        return p >= np || __float_as_int(tab[blk * np + p].z) < 0;
    };
    for (int pb = 0; pb < npb; ++pb) {
        const int64_t p = (int64_t)pb * 128 + threadIdx.x;
        int hb0 = 0;
        for (int h = 1; m + 128 * h <= lmax; ++h) {
            const bool dead = (h & 1) ? dead_at(ckh, b0 + (h - 1) / 2, p) : dead_at(ck, b0 + h / 2, p);
            if (!__syncthreads_and(dead)) break;
            hb0 = h;
        }
        if (threadIdx.x == 0) syn[(int64_t)m * npb + pb] = hb0;
    }
    __shared__ int first_live;
    for (int64_t jb = 0; jb < nb; ++jb) {
        if (threadIdx.x == 0) first_live = npc * 32;
        __syncthreads();
        if (jb + 1 < nb) {
            for (int64_t p = threadIdx.x; p < np; p += blockDim.x)
                if (!dead_at(ck, b0 + jb + 1, p)) atomicMin(&first_live, (int)p);
        } else if (threadIdx.x == 0) {
            first_live = 0;
        }
        __syncthreads();
        if (threadIdx.x == 0) ana[b0 + jb] = min(first_live / 32, npc - 1);
        __syncthreads();
    }
}

// ------------------------------------------------------------------------------------ pipeline
// Both kernels: twelve producer warps generate A tiles (recursion, one ring pair per thread) and
// run the epilogue (TMEM lane quarter = warp % 4, column blocks split between the warps of one
// quarter); the next warp allocates TMEM and one of its threads issues the MMAs; one thread of
// the last warp streams the pre-split batch tiles with bulk copies.  Several producer warps per
// SM sub-partition hide the recursion's dependency latency.  The recursion restarts from the
// plan's FP64 checkpoints (every 128 l in the synthesis: block starts and the mid-block table;
// every 64 l in the analysis: the quarter tables too), which is what lets several warps share
// one row's l range.  Stages hold one 16-K MMA step per parity (TC_A_STAGE + tc_b_stage).
// synthesis: SYN_GROUPS groups of four producer warps, group g owning stages 2g and 2g + 1
constexpr int SYN_GROUPS = 3;
constexpr int SYN_PW = 4 * SYN_GROUPS;
constexpr int SYN_THREADS = 32 * (SYN_PW + 2);
// analysis: ANA_ST stages of 16 ring pairs (one MMA K-step per parity), two producer warps per
// stage, each thread one (pair, l-quarter) of the unit's 256-l block
constexpr int ANA_ST = 6;
constexpr int ANA_PW = 2 * ANA_ST;
constexpr int ANA_THREADS = 32 * (ANA_PW + 2);
// Dynamic unit queue.  The CTAs draw units from a per-launch global counter (atomicAdd) in list
// order, so a CTA that is done early takes the next unit instead of waiting out a fixed share.
// The loader's thread draws each of its CTA's units and publishes it in a shared-memory ring of
// UQ slots; every role (producer warps, MMA thread, loader) walks the ring in the same order.
// Slot i % UQ has two barriers: uq_full (one arrival: published) and uq_empty (one arrival per
// consumer: producer warp or MMA thread, read), so the drawer runs at most UQ units ahead of the
// slowest role; unit -1 ends every role's walk.
constexpr int UQ = 8;
// stages, then per producer warp 128 coefficients (float2) and 64 inverse scales, then barriers
// and the unit ring
template <int ST, int N, int PW, int STAGE = TC_A_STAGE + tc_b_stage<N>()> constexpr int tc_smem() {
    return ST * STAGE + PW * (128 * 8 + 64 * 4) + 320;
}

struct TcSmem {
    float2 *coef;  // this producer warp's 128 recursion coefficients
    float *inv;    // this producer warp's inverse batch scales 1 / (ls s_b) of the unit's m, b < 64
    uint64_t *full, *empty, *accum, *tfree, *drain;
    uint32_t *tmem_slot;
    uint64_t *uq_full, *uq_empty;  // unit ring barriers, UQ each
    int *uq;                       // unit ring slots
};
template <int ST, int N, int PW, int STAGE = TC_A_STAGE + tc_b_stage<N>()>
__device__ __forceinline__ TcSmem tc_smem_layout(uint8_t *smem, int warp) {
    const int pw = warp < PW ? warp : 0;
    TcSmem L;
    L.coef = reinterpret_cast<float2 *>(smem + ST * STAGE) + pw * 128;
    L.inv = reinterpret_cast<float *>(smem + ST * STAGE + PW * 128 * sizeof(float2)) + pw * 64;
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + ST * STAGE + PW * 128 * sizeof(float2) + PW * 64 * sizeof(float));
    L.full = bars;
    L.empty = bars + ST;
    L.accum = bars + 2 * ST;
    L.tfree = L.accum + 1;
    L.drain = L.tfree + 1;
    L.tmem_slot = reinterpret_cast<uint32_t *>(L.drain + 1);
    L.uq_full = L.drain + 2;  // after the tensor-memory slot (8 bytes)
    L.uq_empty = L.uq_full + UQ;
    L.uq = reinterpret_cast<int *>(L.uq_empty + UQ);
    static_assert(8 * (2 * ST + 3) + 8 + 16 * UQ + 4 * UQ <= 320, "barrier and ring area");
    return L;
}

template <int ST>
__device__ __forceinline__ void tc_init_barriers(const TcSmem &L, int full_count, int tfree_count, int uq_consumers) {
    for (int s = 0; s < ST; ++s) {
        tc::mbar_init(&L.full[s], full_count);
        tc::mbar_init(&L.empty[s], 1);
    }
    tc::mbar_init(L.accum, 1);
    tc::mbar_init(L.tfree, tfree_count);
    tc::mbar_init(L.drain, 1);
    for (int i = 0; i < UQ; ++i) {
        tc::mbar_init(&L.uq_full[i], 1);
        tc::mbar_init(&L.uq_empty[i], uq_consumers);
    }
    tc::fence_mbar_init();
}

// the drawer (the loader's thread): the CTA's ui-th unit from the global counter into ring slot
// ui % UQ, -1 when the list is exhausted; -2 when a role did not release the slot in time
__device__ __forceinline__ int uq_publish(const TcSmem &L, int ui, int *ctr, int nunits, uint64_t ns) {
    const int slot = ui % UQ;
    if (ui >= UQ && !tc::mbar_wait(&L.uq_empty[slot], ((ui / UQ) - 1) & 1, ns)) return -2;
    int u = atomicAdd(ctr, 1);
    if (u >= nunits) u = -1;
    L.uq[slot] = u;
    tc::mbar_arrive(&L.uq_full[slot]);  // release: the slot's value is visible to the waiters
    return u;
}
// a consumer's ui-th unit: lane 0 waits, reads the slot and releases it, the warp takes lane 0's
// value (the MMA thread calls this as lane 0 of its warp alone); -2 when nothing was published
// in time
__device__ __forceinline__ int uq_take(const TcSmem &L, int ui, uint64_t ns, bool whole_warp) {
    const int slot = ui % UQ;
    int u = -2;
    if ((threadIdx.x & 31) == 0 && tc::mbar_wait(&L.uq_full[slot], (ui / UQ) & 1, ns)) {
        u = *reinterpret_cast<volatile int *>(&L.uq[slot]);
        tc::mbar_arrive(&L.uq_empty[slot]);
    }
    return whole_warp ? __shfl_sync(0xffffffffu, u, 0) : u;
}

// the epilogue's inverse batch scales 1 / (ls s_b) of one m into this warp's table (maps b < nmaps)
__device__ __forceinline__ void load_inv_scales(float *inv, const float *scl, int nmaps, int nb, float ls) {
    for (int b = threadIdx.x & 31; b < nb; b += 32) inv[b] = b < nmaps ? 1.0f / (ls * scl[b]) : 0.f;
    __syncwarp();
}

// write 8 even + 8 odd split values of one A-tile row group: A + {0,1,2,3} * AT + off
template <bool BF16, int AT = TC_A_TILE>
__device__ __forceinline__ void store_split(uint8_t *A, int off, const float (&ev)[8], const float (&od)[8]) {
    uint4 hi, lo;
    tc::split8<BF16>(ev, hi, lo);
    *reinterpret_cast<uint4 *>(A + 0 * AT + off) = hi;
    *reinterpret_cast<uint4 *>(A + 1 * AT + off) = lo;
    tc::split8<BF16>(od, hi, lo);
    *reinterpret_cast<uint4 *>(A + 2 * AT + off) = hi;
    *reinterpret_cast<uint4 *>(A + 3 * AT + off) = lo;
}

// The MMAs of one stage (2 parities x 3 split passes, one 16-K step each).  The hi*hi products go to
// the "hi" set of a set pair, the two cross products (about 2^-11 smaller) to its "lo" set: the
// tensor core's FP32 accumulation loses about one ulp of the accumulator per MMA, so keeping the
// large products' set free of the cross products cuts the steps that round the result by 3x.
// TMEM columns of set pair j, parity q: hi at 4N j + 2N q, lo N further.  A_hi times the
// batch tiles (hi | lo), which lie back to back in shared memory, is one MMA of width 2N into
// (hi | lo); A_lo times B_hi is a second one into lo.  `first` starts the pair afresh (the
// stage's MMAs overwrite instead of accumulating).
template <int N>
__device__ __forceinline__ void issue_stage(uint32_t tmem, uint32_t a0, int pair, bool first, uint32_t idesc_n,
                                            uint32_t idesc_2n) {
    // one cta_group::1 MMA is at most 256 wide and N a multiple of 16; the 2N-wide MMA reads the
    // lo batch tile as B rows N .. 2N-1, so it must follow the hi tile directly (N * 32 bytes)
    static_assert(2 * N <= 256 && N % 16 == 0, "the hi x (hi | lo) MMA needs 2N <= 256, N % 16 == 0");
    // core matrices (8 rows x 16 bytes): 128 bytes apart along K, 256 bytes apart along the rows
    constexpr int AT = TC_A_TILE, BT = N * 32, SBO = 256;
    static_assert(4 * BT == tc_b_stage<N>(), "B tiles [q][h][N x 16]");
    const uint32_t b0 = a0 + 4 * AT;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const uint32_t d = tmem + pair * 4 * N + q * 2 * N;
        const uint64_t ah = tc::sdesc(a0 + (q * 2 + 0) * AT, 128, SBO);
        const uint64_t al = tc::sdesc(a0 + (q * 2 + 1) * AT, 128, SBO);
        const uint64_t bh = tc::sdesc(b0 + (q * 2 + 0) * BT, 128, SBO);
        tc::mma_bf16(d, ah, bh, idesc_2n, first ? 0u : 1u);  // B rows N .. 2N-1: the lo tile
        tc::mma_bf16(d + N, al, bh, idesc_n, 1u);
    }
}

// epilogue helper: columns [16j, 16j+16) of both parities, summed over the nsets accumulator sets
// (set st: pair st / 2, hi or lo by st % 2; see issue_stage)
template <int N>
__device__ __forceinline__ void load_sets(uint32_t taddr, int j, int nsets, float (&de)[16], float (&dd)[16]) {
    tc::tmem_ld16(taddr + j * 16, de);
    tc::tmem_ld16(taddr + 2 * N + j * 16, dd);
    tc::tmem_wait_ld();
    for (int st = 1; st < nsets; ++st) {
        float xe[16], xd[16];
        const uint32_t col = (uint32_t)((st >> 1) * 4 * N + (st & 1) * N);
        tc::tmem_ld16(taddr + col + j * 16, xe);
        tc::tmem_ld16(taddr + col + 2 * N + j * 16, xd);
        tc::tmem_wait_ld();
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            de[i] += xe[i];
            dd[i] += xd[i];
        }
    }
}

// ------------------------------------------------------------------------------------ synthesis
// one synthesis chunk of one row: 64 l in four groups of 8 even + 8 odd values
template <bool CHECKED, bool BF16>
__device__ __forceinline__ void gen_half_syn(Rec &R, const float2 *cf, uint8_t *A, int off) {
#pragma unroll
    for (int grp = 0; grp < 2; ++grp) {
        float ev[8], od[8];
        gen16<CHECKED>(R, cf + 16 * grp, ev, od);
        store_split<BF16, TC_A_TILE>(A, off + grp * 128, ev, od);
    }
}

// Chunk c (64 l) of a unit belongs to half-block hb = c / 2 (128 l).  The unit's live half-blocks
// hb0, hb0 + 1, ... go round-robin to SYN_GROUPS producer groups of four warps (three producer
// warps per SM sub-partition hide the recursion's latency); group g fills stages 2g (the first 32
// l of each chunk: one 16-K MMA step per parity) and 2g + 1 (the last 32 l), two chunks per
// half-block, so its producers fill one half-stage while the MMAs drain the other.  The MMA
// thread (and the batch-tile loader) take the chunks in rounds: (group 0, 1, 2) for the first
// chunk of their half-blocks, then for the second, then the next three half-blocks, each chunk's
// two half-stages in turn, so every stage is consumed in the order its group fills it.
template <int N, bool BF16, int S>
__global__ void __launch_bounds__(SYN_THREADS, 1)
    synth_tc_kernel(const TcGroup *__restrict__ groups, const int4 *__restrict__ units, int nunits, int *err,
                    int *qctr, TcCtl ctl) {
    constexpr int ST = 2 * SYN_GROUPS;
    constexpr int B_STAGE = tc_b_stage<N>();      // [q][h][N x 16] 16-bit: half a chunk's alm tiles
    constexpr int STAGE = TC_A_STAGE + B_STAGE;   // 16-K A tiles [q][h][128 x 16]
    constexpr uint32_t IDESC = tc::idesc_f16kind(128, N, 0, 0, BF16);
    constexpr uint32_t IDESC2 = tc::idesc_f16kind(128, 2 * N, 0, 0, BF16);
    // lambda scale, a power of two in both formats: |lambda| < 2^7 -> < 2^15 in IEEE half.  It
    // also sets where a row leaves its gated state (e < 0: |lambda LS| < 2^-32), so 256 moves that
    // 8 bits of lambda earlier and more chunks take the unchecked path (BF16 analysis measured
    // 22.1 -> 19.4 ms at nside 2048, 64 maps, against LS = 1)
    constexpr float LS = 256.0f;
    // S accumulator sets in S/2 (hi*hi, cross products) pairs, the k-th chunk of a unit (in MMA
    // order) using pair k mod S/2 (issue_stage): the tensor core's FP32 accumulation error grows
    // with the number of accumulate steps into one set; the epilogue sums the sets in IEEE FP32.
    constexpr int TCOLS = (2 * N * S < 32) ? 32 : 2 * N * S;
    static_assert(2 * N * S <= 512, "TMEM holds 512 columns");
    static_assert(S >= 2 && S % 2 == 0, "accumulator sets come in (hi, cross) pairs");
    extern __shared__ __align__(1024) uint8_t smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const TcSmem L = tc_smem_layout<ST, N, SYN_PW, STAGE>(smem, warp);

    if (threadIdx.x == 0) tc_init_barriers<ST>(L, 128 + 1, 32 * SYN_PW, SYN_PW + 1);
    if (warp == SYN_PW) {
        tc::tmem_alloc(L.tmem_slot, TCOLS);
        tc::tmem_relinquish();
    }
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = *L.tmem_slot;
    bool ok = true;

    if (warp < SYN_PW) {
        // ---------------- producers + epilogue
        const int wg = warp >> 2;                // producer group: stages 2 wg and 2 wg + 1
        const int r = ((warp & 3) << 5) | lane;  // row = pair within the block
        uint32_t gc = 0;  // chunks this group has filled (uses of each of its two stages)
        for (int ui = 0; ok; ++ui) {
            const int u = uq_take(L, ui, ctl.wait_ns, true);
            if (u == -2) {
                if (lane == 0) set_err(err, 6);
                ok = false;
                break;
            }
            if (u < 0) break;
            const int4 U = units[u];
            const TcGroup &G = groups[U.x];
            const int m = U.y, lmax = G.lmax;
            const int64_t np = G.g.npairs, p = (int64_t)U.z * 128 + r;
            const bool live = p < np;
            Rec R;
            R.xh = live ? G.g.pair_xhi[p] : 0.f;
            R.xl = live ? G.g.pair_xlo[p] : 0.f;
            const int nch = (lmax - m + 64) / 64, nhb = (nch + 1) / 2;
            const int c0 = U.w, hbs = c0 / 2 + wg;  // c0 is even: skips are whole half-blocks
            const int64_t b0 = G.blk_ofs[m];
            // the next half-block's coefficients and checkpoint are fetched one half-block ahead
            float2 cpre[4];
            float4 kpre = make_float4(0.f, 0.f, 0.f, 0.f);
            auto fetch = [&](int hb) {
                const int64_t blk = b0 + (hb >> 1);
#pragma unroll
                for (int i = 0; i < 4; ++i) cpre[i] = G.coef[blk * 256 + (hb & 1) * 128 + lane + 32 * i];
                kpre = live ? ((hb & 1) ? G.ckh : G.ck)[blk * np + p] : make_float4(0.f, 0.f, 0.f, 0.f);
            };
            if (hbs < nhb) fetch(hbs);
            for (int hb = hbs; hb < nhb && ok; hb += SYN_GROUPS) {
                __syncwarp();
#pragma unroll
                for (int i = 0; i < 4; ++i) L.coef[lane + 32 * i] = cpre[i];
                __syncwarp();
                R.load(kpre, LS);
                const bool fast = __all_sync(0xffffffffu, R.e == 0);
                if (hb + SYN_GROUPS < nhb) fetch(hb + SYN_GROUPS);
                for (int cc = 0; cc < 2 && 2 * hb + cc < nch && ok; ++cc, ++gc) {
                    const int off = (r & 7) * 16 + (r >> 3) * 256;  // K-major, row groups 256 bytes apart
#pragma unroll
                    for (int half = 0; half < 2; ++half) {
                        const int sg = 2 * wg + half;
                        if (gc >= 1 && !warp_wait(&L.empty[sg], (gc + 1) & 1, ctl.wait_ns)) {
                            if (lane == 0) set_err(err, 1);
                            ok = false;
                            break;
                        }
                        const float2 *cf = L.coef + cc * 64 + half * 32;
                        uint8_t *A = smem + sg * STAGE;
                        if (fast)  // one branch per half-chunk: straight-line code over its two row groups
                            gen_half_syn<false, BF16>(R, cf, A, off);
                        else
                            gen_half_syn<true, BF16>(R, cf, A, off);
                        tc::fence_proxy_async_smem();
                        tc::mbar_arrive(&L.full[sg]);
                    }
                }
            }
            if (!ok) break;
            // epilogue: this warp's lane quarter, column blocks j with j % SYN_GROUPS == wg; the
            // scales are fetched while the last MMAs drain
            load_inv_scales(L.inv, G.dscale + (int64_t)m * (N / 2), G.nmaps, N / 2, LS);
            if (!warp_wait(L.accum, ui & 1, ctl.wait_ns)) {
                if (lane == 0) set_err(err, 2);
                ok = false;
                break;
            }
            tc::fence_after();
            const uint32_t taddr = tmem + ((uint32_t)((warp & 3) * 32) << 16);
            const int nsets = 2 * (nch - c0) < S ? 2 * (nch - c0) : S;
#pragma unroll 1
            for (int j = wg; j < N / 16; j += SYN_GROUPS) {
                float de[16], dd[16];
                load_sets<N>(taddr, j, nsets, de, dd);
                if (live) {
#pragma unroll
                    for (int h = 0; h < 8; ++h) {
                        const int b = j * 8 + h;
                        if (b < G.nmaps) {
                            float2 *dst = G.Gm + (int64_t)b * G.gm_stride + ((int64_t)m * np + p) * 2;
                            const float inv = L.inv[b];
                            const float re = de[2 * h] * inv, im = de[2 * h + 1] * inv, ro = dd[2 * h] * inv,
                                        io = dd[2 * h + 1] * inv;
                            *reinterpret_cast<float4 *>(dst) = make_float4(re + ro, im + io, re - ro, im - io);
                        }
                    }
                }
            }
            tc::fence_before();
            tc::mbar_arrive(L.tfree);
        }
    } else if (warp == SYN_PW) {
        // ---------------- MMA issuer
        if (lane == 0) {
            uint32_t fbits = 0;  // bit s: parity of stage s's next fill
            for (int ui = 0; ok; ++ui) {
                const int u = uq_take(L, ui, ctl.wait_ns, false);
                if (u == -2) {
                    set_err(err, 7);
                    ok = false;
                    break;
                }
                if (u < 0) break;
                const int4 U = units[u];
                const int nch = (groups[U.x].lmax - U.y + 64) / 64, hb0 = U.w / 2, nhb = (nch + 1) / 2;
                if (ui > 0 && !tc::mbar_wait(L.tfree, (ui - 1) & 1, ctl.wait_ns)) {
                    set_err(err, 3);
                    ok = false;
                    break;
                }
                tc::fence_after();
                int k = 0;  // chunk count of this unit in MMA order
                for (int h3 = hb0; h3 < nhb && ok; h3 += SYN_GROUPS) {
                    for (int cc = 0; cc < 2 && ok; ++cc) {
                        for (int g = 0; g < SYN_GROUPS; ++g) {
                            const int hb = h3 + g;
                            if (hb >= nhb || 2 * hb + cc >= nch) continue;
                            for (int half = 0; half < 2; ++half) {
                                const int sg = 2 * g + half;
                                if (!tc::mbar_wait(&L.full[sg], (fbits >> sg) & 1u, ctl.wait_ns)) {
                                    set_err(err, 4);
                                    ok = false;
                                    break;
                                }
                                fbits ^= 1u << sg;
                                tc::fence_after();
                                // the second half accumulates onto the first
                                issue_stage<N>(tmem, tc::smem_u32(smem + sg * STAGE), k % (S / 2),
                                                  half == 0 && k < S / 2, IDESC, IDESC2);
                                tc::mma_commit(&L.empty[sg]);
                            }
                            if (!ok) break;
                            ++k;
                        }
                    }
                }
                if (!ok) break;
                tc::mma_commit(L.accum);
            }
            if (!ok) {  // let issued MMAs finish before the tensor memory is released
                tc::mma_commit(L.drain);
                tc::mbar_wait(L.drain, 0, ctl.wait_ns);
            }
        }
        __syncwarp();
    } else {
        // ---------------- loader of the pre-split alm tiles (same order as the MMA thread)
        if (lane == 0) {
            uint32_t ebits = 0, used = 0;  // bit s: parity of stage s's next drain / stage s used
            bool withheld = false;
            for (int ui = 0; ok; ++ui) {
                const int u = uq_publish(L, ui, qctr, nunits, ctl.wait_ns);
                if (u == -2) {
                    set_err(err, 8);
                    ok = false;
                    break;
                }
                if (u < 0) break;
                const int4 U = units[u];
                const TcGroup &G = groups[U.x];
                const int m = U.y;
                const int nch = (G.lmax - m + 64) / 64, hb0 = U.w / 2, nhb = (nch + 1) / 2;
                const uint4 *src = G.alm_tiles + G.alm_tile_ofs[m] * (16 * N);
                for (int h3 = hb0; h3 < nhb && ok; h3 += SYN_GROUPS) {
                    for (int cc = 0; cc < 2 && ok; ++cc) {
                        for (int g = 0; g < SYN_GROUPS; ++g) {
                            const int hb = h3 + g, c = 2 * hb + cc;
                            if (hb >= nhb || c >= nch) continue;
                            for (int half = 0; half < 2; ++half) {  // the chunk's K-step halves, 8N uint4 each
                                const int sg = 2 * g + half;
                                if (used & (1u << sg)) {
                                    if (!tc::mbar_wait(&L.empty[sg], (ebits >> sg) & 1u, ctl.wait_ns)) {
                                        set_err(err, 5);
                                        ok = false;
                                        break;
                                    }
                                    ebits ^= 1u << sg;
                                }
                                used |= 1u << sg;
                                if (ctl.inject == 1 && blockIdx.x == 0 && !withheld) {  // failure-detection test
                                    withheld = true;
                                    continue;
                                }
                                tc::mbar_arrive_expect_tx(&L.full[sg], B_STAGE);
                                tc::bulk_g2s(smem + sg * STAGE + TC_A_STAGE,
                                             src + (int64_t)c * (16 * N) + half * (8 * N), B_STAGE, &L.full[sg]);
                            }
                            if (!ok) break;
                        }
                    }
                }
            }
        }
        __syncwarp();
    }
    tc::fence_before();
    __syncthreads();
    if (warp == SYN_PW) {
        tc::fence_after();
        tc::tmem_dealloc(tmem, TCOLS);
    }
}

// ------------------------------------------------------------------------------------ analysis
// one analysis chunk of one (pair, l-quarter): 64 l in four groups of 8 even + 8 odd values,
// row groups of 8 rows 256 bytes apart (16-K tiles)
template <bool CHECKED, bool BF16>
__device__ __forceinline__ void gen_chunk_ana(Rec &R, const float2 *cf, uint8_t *A, int off0) {
#pragma unroll 2
    for (int grp = 0; grp < 4; ++grp) {
        float ev[8], od[8];
        gen16<CHECKED>(R, cf + 16 * grp, ev, od);
        store_split<BF16, TC_A_TILE>(A, off0 + grp * 256, ev, od);
    }
}
// Unit = (m, 256-l block); its chunks of 16 ring pairs go to stage c' % ANA_ST (c' = running
// chunk count).  Warps 2s and 2s + 1 fill stage s (on different SM sub-partitions): thread
// (warp w, lane) runs the recursion of pair 16 c + lane % 16 over the l-quarter
// q = 2 (w % 2) + lane / 16 of the block, the 64 l from l0 + 64 q, restarting from the plan's
// checkpoint there (block start, l0 + 64, the mid-block table, l0 + 192), and writes A-tile rows
// 32 q .. 32 q + 31 of both parities.  Twelve producer warps fill six stages at once; each stage
// is one MMA K-step per parity.
template <int N, bool BF16, int S>
__global__ void __launch_bounds__(ANA_THREADS, 1)
    anal_tc_kernel(const TcGroup *__restrict__ groups, const int4 *__restrict__ units, int nunits, float2 *alm_out,
                   int *err, int *qctr, const float *__restrict__ fl, TcCtl ctl) {
    constexpr int ST = ANA_ST;
    constexpr int B_STAGE = tc_b_stage<N>();
    constexpr int STAGE = TC_A_STAGE + B_STAGE;
    constexpr uint32_t IDESC = tc::idesc_f16kind(128, N, 1, 0, BF16);
    constexpr uint32_t IDESC2 = tc::idesc_f16kind(128, 2 * N, 1, 0, BF16);
    constexpr float LS = 256.0f;  // lambda scale: as in synth_tc_kernel
    constexpr int TCOLS = (2 * N * S < 32) ? 32 : 2 * N * S;  // S accumulator sets, see synth_tc_kernel
    static_assert(2 * N * S <= 512, "TMEM holds 512 columns");
    static_assert(S >= 2 && S % 2 == 0, "accumulator sets come in (hi, cross) pairs");
    extern __shared__ __align__(1024) uint8_t smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const TcSmem L = tc_smem_layout<ST, N, ANA_PW, STAGE>(smem, warp);

    if (threadIdx.x == 0) tc_init_barriers<ST>(L, 64 + 1, 32 * ANA_PW, ANA_PW + 1);
    if (warp == ANA_PW) {
        tc::tmem_alloc(L.tmem_slot, TCOLS);
        tc::tmem_relinquish();
    }
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = *L.tmem_slot;
    bool ok = true;

    if (warp < ANA_PW) {
        // ---------------- producers + epilogue
        const int owner = warp >> 1;                      // stage this warp fills
        const int qt = 2 * (warp & 1) + (lane >> 4);      // l-quarter of this thread
        const int pl = lane & 15;                         // pair within the chunk
        const int quarter = warp & 3, eg = warp >> 2;     // epilogue: TMEM lane quarter, column group
        uint32_t it = 0;
        for (int ui = 0; ok; ++ui) {
            const int u = uq_take(L, ui, ctl.wait_ns, true);
            if (u == -2) {
                if (lane == 0) set_err(err, 16);
                ok = false;
                break;
            }
            if (u < 0) break;
            const int4 U = units[u];
            const TcGroup &G = groups[U.x];
            const int m = U.y, jb = U.z, lmax = G.lmax;
            const int l0 = m + 256 * jb;
            const bool active = l0 + 64 * qt <= lmax;  // this quarter of the block has rows <= lmax
            const int64_t np = G.g.npairs;
            const int nck = 2 * (int)G.npc, c0 = 2 * U.w;  // 16-pair chunks (skip counts are in 32-pair chunks)
            const int64_t blk = G.blk_ofs[m] + jb;
            const float4 *ckt = qt == 0 ? G.ck : qt == 1 ? G.ckq1 : qt == 2 ? G.ckh : G.ckq3;
            __syncwarp();
#pragma unroll
            for (int i = 0; i < 4; ++i)  // the coefficients of this warp's two quarters
                L.coef[lane + 32 * i] = G.coef[blk * 256 + (warp & 1) * 128 + lane + 32 * i];
            __syncwarp();
            // this warp's next chunk (c + ST) has its checkpoint and x fetched one chunk ahead
            float4 knext = make_float4(0.f, 0.f, 0.f, 0.f);
            float xhn = 0.f, xln = 0.f;
            auto fetch = [&](int cc) {
                const int64_t pp = (int64_t)cc * 16 + pl;
                const bool lv = active && cc < nck && pp < np;
                knext = lv ? ckt[blk * np + pp] : make_float4(0.f, 0.f, 0.f, 0.f);
                xhn = lv ? G.g.pair_xhi[pp] : 0.f;
                xln = lv ? G.g.pair_xlo[pp] : 0.f;
            };
            bool first = true;
            for (int c = c0; c < nck; ++c, ++it) {
                const int s = it % ST;
                if (s != owner) continue;
                if (first) fetch(c);
                first = false;
                Rec R;
                R.xh = xhn;
                R.xl = xln;
                R.load(knext, LS);
                fetch(c + ST);
                const bool fast = __all_sync(0xffffffffu, R.e == 0);
                if (it >= ST && !warp_wait(&L.empty[s], ((it / ST) + 1) & 1, ctl.wait_ns)) {
                    if (lane == 0) set_err(err, 11);
                    ok = false;
                    break;
                }
                uint8_t *A = smem + s * STAGE;
                // MN-major 16-K tile: 8 consecutive rows (l of one parity) of pair pl at
                // (pl % 8) 16 + (pl / 8) 128, row groups 256 bytes apart; rows 32 qt ..
                const int off0 = (pl & 7) * 16 + (pl >> 3) * 128 + qt * 4 * 256;
                const float2 *cf = L.coef + (lane >> 4) * 64;
                if (fast)
                    gen_chunk_ana<false, BF16>(R, cf, A, off0);
                else
                    gen_chunk_ana<true, BF16>(R, cf, A, off0);
                tc::fence_proxy_async_smem();
                tc::mbar_arrive(&L.full[s]);
            }
            if (!ok) break;
            // epilogue: lane quarter warp % 4 = rows 32w'..32w'+31 (l = l0 + 2 row + parity),
            // column blocks j with j % 3 == warp / 4; the scales are fetched while the MMAs drain
            load_inv_scales(L.inv, G.dscale + (int64_t)m * (N / 2), G.nmaps, N / 2, LS);
            if (!warp_wait(L.accum, ui & 1, ctl.wait_ns)) {
                if (lane == 0) set_err(err, 12);
                ok = false;
                break;
            }
            tc::fence_after();
            const int row = quarter * 32 + lane;
            const int le = l0 + 2 * row;
            const uint32_t taddr = tmem + ((uint32_t)(quarter * 32) << 16);
            const int nsets = 2 * (nck - c0) < S ? 2 * (nck - c0) : S;
            // optional per-l filter (almxfl fused into the store)
            const float fl0 = fl && le <= lmax ? fl[le] : 1.f, fl1 = fl && le + 1 <= lmax ? fl[le + 1] : 1.f;
#pragma unroll 1
            for (int j = eg; j < N / 16; j += 3) {
                float de[16], dd[16];
                load_sets<N>(taddr, j, nsets, de, dd);
#pragma unroll
                for (int h = 0; h < 8; ++h) {
                    const int b = j * 8 + h;
                    if (b < G.nmaps) {
                        float2 *dst = alm_out + G.alm_out_ofs + (int64_t)b * G.alm_stride + alm_idx(lmax, le, m);
                        const float inv = L.inv[b];
                        const float f0 = fl0 * inv, f1 = fl1 * inv;
                        if (le <= lmax) dst[0] = make_float2(de[2 * h] * f0, de[2 * h + 1] * f0);
                        if (le + 1 <= lmax) dst[1] = make_float2(dd[2 * h] * f1, dd[2 * h + 1] * f1);
                    }
                }
            }
            tc::fence_before();
            tc::mbar_arrive(L.tfree);
        }
    } else if (warp == ANA_PW) {
        // ---------------- MMA issuer
        if (lane == 0) {
            uint32_t it = 0;
            for (int ui = 0; ok; ++ui) {
                const int u = uq_take(L, ui, ctl.wait_ns, false);
                if (u == -2) {
                    set_err(err, 17);
                    ok = false;
                    break;
                }
                if (u < 0) break;
                const int nck = 2 * (int)groups[units[u].x].npc, c0 = 2 * units[u].w;
                if (ui > 0 && !tc::mbar_wait(L.tfree, (ui - 1) & 1, ctl.wait_ns)) {
                    set_err(err, 13);
                    ok = false;
                    break;
                }
                tc::fence_after();
                for (int c = c0; c < nck; ++c, ++it) {
                    const int s = it % ST;
                    if (!tc::mbar_wait(&L.full[s], (it / ST) & 1, ctl.wait_ns)) {
                        set_err(err, 14);
                        ok = false;
                        break;
                    }
                    tc::fence_after();
                    issue_stage<N>(tmem, tc::smem_u32(smem + s * STAGE), (c - c0) % (S / 2), c - c0 < S / 2,
                                      IDESC, IDESC2);
                    tc::mma_commit(&L.empty[s]);
                }
                if (!ok) break;
                tc::mma_commit(L.accum);
            }
            if (!ok) {
                tc::mma_commit(L.drain);
                tc::mbar_wait(L.drain, 0, ctl.wait_ns);
            }
        }
        __syncwarp();
    } else {
        // ---------------- loader of the pre-split E/O tiles
        if (lane == 0) {
            uint32_t it = 0;
            for (int ui = 0; ok; ++ui) {
                const int u = uq_publish(L, ui, qctr, nunits, ctl.wait_ns);
                if (u == -2) {
                    set_err(err, 18);
                    ok = false;
                    break;
                }
                if (u < 0) break;
                const int4 U = units[u];
                const TcGroup &G = groups[U.x];
                const int m = U.y;
                const int nck = 2 * (int)G.npc, c0 = 2 * U.w;
                const uint4 *src = G.g_tiles + (int64_t)m * nck * (B_STAGE / 16);
                for (int c = c0; c < nck; ++c, ++it) {
                    const int s = it % ST;
                    if (it >= ST && !tc::mbar_wait(&L.empty[s], ((it / ST) + 1) & 1, ctl.wait_ns)) {
                        set_err(err, 15);
                        ok = false;
                        break;
                    }
                    tc::mbar_arrive_expect_tx(&L.full[s], B_STAGE);
                    tc::bulk_g2s(smem + s * STAGE + TC_A_STAGE, src + (int64_t)c * (B_STAGE / 16), B_STAGE, &L.full[s]);
                }
            }
        }
        __syncwarp();
    }
    tc::fence_before();
    __syncthreads();
    if (warp == ANA_PW) {
        tc::fence_after();
        tc::tmem_dealloc(tmem, TCOLS);
    }
}

// ------------------------------------------------------------------------------------ host

}  // namespace hb

using namespace hb;

struct hb_batched_plan {
    struct PlanPart {
        const hb_plan *p;
        int nmaps;
        int64_t map_ofs, alm_ofs;     // offsets of this plan's maps / alm in the caller's buffers (elements)
        // G (synthesis, m-major [nmaps][mmax+1][np][2]) / F (analysis, m-blocked [nmaps][rows/8][np][8][2],
        // rows = mmax+1 padded to a multiple of 8: fg_off) buffer; complex elements per map of each
        float2 *GF;
        int64_t gf_stride, ff_stride;
        int64_t *tile_ofs;            // device [mmax+1] alm chunk offsets
        float2 *coef;                 // recursion coefficient table (coef_table_kernel)
        float4 *ckh;                  // mid-block recursion checkpoints (launch_ck_mid)
        float4 *ckq1, *ckq3;          // quarter-block checkpoints (l0 + 64, l0 + 192)
    };
    std::vector<PlanPart> parts;
    std::vector<TcGroup> hgroups;
    std::vector<int> group_part, group_first_map;
    bool bf16 = false;
    TcGroup *dgroups = nullptr;
    int4 *syn_units = nullptr, *ana_units = nullptr;
    int n_syn = 0, n_ana = 0, N = 128;
    int *err = nullptr;
    uint64_t wait_ns = HB_TC_WAIT_NS;  // bound of every mbarrier wait of the tensor-core kernels
    int inject = 0;                    // failure-detection test switch (hb_batched_fault_test)
    void *base = nullptr;
    size_t bytes = 0;
    bool profile = false;
    cudaEvent_t ev[8] = {};  // synthesis: 0 prep 1 tensor 2 ring 3 end; analysis: 4 ring 5 prep 6 tensor 7 end
    cudaGraphExec_t graph = nullptr;  // hb_batched_graph_capture
    int64_t live_syn = 0, live_ana = 0;  // chunks the tensor kernels run after the evanescent skip
    int64_t total_maps = 0, total_pix = 0, total_alm = 0;
};

namespace hb {

static int sm_count() {
    static int v = 0;
    if (!v) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
        if (v <= 0) v = 148;
    }
    return v;
}

template <int N> constexpr int nsets() { return 512 / (2 * N) > 4 ? 4 : 512 / (2 * N); }

template <int N, bool BF16>
static int launch_syn(hb_batched_plan *bp, cudaStream_t st) {
    const int smem = tc_smem<2 * SYN_GROUPS, N, SYN_PW, TC_A_STAGE + tc_b_stage<N>()>();
    constexpr int S = nsets<N>();
    HB_CUDA_TRY(cudaFuncSetAttribute(synth_tc_kernel<N, BF16, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    const int grid = std::min(bp->n_syn, sm_count());
    HB_CUDA_TRY(cudaMemsetAsync(bp->err + 16, 0, sizeof(int), st));  // unit queue counter
    synth_tc_kernel<N, BF16, S><<<grid, SYN_THREADS, smem, st>>>(bp->dgroups, bp->syn_units, bp->n_syn, bp->err,
                                                                 bp->err + 16, TcCtl{bp->wait_ns, bp->inject});
    HB_CHECK_LAUNCH();
    return HB_OK;
}
template <int N, bool BF16>
static int launch_ana(hb_batched_plan *bp, float2 *alm_out, const float *fl, cudaStream_t st) {
    const int smem = tc_smem<ANA_ST, N, ANA_PW, TC_A_STAGE + tc_b_stage<N>()>();
    constexpr int S = nsets<N>();
    HB_CUDA_TRY(cudaFuncSetAttribute(anal_tc_kernel<N, BF16, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    const int grid = std::min(bp->n_ana, sm_count());
    HB_CUDA_TRY(cudaMemsetAsync(bp->err + 17, 0, sizeof(int), st));  // unit queue counter
    anal_tc_kernel<N, BF16, S><<<grid, ANA_THREADS, smem, st>>>(bp->dgroups, bp->ana_units, bp->n_ana, alm_out,
                                                                 bp->err, bp->err + 17, fl, TcCtl{bp->wait_ns, 0});
    HB_CHECK_LAUNCH();
    return HB_OK;
}
// prep launches: persistent CTAs over the (order or order block, map quad) items, 3 to 4 per SM
template <int N, bool BF16>
static int launch_prep_alm(hb_batched_plan *bp, int gi, const float2 *alm, int64_t stride, cudaStream_t st) {
    const TcGroup &G = bp->hgroups[gi];
    HB_CUDA_TRY(cudaFuncSetAttribute(prep_alm_tiles_kernel<N, BF16>, cudaFuncAttributeMaxDynamicSharedMemorySize, PA_SMEM));
    const int grid = std::min((G.mmax + 1) * (N / 2 / PA_MAPS), sm_count() * 4);
    prep_alm_tiles_kernel<N, BF16><<<grid, PA_THREADS, PA_SMEM, st>>>(bp->dgroups, gi, alm, stride);
    HB_CHECK_LAUNCH();
    return HB_OK;
}
// F: the group's first map in the m-blocked F (stride: complex elements per map)
template <int N, bool BF16>
static int launch_prep_f(hb_batched_plan *bp, int gi, const float2 *F, int64_t stride, cudaStream_t st) {
    const TcGroup &G = bp->hgroups[gi];
    HB_CUDA_TRY(cudaFuncSetAttribute(prep_f_tiles_kernel<N, BF16>, cudaFuncAttributeMaxDynamicSharedMemorySize, PF_SMEM));
    const int grid = std::min((G.mmax / 8 + 1) * (N / 2 / PF_MAPS), sm_count() * 3);
    prep_f_tiles_kernel<N, BF16><<<grid, PF_THREADS, PF_SMEM, st>>>(bp->dgroups, gi,
                                                                     reinterpret_cast<const float4 *>(F), stride / 2);
    HB_CHECK_LAUNCH();
    return HB_OK;
}

#define HB_DISPATCH_N(bp_, call)                                                                      \
    ((bp_)->bf16 ? ((bp_)->N == 32 ? call<32, true> : (bp_)->N == 64 ? call<64, true> : call<128, true>) \
                 : ((bp_)->N == 32 ? call<32, false> : (bp_)->N == 64 ? call<64, false> : call<128, false>))

}  // namespace hb

extern "C" {

int hb_batched_plan_create(const hb_plan *const *plans, const int *nmaps, int nplans, int flags,
                           hb_batched_plan **out) {
    if (!plans || !nmaps || nplans <= 0 || !out) return fail(HB_ERR_INVALID, "hb_batched_plan_create: bad arguments");
    hb_batched_plan *bp = new hb_batched_plan();
    bp->bf16 = (flags & HB_BATCHED_BF16) != 0;
    const int GM = (flags & HB_BATCHED_WIDE) ? 64 : 32;  // maps per group (MMA N = 2 GM)
    int maxg = 0;
    for (int i = 0; i < nplans; ++i) {
        if (!plans[i] || !plans[i]->ck || nmaps[i] <= 0) {
            delete bp;
            return fail(HB_ERR_INVALID, "hb_batched_plan_create: every plan needs HB_PLAN_FP32 and nmaps > 0");
        }
        maxg = std::max(maxg, std::min(nmaps[i], GM));
    }
    bp->N = (2 * maxg <= 32) ? 32 : (2 * maxg <= 64 ? 64 : 128);
    const int N = bp->N;
    // sizes and layout of the single allocation
    size_t total = 0;
    auto carve = [&](size_t b) { size_t o = total; total += (b + 255) & ~(size_t)255; return o; };
    struct Off { size_t gf, tofs, tiles_a, tiles_g, scales, coef, ckh, ckq1, ckq3; };
    std::vector<Off> offs(nplans);
    std::vector<std::vector<int64_t>> tile_ofs(nplans);
    std::vector<int64_t> chunks_a(nplans);
    int64_t map_ofs = 0, alm_ofs = 0;
    for (int i = 0; i < nplans; ++i) {
        const hb_plan *p = plans[i];
        const int64_t np = p->g->d.npairs;
        auto &to = tile_ofs[i];
        to.resize(p->mmax + 2);
        to[0] = 0;
        for (int m = 0; m <= p->mmax; ++m) to[m + 1] = to[m] + (p->lmax - m + 64) / 64;
        chunks_a[i] = to[p->mmax + 1];
        const int ng = (nmaps[i] + GM - 1) / GM;
        offs[i].gf = carve((size_t)nmaps[i] * fg_rows(p->mmax, true) * np * 2 * sizeof(float2));
        offs[i].tofs = carve(8 * (size_t)(p->mmax + 2));
        offs[i].tiles_a = carve((size_t)ng * chunks_a[i] * 256 * N);
        offs[i].tiles_g = carve((size_t)ng * (p->mmax + 1) * ((np + 31) / 32) * 256 * N);
        offs[i].scales = carve((size_t)ng * 4 * (p->mmax + 1) * (N / 2));
        int64_t nblocks = 0;  // 256-l blocks over all m, the plan's checkpoint layout
        for (int m = 0; m <= p->mmax; ++m) nblocks += (p->lmax - m) / 256 + 1;
        offs[i].coef = carve((size_t)nblocks * 256 * sizeof(float2));
        offs[i].ckh = carve((size_t)nblocks * np * sizeof(float4));
        offs[i].ckq1 = carve((size_t)nblocks * np * sizeof(float4));
        offs[i].ckq3 = carve((size_t)nblocks * np * sizeof(float4));
        hb_batched_plan::PlanPart part;
        part.p = p;
        part.nmaps = nmaps[i];
        part.map_ofs = map_ofs;
        part.alm_ofs = alm_ofs;
        map_ofs += (int64_t)nmaps[i] * p->g->d.npix;
        alm_ofs += (int64_t)nmaps[i] * alm_size(p->lmax, p->mmax);
        bp->parts.push_back(part);
    }
    bp->total_pix = map_ofs;
    bp->total_alm = alm_ofs;
    const size_t o_err = carve(256);
    // groups of <= 64 maps
    for (int i = 0; i < nplans; ++i) {
        const hb_plan *p = plans[i];
        const int ng = (nmaps[i] + GM - 1) / GM;
        for (int k = 0; k < ng; ++k) {
            TcGroup G{};
            G.g = p->g->d;
            G.lmax = p->lmax;
            G.mmax = p->mmax;
            G.nmaps = std::min(GM, nmaps[i] - GM * k);
            G.npb = (p->g->d.npairs + 127) / 128;
            G.npc = (p->g->d.npairs + 31) / 32;
            G.ck = p->ck;
            G.blk_ofs = p->blk_ofs;
            bp->hgroups.push_back(G);
            bp->group_part.push_back(i);
            bp->group_first_map.push_back(GM * k);
        }
    }
    const int ngroups = (int)bp->hgroups.size();
    const size_t o_groups = carve(sizeof(TcGroup) * ngroups);
    // work units (the skip counts in .w and the order by decreasing work follow once the
    // recursion tables exist)
    int64_t n_su = 0, n_au = 0;
    for (int gi = 0; gi < ngroups; ++gi) {
        const TcGroup &G = bp->hgroups[gi];
        for (int m = 0; m <= G.mmax; ++m) n_su += G.npb, n_au += (G.lmax - m) / 256 + 1;
    }
    bp->n_syn = (int)n_su;
    bp->n_ana = (int)n_au;
    const size_t o_su = carve(sizeof(int4) * n_su), o_au = carve(sizeof(int4) * n_au);
    char *base = nullptr;
    if (cudaMalloc(&base, total) != cudaSuccess) {
        cudaGetLastError();
        delete bp;
        return fail(HB_ERR_ALLOC, "hb_batched_plan_create: cudaMalloc of " + std::to_string(total) + " bytes failed");
    }
    bp->base = base;
    bp->bytes = total;
    bp->err = (int *)(base + o_err);
    bp->dgroups = (TcGroup *)(base + o_groups);
    bp->syn_units = (int4 *)(base + o_su);
    bp->ana_units = (int4 *)(base + o_au);
    for (int i = 0; i < nplans; ++i) {
        auto &part = bp->parts[i];
        part.GF = (float2 *)(base + offs[i].gf);
        part.gf_stride = fg_rows(part.p->mmax, false) * part.p->g->d.npairs * 2;
        part.ff_stride = fg_rows(part.p->mmax, true) * part.p->g->d.npairs * 2;
        part.tile_ofs = (int64_t *)(base + offs[i].tofs);
        part.coef = (float2 *)(base + offs[i].coef);
        part.ckh = (float4 *)(base + offs[i].ckh);
        part.ckq1 = (float4 *)(base + offs[i].ckq1);
        part.ckq3 = (float4 *)(base + offs[i].ckq3);
    }
    {
        int gi = 0;
        for (int i = 0; i < nplans; ++i) {
            const hb_plan *p = plans[i];
            const int ng = (nmaps[i] + GM - 1) / GM;
            for (int k = 0; k < ng; ++k, ++gi) {
                TcGroup &G = bp->hgroups[gi];
                G.alm_tiles = (const uint4 *)(base + offs[i].tiles_a) + (size_t)k * chunks_a[i] * 16 * N;
                G.alm_tile_ofs = bp->parts[i].tile_ofs;
                G.coef = bp->parts[i].coef;
                G.ckh = bp->parts[i].ckh;
                G.ckq1 = bp->parts[i].ckq1;
                G.ckq3 = bp->parts[i].ckq3;
                G.Gm = bp->parts[i].GF + (int64_t)GM * k * bp->parts[i].gf_stride;
                G.gm_stride = bp->parts[i].gf_stride;
                G.g_tiles = (const uint4 *)(base + offs[i].tiles_g) +
                            (size_t)k * (p->mmax + 1) * G.npc * 16 * N;
                G.dscale = (float *)(base + offs[i].scales) + (size_t)k * (p->mmax + 1) * (N / 2);
                G.alm_stride = alm_size(p->lmax, p->mmax);
                G.alm_out_ofs = bp->parts[i].alm_ofs + (int64_t)GM * k * G.alm_stride;
            }
        }
    }
    int rc = HB_OK;
    for (int i = 0; i < nplans && rc == HB_OK; ++i)
        if (cudaMemcpy(bp->parts[i].tile_ofs, tile_ofs[i].data(), 8 * tile_ofs[i].size(), cudaMemcpyHostToDevice) !=
            cudaSuccess)
            rc = fail(HB_ERR_CUDA, "hb_batched_plan_create: upload");
    if (rc == HB_OK &&
        (cudaMemcpy(bp->dgroups, bp->hgroups.data(), sizeof(TcGroup) * ngroups, cudaMemcpyHostToDevice) != cudaSuccess ||
         cudaMemset(bp->err, 0, sizeof(int)) != cudaSuccess))
        rc = fail(HB_ERR_CUDA, "hb_batched_plan_create: upload");
    // recursion coefficient and mid-block tables, then the evanescent skip counts of every plan
    std::vector<std::vector<int>> syn_skip(nplans), ana_skip(nplans);
    for (int i = 0; i < nplans && rc == HB_OK; ++i) {
        const hb_plan *p = plans[i];
        coef_table_kernel<<<p->mmax + 1, 256>>>(p->lmax, p->blk_ofs, bp->parts[i].coef);
        if (cudaGetLastError() != cudaSuccess || launch_ck_mid(p, bp->parts[i].ckh, bp->parts[i].ckq1, bp->parts[i].ckq3) != HB_OK ||
            cudaDeviceSynchronize() != cudaSuccess) {
            rc = fail(HB_ERR_CUDA, "hb_batched_plan_create: coefficient table");
            break;
        }
        const int64_t np = p->g->d.npairs, npb = (np + 127) / 128;
        int64_t nblocks = 0;
        for (int m = 0; m <= p->mmax; ++m) nblocks += (p->lmax - m) / 256 + 1;
        syn_skip[i].assign((size_t)(p->mmax + 1) * npb, 0);
        ana_skip[i].assign((size_t)nblocks, 0);
        int *dsk = nullptr;
        if (cudaMalloc(&dsk, sizeof(int) * (syn_skip[i].size() + ana_skip[i].size())) != cudaSuccess) {
            cudaGetLastError();
            rc = fail(HB_ERR_ALLOC, "hb_batched_plan_create: skip tables");
            break;
        }
        skip_table_kernel<<<p->mmax + 1, 128>>>(p->g->d, p->lmax, p->blk_ofs, p->ck, bp->parts[i].ckh, dsk,
                                                  dsk + syn_skip[i].size());
        if (cudaGetLastError() != cudaSuccess ||
            cudaMemcpy(syn_skip[i].data(), dsk, sizeof(int) * syn_skip[i].size(), cudaMemcpyDeviceToHost) !=
                cudaSuccess ||
            cudaMemcpy(ana_skip[i].data(), dsk + syn_skip[i].size(), sizeof(int) * ana_skip[i].size(),
                       cudaMemcpyDeviceToHost) != cudaSuccess)
            rc = fail(HB_ERR_CUDA, "hb_batched_plan_create: skip tables");
        cudaFree(dsk);
    }
    if (rc == HB_OK) {  // units with their skip counts
        std::vector<std::pair<double, int4>> su, au;
        for (int gi = 0; gi < ngroups; ++gi) {
            const TcGroup &G = bp->hgroups[gi];
            const int pi = bp->group_part[gi];
            std::vector<int64_t> bofs(G.mmax + 2, 0);
            for (int m = 0; m <= G.mmax; ++m) bofs[m + 1] = bofs[m] + (G.lmax - m) / 256 + 1;
            for (int m = 0; m <= G.mmax; ++m) {
                const int nch = (G.lmax - m + 64) / 64;
                for (int64_t pb = 0; pb < G.npb; ++pb) {
                    const int c0 = 2 * syn_skip[pi][(size_t)m * G.npb + pb];
                    su.push_back({-(double)(nch - c0) * N, make_int4(gi, m, (int)pb, c0)});
                }
                for (int jb = 0; m + 256 * jb <= G.lmax; ++jb) {
                    const int c0 = ana_skip[pi][(size_t)(bofs[m] + jb)];
                    au.push_back({-(double)std::min(256, G.lmax - m - 256 * jb + 1) * (G.npc - c0) * N,
                                  make_int4(gi, m, jb, c0)});
                }
            }
        }
        // Order by (group, m), larger work first within an m: the CTAs take units round-robin,
        // so all units of one m run at the same time on neighbouring CTAs and share that m's
        // operand tiles through L2 (each analysis unit streams every pair chunk of its m, each
        // synthesis unit every l chunk); the round-robin keeps the CTAs' totals balanced.
        auto by_m = [](const std::pair<double, int4> &a, const std::pair<double, int4> &b) {
            if (a.second.x != b.second.x) return a.second.x < b.second.x;
            if (a.second.y != b.second.y) return a.second.y < b.second.y;
            return a.first < b.first;
        };
        std::stable_sort(su.begin(), su.end(), by_m);
        std::stable_sort(au.begin(), au.end(), by_m);
        for (const auto &x : su) bp->live_syn += (int64_t)(-x.first / N + 0.5);
        for (const auto &x : au) {
            const TcGroup &G = bp->hgroups[x.second.x];
            bp->live_ana += G.npc - x.second.w;
        }
        std::vector<int4> suv, auv;
        for (auto &x : su) suv.push_back(x.second);
        for (auto &x : au) auv.push_back(x.second);
        if (cudaMemcpy(bp->syn_units, suv.data(), sizeof(int4) * suv.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(bp->ana_units, auv.data(), sizeof(int4) * auv.size(), cudaMemcpyHostToDevice) != cudaSuccess)
            rc = fail(HB_ERR_CUDA, "hb_batched_plan_create: upload");
    }
    if (rc != HB_OK) {
        cudaFree(base);
        delete bp;
        return rc;
    }
    *out = bp;
    return HB_OK;
}

int hb_batched_plan_destroy(hb_batched_plan *bp) {
    if (!bp) return HB_OK;
    if (bp->graph) cudaGraphExecDestroy(bp->graph);
    for (auto &e : bp->ev)
        if (e) cudaEventDestroy(e);
    cudaFree(bp->base);
    delete bp;
    return HB_OK;
}

size_t hb_batched_plan_bytes(const hb_batched_plan *bp) { return bp ? bp->bytes : 0; }

int hb_batched_alm2map(hb_batched_plan *bp, const float *alm, float *maps, hb_stream_t stream) {
    if (!bp || !alm || !maps) return fail(HB_ERR_INVALID, "hb_batched_alm2map: null argument");
    HB_NVTX("hb_batched_alm2map");
    cudaStream_t st = (cudaStream_t)stream;
    int rc;
    if (bp->profile) HB_CUDA_TRY(cudaEventRecord(bp->ev[0], st));
    for (size_t gi = 0; gi < bp->hgroups.size(); ++gi) {
        const auto &part = bp->parts[bp->group_part[gi]];
        const float2 *a = (const float2 *)alm + part.alm_ofs +
                          (int64_t)bp->group_first_map[gi] * alm_size(part.p->lmax, part.p->mmax);
        if ((rc = HB_DISPATCH_N(bp, launch_prep_alm)(bp, (int)gi, a, alm_size(part.p->lmax, part.p->mmax), st)))
            return rc;
    }
    if (bp->profile) HB_CUDA_TRY(cudaEventRecord(bp->ev[1], st));
    if ((rc = HB_DISPATCH_N(bp, launch_syn)(bp, st))) return rc;
    if (bp->profile) HB_CUDA_TRY(cudaEventRecord(bp->ev[2], st));
    for (const auto &part : bp->parts) {
        const GeomDev &d = part.p->g->d;
        if ((rc = launch_ring_synthesis(d, 32, part.nmaps, part.GF, part.p->mmax, maps + part.map_ofs, d.npix, nullptr,
                                        false, true, 0, st)))
            return rc;
    }
    if (bp->profile) HB_CUDA_TRY(cudaEventRecord(bp->ev[3], st));
    return HB_OK;
}

int hb_batched_map2alm(hb_batched_plan *bp, const float *maps, float *alm, hb_stream_t stream) {
    return hb_batched_map2alm_fl(bp, maps, alm, nullptr, stream);
}

int hb_batched_map2alm_fl(hb_batched_plan *bp, const float *maps, float *alm, const float *fl, hb_stream_t stream) {
    if (!bp || !alm || !maps) return fail(HB_ERR_INVALID, "hb_batched_map2alm: null argument");
    HB_NVTX("hb_batched_map2alm");
    cudaStream_t st = (cudaStream_t)stream;
    int rc;
    if (bp->profile) HB_CUDA_TRY(cudaEventRecord(bp->ev[4], st));
    for (const auto &part : bp->parts) {
        const GeomDev &d = part.p->g->d;
        if ((rc = launch_ring_analysis(d, 32, part.nmaps, maps + part.map_ofs, d.npix, nullptr, part.GF, part.p->mmax, 0,
                                       false, false, st, /*mblk=*/true)))
            return rc;
    }
    if (bp->profile) HB_CUDA_TRY(cudaEventRecord(bp->ev[5], st));
    for (size_t gi = 0; gi < bp->hgroups.size(); ++gi) {
        const auto &part = bp->parts[bp->group_part[gi]];
        const float2 *F = part.GF + (int64_t)bp->group_first_map[gi] * part.ff_stride;
        if ((rc = HB_DISPATCH_N(bp, launch_prep_f)(bp, (int)gi, F, part.ff_stride, st))) return rc;
    }
    if (bp->profile) HB_CUDA_TRY(cudaEventRecord(bp->ev[6], st));
    if ((rc = HB_DISPATCH_N(bp, launch_ana)(bp, (float2 *)alm, fl, st))) return rc;
    if (bp->profile) HB_CUDA_TRY(cudaEventRecord(bp->ev[7], st));
    return HB_OK;
}

int hb_batched_graph_capture(hb_batched_plan *bp, const float *alm, float *maps, float *alm_out) {
    if (!bp || !maps || (!alm && !alm_out)) return fail(HB_ERR_INVALID, "hb_batched_graph_capture: bad arguments");
    cudaStream_t s = nullptr;
    HB_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    const bool prof = bp->profile;
    bp->profile = false;  // no event records inside the graph
    int rc = HB_OK;
    cudaGraph_t graph = nullptr;
    if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        rc = fail(HB_ERR_CUDA, "hb_batched_graph_capture: begin capture failed");
    } else {
        if (alm) rc = hb_batched_alm2map(bp, alm, maps, s);
        if (rc == HB_OK && alm_out) rc = hb_batched_map2alm(bp, maps, alm_out, s);
        const cudaError_t e = cudaStreamEndCapture(s, &graph);
        if (rc == HB_OK && e != cudaSuccess)
            rc = fail(HB_ERR_CUDA, std::string("hb_batched_graph_capture: ") + cudaGetErrorString(e));
    }
    bp->profile = prof;
    cudaGraphExec_t exec = nullptr;
    if (rc == HB_OK && cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess)
        rc = fail(HB_ERR_CUDA, "hb_batched_graph_capture: instantiate failed");
    if (graph) cudaGraphDestroy(graph);
    cudaStreamDestroy(s);
    cudaGetLastError();
    if (rc != HB_OK) return rc;
    if (bp->graph) cudaGraphExecDestroy(bp->graph);
    bp->graph = exec;
    return HB_OK;
}

int hb_batched_graph_launch(hb_batched_plan *bp, hb_stream_t stream) {
    if (!bp || !bp->graph) return fail(HB_ERR_INVALID, "hb_batched_graph_launch: no captured graph");
    HB_CUDA_TRY(cudaGraphLaunch(bp->graph, (cudaStream_t)stream));
    return HB_OK;
}

int hb_batched_profile(hb_batched_plan *bp, int enable) {
    if (!bp) return fail(HB_ERR_INVALID, "hb_batched_profile: null plan");
    if (enable && !bp->ev[0])
        for (auto &e : bp->ev) HB_CUDA_TRY(cudaEventCreate(&e));
    bp->profile = enable != 0;
    return HB_OK;
}

int hb_batched_stage_ms(hb_batched_plan *bp, float *ms) {
    if (!bp || !ms || !bp->ev[0]) return fail(HB_ERR_INVALID, "hb_batched_stage_ms: profiling not enabled");
    HB_CUDA_TRY(cudaEventSynchronize(bp->ev[3]));
    HB_CUDA_TRY(cudaEventSynchronize(bp->ev[7]));
    const int pairs[6][2] = {{0, 1}, {1, 2}, {2, 3}, {4, 5}, {5, 6}, {6, 7}};
    for (int i = 0; i < 6; ++i) HB_CUDA_TRY(cudaEventElapsedTime(&ms[i], bp->ev[pairs[i][0]], bp->ev[pairs[i][1]]));
    return HB_OK;
}

int hb_batched_work(const hb_batched_plan *bp, int64_t *chunks, int *mma_n) {
    if (!bp || !chunks || !mma_n) return fail(HB_ERR_INVALID, "hb_batched_work: null argument");
    chunks[0] = bp->live_syn;
    chunks[1] = bp->live_ana;
    *mma_n = bp->N;
    return HB_OK;
}

int hb_batched_fault_test(hb_batched_plan *bp, uint64_t wait_ns, int withhold_copy) {
    if (!bp || wait_ns < 1000000ull || wait_ns > 10000000000ull || withhold_copy < 0 || withhold_copy > 1)
        return fail(HB_ERR_INVALID, "hb_batched_fault_test: wait_ns in [1 ms, 10 s], withhold_copy 0 or 1");
    bp->wait_ns = wait_ns;
    bp->inject = withhold_copy;
    return HB_OK;
}

int hb_batched_reset_status(hb_batched_plan *bp) {
    if (!bp) return fail(HB_ERR_INVALID, "hb_batched_reset_status: null plan");
    HB_CUDA_TRY(cudaMemset(bp->err, 0, sizeof(int)));
    return HB_OK;
}

int hb_batched_status(hb_batched_plan *bp, int *code) {
    if (!bp || !code) return fail(HB_ERR_INVALID, "hb_batched_status: null argument");
    HB_CUDA_TRY(cudaMemcpy(code, bp->err, sizeof(int), cudaMemcpyDeviceToHost));
    return HB_OK;
}

}  // extern "C"
