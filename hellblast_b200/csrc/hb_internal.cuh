// Internal definitions shared by the hbsht CUDA sources (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <stdint.h>
#include <string>

#include "../../include/hbsht.h"

#define HB_MAX_L 16383
// nphi range (log2) of the pair-packed FP32 ring FFT kernels
#define PK_MIN_LOG 9
#define PK_MAX_LOG 14

namespace hb {

// ----------------------------------------------------------------------------- errors
void set_error(const std::string &msg);
int fail(int code, const std::string &msg);
#define HB_CUDA_TRY(call)                                                                         \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess)                                                                    \
            return ::hb::fail(HB_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));   \
    } while (0)
#define HB_CHECK_LAUNCH()                                                                         \
    do {                                                                                          \
        cudaError_t e_ = cudaGetLastError();                                                      \
        if (e_ != cudaSuccess)                                                                    \
            return ::hb::fail(HB_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e_)); \
    } while (0)

// NVTX range over a host-side launch sequence (header-only NVTX; inert unless a profiler is
// attached), so timelines show which entry point and stage queued each kernel
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};
#define HB_NVTX(name) ::hb::NvtxRange hb_nvtx_range_(name)

// ----------------------------------------------------------------------------- complex helpers
template <typename T> struct C2;
template <> struct C2<float> { using type = float2; };
template <> struct C2<double> { using type = double2; };
template <typename T> using c2_t = typename C2<T>::type;

__host__ __device__ __forceinline__ float2 mk2(float a, float b) { return make_float2(a, b); }
__host__ __device__ __forceinline__ double2 mk2(double a, double b) { return make_double2(a, b); }
template <typename V> __host__ __device__ __forceinline__ V cadd(V a, V b) { return mk2(a.x + b.x, a.y + b.y); }
template <typename V> __host__ __device__ __forceinline__ V csub(V a, V b) { return mk2(a.x - b.x, a.y - b.y); }
template <typename V> __host__ __device__ __forceinline__ V cmul(V a, V b) {
    return mk2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename V> __host__ __device__ __forceinline__ V cconj(V a) { return mk2(a.x, -a.y); }
template <typename V, typename S> __host__ __device__ __forceinline__ V cscale(V a, S s) {
    return mk2(a.x * s, a.y * s);
}

__device__ __forceinline__ void sincospi_t(float x, float *s, float *c) { sincospif(x, s, c); }
__device__ __forceinline__ void sincospi_t(double x, double *s, double *c) { sincospi(x, s, c); }

// ----------------------------------------------------------------------------- layout
__host__ __device__ __forceinline__ int64_t alm_idx(int64_t lmax, int64_t l, int64_t m) {
    return m * (2 * lmax + 1 - m) / 2 + l;
}
inline int64_t alm_size(int lmax, int mmax) { return alm_idx(lmax, lmax, mmax) + 1; }

// ----------------------------------------------------------------------------- geometry
// Device-resident ring/pair tables.  A "pair" is a north ring and its mirror south ring
// (theta_S = pi - theta_N) that share |cos theta|; unpaired rings (the equator, or rings of a
// non-symmetric geometry) have south = -1.
struct GeomDev {
    int64_t nr, npix, npairs;
    int32_t *nphi;         // [nr]
    int64_t *ofs;          // [nr] first pixel of ring
    double *phi0_pi;       // [nr] phi0 / pi
    double *w;             // [nr] default per-ring weight (dz convention)
    int32_t *ring_pair;    // [nr]
    int32_t *ring_side;    // [nr] 0 = north/unpaired, 1 = south
    int32_t *pair_ring;    // [npairs][2] ring index of north, south (-1)
    double *pair_x;        // [npairs] cos theta of the north ring
    float *pair_xhi;       // [npairs] float(x)
    float *pair_xlo;       // [npairs] float(x - xhi)
    double *pair_log2sin;  // [npairs] log2 sin theta
    double *pair_log2ch;   // [npairs] log2 cos(theta/2)
    double *pair_log2sh;   // [npairs] log2 sin(theta/2)
    // ragged FFT: per ring the convolution length L (== nphi/2 when that is a power of two:
    // direct FFT; otherwise Bluestein) and the offset of its chirp spectrum in blu_*.
    int32_t *fft_len;      // [nr]
    int64_t *blu_ofs;      // [nr] (-1 for direct)
    // per distinct N: L entries of the chirp spectrum (forward-transform output order, scaled by
    // 1/L), then N entries of the chirp exp(-i pi j^2 / N), j < N
    double2 *blu_f64;
    float2 *blu_f32;
    int32_t *blu_owner;    // [n_blu] first ring using each distinct chirp table
    int64_t n_blu;
    int max_fft_len;       // max L over rings
    // FFT twiddles exp(-2 pi i j / 2^log_tw), j < 2^(log_tw-1), 2^log_tw = max(2, max_fft_len)
    double2 *tw64;
    float2 *tw32;
    int log_tw;
    // pairs grouped by convolution length class (max L of the pair's rings), ascending:
    // class c = pairs cls_pairs[cls_first[c] .. cls_first[c+1]) with length cls_L[c]
    int32_t *cls_pairs;    // [npairs]
    int n_cls;
    int cls_L[32];
    int64_t cls_first[33];
    int max_nphi;
    // FP32 ring FFTs: pairs taken by the pair-packed kernels (hb_ringpack.cu), grouped by
    // class key log2 L | (Bluestein << 8) | (quad split << 9) (quad split: L is the quarter-length
    // sub-transform's), and the remaining pairs in convolution-length classes as above
    int32_t *pk_pairs;     // [npairs]
    int pk_n_cls;
    int pk_logn[16];
    int64_t pk_first[17];
    // pair-packed Bluestein tables per distinct n: chirp spectrum (L), chirp (L/2), then the
    // phase block of the CTA table (pk_bt_entries; quad split: the chirp of length n/4)
    float2 *pkb_bt;
    int64_t *pkb_bt_ofs;   // [npairs] offset of the pair's table in pkb_bt (-1: not Bluestein)
    // per transform length 2^k, k in [PK_MIN_LOG, PK_MAX_LOG]: the pair-packed kernels' shared
    // table block (twiddles, then the phases for n = 2^k), copied by every CTA (pk_tab_entries)
    float2 *pk_tw;
    int64_t pk_tw_ofs[PK_MAX_LOG + 1];
    int32_t *rest_pairs;   // [npairs]
    int rest_n_cls;
    int rest_L[32];
    int64_t rest_first[33];
    double *log2cm;        // [HB_MAX_L+1] log2 sqrt((2m+1)!!/((2m)!! 4 pi)), scalar lambda_mm
    double *log2spin;      // [HB_MAX_L+1] log2 of the constant of N_l0 d^l0_{m,+-2}
};

}  // namespace hb

struct hb_geom {
    hb::GeomDev d;
    int64_t nside;  // 0 when not a HEALPix grid
    void *alloc_base;
};

// A geometry plus (lmax, mmax) and the FP32 recursion checkpoints (see hb_plan.cu).
struct hb_plan {
    const hb_geom *g;
    int lmax, mmax, flags;
    void *alloc_base;
    size_t bytes;
    int64_t *blk_ofs;       // [mmax+2] first checkpoint block of each m (scalar)
    int64_t *blk_ofs_spin;  // [mmax+2] same for the spin-2 recursions (blocks from max(m,2))
    float4 *ck;             // scalar checkpoints, or null
    float4 *ckP, *ckM;      // spin-2 checkpoints, or null
};

namespace hb {
// kernels' host launchers (implemented in the .cu files)
// the plan's scalar recursion states at l0 + 128 of every 256-l block (same indexing as ck), and
// optionally at l0 + 64 and l0 + 192; default stream, asynchronous
int launch_ck_mid(const hb_plan *p, float4 *ck_mid, float4 *ck_q1 = nullptr, float4 *ck_q3 = nullptr);
// F(m, ring pair) workspaces: m-major [m][pair][north, south], or with mblk (the batched FP32
// analysis) blocked by 8 orders, [m/8][pair][m%8][north, south], so that one ring pair's
// consecutive orders share 128-byte lines; rows = orders padded to a multiple of 8
__host__ __device__ __forceinline__ int64_t fg_rows(int mmax, bool mblk) {
    return mblk ? (int64_t)((mmax + 8) / 8) * 8 : (int64_t)mmax + 1;
}
// offset of (m, pair p) in (north, south) complex pairs
__device__ __forceinline__ int64_t fg_off(int m, int64_t p, int64_t np, bool mblk) {
    return mblk ? (((int64_t)(m >> 3) * np + p) << 3) + (m & 7) : (int64_t)m * np + p;
}
int launch_ring_analysis(const GeomDev &g, int precision, int nmaps, const void *maps, int64_t map_stride,
                         const double *w, void *Fm, int mmax, int flags, bool unit_weights, bool mdouble,
                         cudaStream_t st, bool mblk = false);
int launch_ring_synthesis(const GeomDev &g, int precision, int nmaps, const void *Gm, int mmax, void *maps,
                          int64_t map_stride, const double *w, bool apply_weights, bool mdouble, int flags,
                          cudaStream_t st);
// ck / blk_ofs: FP32 recursion checkpoints of a plan (null: no re-anchoring; FP64 ignores them).
// mlist (device, nm entries; null: all orders 0..mmax): the orders to transform, F / G holding
// one row per listed order in list order; alm rows of the other orders are left untouched
// (analysis over several pair chunks clears the whole alm first).
int launch_leg_analysis(const GeomDev &g, int precision, int nmaps, int lmax, int mmax, const void *Fm,
                        void *alm, cudaStream_t st, const float4 *ck, const int64_t *blk_ofs, int nm = 0,
                        const int32_t *mlist = nullptr);
int launch_leg_synthesis(const GeomDev &g, int precision, int nmaps, int lmax, int mmax, const void *alm,
                         void *Gm, cudaStream_t st, const float4 *ck, const int64_t *blk_ofs, int nm = 0,
                         const int32_t *mlist = nullptr);
int launch_spin_analysis(const GeomDev &g, int precision, int nmaps, int lmax, int mmax, const void *QFm,
                         const void *UFm, void *E, void *B, cudaStream_t st, const float4 *ckP, const float4 *ckM,
                         const int64_t *blk_ofs);
int launch_spin_synthesis(const GeomDev &g, int precision, int nmaps, int lmax, int mmax, const void *E,
                          const void *B, void *QGm, void *UGm, cudaStream_t st, const float4 *ckP,
                          const float4 *ckM, const int64_t *blk_ofs);
// FFT twiddle table and Bluestein chirp spectra of a geometry
int build_fft_tables(GeomDev &g, cudaStream_t st);
// pair-packed FP32 ring FFTs (hb_ringpack.cu) over the geometry's pk_* pairs
bool pk_pair_ok(int nphiN, int nphiS, double phi0N_pi, double phi0S_pi, int *logL, bool *blu);
// log2 of the quarter-length sub-transform when a Bluestein pair of ring length n and whole-ring
// Bluestein length 2^logL runs split in four (hb_ringpack.cu), else 0
int pk_quad_log(int n, int logL);
// chirp spectra of the pair-packed Bluestein pairs: count tables, table e of length 2^logL[e]
// for chirp length ns[e] (the ring length, or a quarter of it for a quad-split ring) at
// out + ofs[e] (device arrays); FP64 computed, FP32 stored
int build_pk_chirp_tables(const GeomDev &g, int count, const int32_t *ns, const int32_t *logL, const int64_t *ofs,
                          int max_logL, float2 *out, cudaStream_t st);
// the pair-packed kernels' table blocks: entries of the block for transform length 2^logL
// (twiddles and phases) and of its phase part (one per Bluestein ring length)
int64_t pk_tab_entries(int logL);
int64_t pk_phase_entries(int logL);
// entries of one Bluestein pair's table (chirp spectrum, chirp, phase block) for chirp length
// 2^logL, quad-split or not
int64_t pk_bt_entries(int logL, bool quad);
// fills g.pk_tw (every length class) and the phase part of each Bluestein table (count tables as
// for build_pk_chirp_tables, ring lengths rn[e], phase block at ofs[e] + 3 L / 2)
int build_pk_tables(const GeomDev &g, int count, const int32_t *ns, const int32_t *rn, const int32_t *logL,
                    const int64_t *ofs, cudaStream_t st);
int launch_pk_synthesis(const GeomDev &g, int nmaps, const float2 *Gm, int mmax, float *maps, int64_t map_stride,
                        const double *w, bool apply_w, bool mdouble, int flags, cudaStream_t st);
int launch_pk_analysis(const GeomDev &g, int nmaps, const float *maps, int64_t map_stride, const double *w,
                       float2 *Fm, int mmax, int flags, bool unit_w, bool mdouble, cudaStream_t st, bool mblk);
}  // namespace hb
