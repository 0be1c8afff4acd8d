// C-ABI entry points of the transforms, stages and alm2cl (declared in include/hbsht.h).
//
// Host orchestration only: validate, carve the caller's workspace, launch the ring-FFT and
// Legendre kernels on the caller's stream.  No allocation, no synchronisation.
#include <cstdio>
#include <string>

#include "hb_internal.cuh"

namespace hb {

static int check_plan(const hb_plan *p, int nmaps, int prec, bool spin, const char *who) {
    if (!p || !p->g) return fail(HB_ERR_INVALID, std::string(who) + ": null plan");
    if (nmaps <= 0 || nmaps > 65535) return fail(HB_ERR_INVALID, std::string(who) + ": nmaps must lie in [1, 65535]");
    if (prec == 32 && !spin && !p->ck)
        return fail(HB_ERR_INVALID, std::string(who) + ": FP32 transforms need a plan created with HB_PLAN_FP32");
    if (prec == 32 && spin && !p->ckP)
        return fail(HB_ERR_INVALID,
                    std::string(who) + ": FP32 spin-2 transforms need a plan created with HB_PLAN_SPIN2_FP32");
    return HB_OK;
}

static size_t fm_bytes(const hb_plan *p, int precision, int nmaps) {
    return (size_t)nmaps * (size_t)(p->mmax + 1) * (size_t)p->g->d.npairs * 2 * (precision == 32 ? 8 : 16);
}

static int check_ws(void *ws, size_t have, size_t need, const char *who) {
    if (!ws || have < need)
        return fail(HB_ERR_WORKSPACE, std::string(who) + ": workspace needs " + std::to_string(need) + " bytes");
    return HB_OK;
}

#define HB_PLAN_ARGS(p) (p)->g->d, prec, nmaps, (p)->lmax, (p)->mmax
static const float4 *ck_of(const hb_plan *p, int prec) { return prec == 32 ? p->ck : nullptr; }

static int map2alm_impl(const hb_plan *p, int nmaps, const void *maps, const double *w, void *alm, void *ws,
                        size_t wsb, int flags, cudaStream_t st, int prec, const char *who) {
    int rc = check_plan(p, nmaps, prec, false, who);
    if (rc) return rc;
    if (!maps || !alm) return fail(HB_ERR_INVALID, std::string(who) + ": null data pointer");
    if ((rc = check_ws(ws, wsb, fm_bytes(p, prec, nmaps), who))) return rc;
    const GeomDev &d = p->g->d;
    if ((rc = launch_ring_analysis(d, prec, nmaps, maps, d.npix, w, ws, p->mmax, flags, false, false, st))) return rc;
    return launch_leg_analysis(HB_PLAN_ARGS(p), ws, alm, st, ck_of(p, prec), p->blk_ofs);
}

static int alm2map_impl(const hb_plan *p, int nmaps, const void *alm, void *maps, void *ws, size_t wsb, int flags,
                        cudaStream_t st, int prec, const char *who) {
    int rc = check_plan(p, nmaps, prec, false, who);
    if (rc) return rc;
    if (!maps || !alm) return fail(HB_ERR_INVALID, std::string(who) + ": null data pointer");
    if ((rc = check_ws(ws, wsb, fm_bytes(p, prec, nmaps), who))) return rc;
    const GeomDev &d = p->g->d;
    if ((rc = launch_leg_synthesis(HB_PLAN_ARGS(p), alm, ws, st, ck_of(p, prec), p->blk_ofs))) return rc;
    return launch_ring_synthesis(d, prec, nmaps, ws, p->mmax, maps, d.npix, nullptr, false, true, flags, st);
}

// transpose of alm2map: ring analysis with unit pixel weights and c_m = 2 for m > 0
static int alm2map_adj_impl(const hb_plan *p, int nmaps, const void *maps, void *alm, void *ws, size_t wsb,
                            int flags, cudaStream_t st, int prec, const char *who) {
    int rc = check_plan(p, nmaps, prec, false, who);
    if (rc) return rc;
    if (!maps || !alm) return fail(HB_ERR_INVALID, std::string(who) + ": null data pointer");
    if ((rc = check_ws(ws, wsb, fm_bytes(p, prec, nmaps), who))) return rc;
    const GeomDev &d = p->g->d;
    if ((rc = launch_ring_analysis(d, prec, nmaps, maps, d.npix, nullptr, ws, p->mmax, flags & ~HB_F_NOFOLD, true,
                                   true, st)))
        return rc;
    return launch_leg_analysis(HB_PLAN_ARGS(p), ws, alm, st, ck_of(p, prec), p->blk_ofs);
}

// transpose of map2alm: Legendre synthesis, then ring synthesis with c_m = 1 and pixel weights
static int map2alm_adj_impl(const hb_plan *p, int nmaps, const void *alm, const double *w, void *maps, void *ws,
                            size_t wsb, int flags, cudaStream_t st, int prec, const char *who) {
    int rc = check_plan(p, nmaps, prec, false, who);
    if (rc) return rc;
    if (!maps || !alm) return fail(HB_ERR_INVALID, std::string(who) + ": null data pointer");
    if (flags & HB_F_NOFOLD) return fail(HB_ERR_UNSUPPORTED, std::string(who) + ": HB_F_NOFOLD has no adjoint here");
    if ((rc = check_ws(ws, wsb, fm_bytes(p, prec, nmaps), who))) return rc;
    const GeomDev &d = p->g->d;
    if ((rc = launch_leg_synthesis(HB_PLAN_ARGS(p), alm, ws, st, ck_of(p, prec), p->blk_ofs))) return rc;
    return launch_ring_synthesis(d, prec, nmaps, ws, p->mmax, maps, d.npix, w, true, false, flags, st);
}

// spin-2 analysis; with adjoint_of_synth the ring analysis uses unit weights and c_m = 2
// (the transpose of the spin-2 synthesis)
static int map2alm_spin_impl(const hb_plan *p, int nmaps, const void *Q, const void *U, const double *w, void *E,
                             void *B, void *ws, size_t wsb, int flags, cudaStream_t st, int prec, bool adjoint_of_synth,
                             const char *who) {
    int rc = check_plan(p, nmaps, prec, true, who);
    if (rc) return rc;
    if (!Q || !U || !E || !B) return fail(HB_ERR_INVALID, std::string(who) + ": null data pointer");
    const size_t half = fm_bytes(p, prec, nmaps);
    if ((rc = check_ws(ws, wsb, 2 * half, who))) return rc;
    const GeomDev &d = p->g->d;
    char *QF = (char *)ws, *UF = (char *)ws + half;
    const int f = adjoint_of_synth ? (flags & ~HB_F_NOFOLD) : flags;
    const double *wr = adjoint_of_synth ? nullptr : w;
    if ((rc = launch_ring_analysis(d, prec, nmaps, Q, d.npix, wr, QF, p->mmax, f, adjoint_of_synth, adjoint_of_synth,
                                   st)))
        return rc;
    if ((rc = launch_ring_analysis(d, prec, nmaps, U, d.npix, wr, UF, p->mmax, f, adjoint_of_synth, adjoint_of_synth,
                                   st)))
        return rc;
    return launch_spin_analysis(HB_PLAN_ARGS(p), QF, UF, E, B, st, prec == 32 ? p->ckP : nullptr,
                                prec == 32 ? p->ckM : nullptr, p->blk_ofs_spin);
}

// spin-2 synthesis; with adjoint_of_anal the ring synthesis applies the pixel weights and c_m = 1
// (the transpose of the weighted spin-2 analysis)
static int alm2map_spin_impl(const hb_plan *p, int nmaps, const void *E, const void *B, const double *w, void *Q,
                             void *U, void *ws, size_t wsb, int flags, cudaStream_t st, int prec, bool adjoint_of_anal,
                             const char *who) {
    int rc = check_plan(p, nmaps, prec, true, who);
    if (rc) return rc;
    if (!Q || !U || !E || !B) return fail(HB_ERR_INVALID, std::string(who) + ": null data pointer");
    if (adjoint_of_anal && (flags & HB_F_NOFOLD))
        return fail(HB_ERR_UNSUPPORTED, std::string(who) + ": HB_F_NOFOLD has no adjoint here");
    const size_t half = fm_bytes(p, prec, nmaps);
    if ((rc = check_ws(ws, wsb, 2 * half, who))) return rc;
    const GeomDev &d = p->g->d;
    char *QG = (char *)ws, *UG = (char *)ws + half;
    if ((rc = launch_spin_synthesis(HB_PLAN_ARGS(p), E, B, QG, UG, st, prec == 32 ? p->ckP : nullptr,
                                    prec == 32 ? p->ckM : nullptr, p->blk_ofs_spin)))
        return rc;
    if ((rc = launch_ring_synthesis(d, prec, nmaps, QG, p->mmax, Q, d.npix, w, adjoint_of_anal, !adjoint_of_anal, flags,
                                    st)))
        return rc;
    return launch_ring_synthesis(d, prec, nmaps, UG, p->mmax, U, d.npix, w, adjoint_of_anal, !adjoint_of_anal, flags,
                                 st);
}

// alm2cl (alm_ops.py:19-32): a CTA owns 32 consecutive l of one map (the lanes) and its 8 warps
// split the m range (m = warp mod 8), so every warp load reads 32 consecutive l of one healpy
// m-column (256 B); FP64 accumulation, one shared-memory reduction over the warps, no atomics.
template <typename V>
__global__ void __launch_bounds__(256) alm2cl_kernel(int lmax, int mmax, const V *__restrict__ a1,
                                                     const V *__restrict__ a2, int64_t stride, double *__restrict__ cl) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int l = blockIdx.x * 32 + lane, b = blockIdx.y;
    const V *p1 = a1 + b * stride, *p2 = (a2 ? a2 : a1) + b * stride;
    const int mtop = l < mmax ? l : mmax;
    auto term = [&](int m) -> double {
        const int64_t k = alm_idx(lmax, l, m);
        const V u = p1[k], v = p2[k];
        return (m == 0 ? 1.0 : 2.0) * ((double)u.x * (double)v.x + (double)u.y * (double)v.y);
    };
    double acc = 0.0;
    if (l <= lmax) {
        int m = warp;
        for (; m + 24 <= mtop; m += 32) {  // four independent loads in flight per thread
            const double t0 = term(m), t1 = term(m + 8), t2 = term(m + 16), t3 = term(m + 24);
            acc += (t0 + t1) + (t2 + t3);
        }
        for (; m <= mtop; m += 8) acc += term(m);
    }
    __shared__ double red[8][33];
    red[warp][lane] = acc;
    __syncthreads();
    if (warp == 0 && l <= lmax) {
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < 8; ++w) s += red[w][lane];
        cl[(int64_t)b * (lmax + 1) + l] = s / (2.0 * l + 1.0);
    }
}

template <typename V>
static int alm2cl_impl(int lmax, int mmax, int nmaps, const V *a1, const V *a2, double *cl, cudaStream_t st) {
    if (lmax < 0 || mmax < 0 || mmax > lmax || nmaps <= 0 || nmaps > 65535 || !a1 || !cl)
        return fail(HB_ERR_INVALID, "hb_alm2cl: bad arguments");
    dim3 grid((unsigned)((lmax + 32) / 32), (unsigned)nmaps);
    alm2cl_kernel<V><<<grid, 256, 0, st>>>(lmax, mmax, a1, a2, alm_size(lmax, mmax), cl);
    HB_CHECK_LAUNCH();
    return HB_OK;
}

// FP32 FMA throughput probe: each thread runs `iters` rounds of 8 independent FMA chains
// (2 flop each); out receives one value per thread so nothing is optimised away.
__global__ void fp32_probe_kernel(int iters, float *out) {
    float a[8];
    const float s = 1.0f + 1e-7f * threadIdx.x, c = 1e-8f;
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = (float)(k + 1) * 1e-3f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) a[k] = fmaf(a[k], s, c);
    }
    float r = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) r += a[k];
    out[blockIdx.x * blockDim.x + threadIdx.x] = r;
}

}  // namespace hb

using namespace hb;

extern "C" {

size_t hb_sht_workspace_size(const hb_plan *p, int precision, int nmaps) {
    if (!p || nmaps <= 0 || (precision != 32 && precision != 64)) return 0;
    return fm_bytes(p, precision, nmaps);
}

size_t hb_spin2_workspace_size(const hb_plan *p, int precision, int nmaps) {
    return 2 * hb_sht_workspace_size(p, precision, nmaps);
}

#define ST(s) ((cudaStream_t)(s))
int hb_map2alm_f32(const hb_plan *p, int nmaps, const float *maps, const double *w, float *alm, void *ws, size_t wsb,
                   int flags, hb_stream_t s) {
    return map2alm_impl(p, nmaps, maps, w, alm, ws, wsb, flags, ST(s), 32, "hb_map2alm_f32");
}
int hb_map2alm_f64(const hb_plan *p, int nmaps, const double *maps, const double *w, double *alm, void *ws,
                   size_t wsb, int flags, hb_stream_t s) {
    return map2alm_impl(p, nmaps, maps, w, alm, ws, wsb, flags, ST(s), 64, "hb_map2alm_f64");
}
int hb_alm2map_f32(const hb_plan *p, int nmaps, const float *alm, float *maps, void *ws, size_t wsb, int flags,
                   hb_stream_t s) {
    return alm2map_impl(p, nmaps, alm, maps, ws, wsb, flags, ST(s), 32, "hb_alm2map_f32");
}
int hb_alm2map_f64(const hb_plan *p, int nmaps, const double *alm, double *maps, void *ws, size_t wsb, int flags,
                   hb_stream_t s) {
    return alm2map_impl(p, nmaps, alm, maps, ws, wsb, flags, ST(s), 64, "hb_alm2map_f64");
}
int hb_alm2map_adjoint_f32(const hb_plan *p, int nmaps, const float *maps, float *alm, void *ws, size_t wsb,
                           int flags, hb_stream_t s) {
    return alm2map_adj_impl(p, nmaps, maps, alm, ws, wsb, flags, ST(s), 32, "hb_alm2map_adjoint_f32");
}
int hb_alm2map_adjoint_f64(const hb_plan *p, int nmaps, const double *maps, double *alm, void *ws, size_t wsb,
                           int flags, hb_stream_t s) {
    return alm2map_adj_impl(p, nmaps, maps, alm, ws, wsb, flags, ST(s), 64, "hb_alm2map_adjoint_f64");
}
int hb_map2alm_adjoint_f32(const hb_plan *p, int nmaps, const float *alm, const double *w, float *maps, void *ws,
                           size_t wsb, int flags, hb_stream_t s) {
    return map2alm_adj_impl(p, nmaps, alm, w, maps, ws, wsb, flags, ST(s), 32, "hb_map2alm_adjoint_f32");
}
int hb_map2alm_adjoint_f64(const hb_plan *p, int nmaps, const double *alm, const double *w, double *maps, void *ws,
                           size_t wsb, int flags, hb_stream_t s) {
    return map2alm_adj_impl(p, nmaps, alm, w, maps, ws, wsb, flags, ST(s), 64, "hb_map2alm_adjoint_f64");
}
int hb_map2alm_spin2_f32(const hb_plan *p, int nmaps, const float *Q, const float *U, const double *w, float *E,
                         float *B, void *ws, size_t wsb, int flags, hb_stream_t s) {
    return map2alm_spin_impl(p, nmaps, Q, U, w, E, B, ws, wsb, flags, ST(s), 32, false, "hb_map2alm_spin2_f32");
}
int hb_map2alm_spin2_f64(const hb_plan *p, int nmaps, const double *Q, const double *U, const double *w, double *E,
                         double *B, void *ws, size_t wsb, int flags, hb_stream_t s) {
    return map2alm_spin_impl(p, nmaps, Q, U, w, E, B, ws, wsb, flags, ST(s), 64, false, "hb_map2alm_spin2_f64");
}
int hb_alm2map_spin2_f32(const hb_plan *p, int nmaps, const float *E, const float *B, float *Q, float *U, void *ws,
                         size_t wsb, int flags, hb_stream_t s) {
    return alm2map_spin_impl(p, nmaps, E, B, nullptr, Q, U, ws, wsb, flags, ST(s), 32, false, "hb_alm2map_spin2_f32");
}
int hb_alm2map_spin2_f64(const hb_plan *p, int nmaps, const double *E, const double *B, double *Q, double *U,
                         void *ws, size_t wsb, int flags, hb_stream_t s) {
    return alm2map_spin_impl(p, nmaps, E, B, nullptr, Q, U, ws, wsb, flags, ST(s), 64, false, "hb_alm2map_spin2_f64");
}
int hb_alm2map_spin2_adjoint_f32(const hb_plan *p, int nmaps, const float *gQ, const float *gU, float *gE, float *gB,
                                 void *ws, size_t wsb, int flags, hb_stream_t s) {
    return map2alm_spin_impl(p, nmaps, gQ, gU, nullptr, gE, gB, ws, wsb, flags, ST(s), 32, true,
                             "hb_alm2map_spin2_adjoint_f32");
}
int hb_alm2map_spin2_adjoint_f64(const hb_plan *p, int nmaps, const double *gQ, const double *gU, double *gE,
                                 double *gB, void *ws, size_t wsb, int flags, hb_stream_t s) {
    return map2alm_spin_impl(p, nmaps, gQ, gU, nullptr, gE, gB, ws, wsb, flags, ST(s), 64, true,
                             "hb_alm2map_spin2_adjoint_f64");
}
int hb_map2alm_spin2_adjoint_f32(const hb_plan *p, int nmaps, const float *gE, const float *gB, const double *w,
                                 float *gQ, float *gU, void *ws, size_t wsb, int flags, hb_stream_t s) {
    return alm2map_spin_impl(p, nmaps, gE, gB, w, gQ, gU, ws, wsb, flags, ST(s), 32, true,
                             "hb_map2alm_spin2_adjoint_f32");
}
int hb_map2alm_spin2_adjoint_f64(const hb_plan *p, int nmaps, const double *gE, const double *gB, const double *w,
                                 double *gQ, double *gU, void *ws, size_t wsb, int flags, hb_stream_t s) {
    return alm2map_spin_impl(p, nmaps, gE, gB, w, gQ, gU, ws, wsb, flags, ST(s), 64, true,
                             "hb_map2alm_spin2_adjoint_f64");
}

// ---- pipeline stages
int hb_ring_analysis(const hb_plan *p, int prec, int nmaps, const void *maps, const double *w, void *F, int flags,
                     hb_stream_t s) {
    if ((prec != 32 && prec != 64) || !maps || !F) return fail(HB_ERR_INVALID, "hb_ring_analysis: bad args");
    int rc = check_plan(p, nmaps, 64, false, "hb_ring_analysis");
    if (rc) return rc;
    return launch_ring_analysis(p->g->d, prec, nmaps, maps, p->g->d.npix, w, F, p->mmax, flags, false, false, ST(s));
}
int hb_ring_synthesis(const hb_plan *p, int prec, int nmaps, const void *G, void *maps, int flags, hb_stream_t s) {
    if ((prec != 32 && prec != 64) || !maps || !G) return fail(HB_ERR_INVALID, "hb_ring_synthesis: bad args");
    int rc = check_plan(p, nmaps, 64, false, "hb_ring_synthesis");
    if (rc) return rc;
    return launch_ring_synthesis(p->g->d, prec, nmaps, G, p->mmax, maps, p->g->d.npix, nullptr, false, true, flags,
                                 ST(s));
}
int hb_legendre_analysis_ms(const hb_plan *p, int prec, int nmaps, int nm, const int32_t *mlist, const void *F,
                            void *alm, hb_stream_t s) {
    if ((prec != 32 && prec != 64) || !F || !alm || !mlist || nm < 1 || nm > 65535)
        return fail(HB_ERR_INVALID, "hb_legendre_analysis_ms: bad args");
    int rc = check_plan(p, nmaps, prec, false, "hb_legendre_analysis_ms");
    if (rc) return rc;
    return launch_leg_analysis(HB_PLAN_ARGS(p), F, alm, ST(s), ck_of(p, prec), p->blk_ofs, nm, mlist);
}
int hb_legendre_synthesis_ms(const hb_plan *p, int prec, int nmaps, int nm, const int32_t *mlist, const void *alm,
                             void *G, hb_stream_t s) {
    if ((prec != 32 && prec != 64) || !G || !alm || !mlist || nm < 1 || nm > 65535)
        return fail(HB_ERR_INVALID, "hb_legendre_synthesis_ms: bad args");
    int rc = check_plan(p, nmaps, prec, false, "hb_legendre_synthesis_ms");
    if (rc) return rc;
    return launch_leg_synthesis(HB_PLAN_ARGS(p), alm, G, ST(s), ck_of(p, prec), p->blk_ofs, nm, mlist);
}
int hb_legendre_analysis(const hb_plan *p, int prec, int nmaps, const void *F, void *alm, hb_stream_t s) {
    if ((prec != 32 && prec != 64) || !F || !alm) return fail(HB_ERR_INVALID, "hb_legendre_analysis: bad args");
    int rc = check_plan(p, nmaps, prec, false, "hb_legendre_analysis");
    if (rc) return rc;
    return launch_leg_analysis(HB_PLAN_ARGS(p), F, alm, ST(s), ck_of(p, prec), p->blk_ofs);
}
int hb_legendre_synthesis(const hb_plan *p, int prec, int nmaps, const void *alm, void *G, hb_stream_t s) {
    if ((prec != 32 && prec != 64) || !G || !alm) return fail(HB_ERR_INVALID, "hb_legendre_synthesis: bad args");
    int rc = check_plan(p, nmaps, prec, false, "hb_legendre_synthesis");
    if (rc) return rc;
    return launch_leg_synthesis(HB_PLAN_ARGS(p), alm, G, ST(s), ck_of(p, prec), p->blk_ofs);
}

int hb_probe_fp32(int blocks, int threads, int iters, float *out, hb_stream_t s) {
    if (blocks <= 0 || threads <= 0 || threads > 1024 || iters <= 0 || !out)
        return fail(HB_ERR_INVALID, "hb_probe_fp32: bad args");
    fp32_probe_kernel<<<blocks, threads, 0, ST(s)>>>(iters, out);
    HB_CHECK_LAUNCH();
    return HB_OK;
}

int hb_alm2cl_f32(int lmax, int mmax, int nmaps, const float *alm1, const float *alm2, double *cl, hb_stream_t s) {
    return alm2cl_impl<float2>(lmax, mmax, nmaps, (const float2 *)alm1, (const float2 *)alm2, cl, ST(s));
}
int hb_alm2cl_f64(int lmax, int mmax, int nmaps, const double *alm1, const double *alm2, double *cl, hb_stream_t s) {
    return alm2cl_impl<double2>(lmax, mmax, nmaps, (const double2 *)alm1, (const double2 *)alm2, cl, ST(s));
}

}  // extern "C"
