// C-ABI entry points of the scalar transforms and alm2cl (declared in include/hbsht.h).
//
// Host orchestration only: validate, carve the caller's workspace, launch the ring-FFT and
// Legendre kernels on the caller's stream.  No allocation, no synchronisation.
#include <cstdio>
#include <string>

#include "hb_internal.cuh"

namespace hb {

static int check_common(const hb_geom *g, int lmax, int mmax, int nmaps, const char *who) {
    if (!g) return fail(HB_ERR_INVALID, std::string(who) + ": null geometry");
    if (lmax < 0 || lmax > HB_MAX_L) return fail(HB_ERR_INVALID, std::string(who) + ": lmax out of [0, 16383]");
    if (mmax < 0 || mmax > lmax) return fail(HB_ERR_INVALID, std::string(who) + ": mmax must lie in [0, lmax]");
    if (nmaps <= 0 || nmaps > 65535) return fail(HB_ERR_INVALID, std::string(who) + ": nmaps must lie in [1, 65535]");
    return HB_OK;
}

static size_t fm_bytes(const hb_geom *g, int mmax, int precision, int nmaps) {
    return (size_t)nmaps * (size_t)(mmax + 1) * (size_t)g->d.npairs * 2 * (precision == 32 ? 8 : 16);
}

static int check_ws(void *ws, size_t have, size_t need, const char *who) {
    if (!ws || have < need)
        return fail(HB_ERR_WORKSPACE, std::string(who) + ": workspace needs " + std::to_string(need) + " bytes");
    return HB_OK;
}

static int map2alm_impl(const hb_geom *g, int lmax, int mmax, int nmaps, const void *maps, const double *w, void *alm,
                        void *ws, size_t wsb, int flags, cudaStream_t st, int prec, const char *who) {
    int rc = check_common(g, lmax, mmax, nmaps, who);
    if (rc) return rc;
    if (!maps || !alm) return fail(HB_ERR_INVALID, std::string(who) + ": null data pointer");
    if ((rc = check_ws(ws, wsb, fm_bytes(g, mmax, prec, nmaps), who))) return rc;
    if ((rc = launch_ring_analysis(g->d, prec, nmaps, maps, g->d.npix, w, ws, mmax, flags, false, false, st))) return rc;
    return launch_leg_analysis(g->d, prec, nmaps, lmax, mmax, ws, alm, st);
}

static int alm2map_impl(const hb_geom *g, int lmax, int mmax, int nmaps, const void *alm, void *maps, void *ws,
                        size_t wsb, int flags, cudaStream_t st, int prec, const char *who) {
    int rc = check_common(g, lmax, mmax, nmaps, who);
    if (rc) return rc;
    if (!maps || !alm) return fail(HB_ERR_INVALID, std::string(who) + ": null data pointer");
    if ((rc = check_ws(ws, wsb, fm_bytes(g, mmax, prec, nmaps), who))) return rc;
    if ((rc = launch_leg_synthesis(g->d, prec, nmaps, lmax, mmax, alm, ws, st))) return rc;
    return launch_ring_synthesis(g->d, prec, nmaps, ws, mmax, maps, g->d.npix, nullptr, false, true, flags, st);
}

// transpose of alm2map: ring analysis with unit pixel weights and c_m = 2 for m > 0
static int alm2map_adj_impl(const hb_geom *g, int lmax, int mmax, int nmaps, const void *maps, void *alm, void *ws,
                            size_t wsb, int flags, cudaStream_t st, int prec, const char *who) {
    int rc = check_common(g, lmax, mmax, nmaps, who);
    if (rc) return rc;
    if (!maps || !alm) return fail(HB_ERR_INVALID, std::string(who) + ": null data pointer");
    if ((rc = check_ws(ws, wsb, fm_bytes(g, mmax, prec, nmaps), who))) return rc;
    if ((rc = launch_ring_analysis(g->d, prec, nmaps, maps, g->d.npix, nullptr, ws, mmax, flags & ~HB_F_NOFOLD, true,
                                   true, st)))
        return rc;
    return launch_leg_analysis(g->d, prec, nmaps, lmax, mmax, ws, alm, st);
}

// transpose of map2alm: Legendre synthesis, then ring synthesis with c_m = 1 and pixel weights
static int map2alm_adj_impl(const hb_geom *g, int lmax, int mmax, int nmaps, const void *alm, const double *w,
                            void *maps, void *ws, size_t wsb, int flags, cudaStream_t st, int prec, const char *who) {
    int rc = check_common(g, lmax, mmax, nmaps, who);
    if (rc) return rc;
    if (!maps || !alm) return fail(HB_ERR_INVALID, std::string(who) + ": null data pointer");
    if (flags & HB_F_NOFOLD) return fail(HB_ERR_UNSUPPORTED, std::string(who) + ": HB_F_NOFOLD has no adjoint here");
    if ((rc = check_ws(ws, wsb, fm_bytes(g, mmax, prec, nmaps), who))) return rc;
    if ((rc = launch_leg_synthesis(g->d, prec, nmaps, lmax, mmax, alm, ws, st))) return rc;
    return launch_ring_synthesis(g->d, prec, nmaps, ws, mmax, maps, g->d.npix, w, true, false, flags, st);
}

static int map2alm_spin_impl(const hb_geom *g, int lmax, int mmax, int nmaps, const void *Q, const void *U,
                             const double *w, void *E, void *B, void *ws, size_t wsb, int flags, cudaStream_t st,
                             int prec, const char *who) {
    int rc = check_common(g, lmax, mmax, nmaps, who);
    if (rc) return rc;
    if (!Q || !U || !E || !B) return fail(HB_ERR_INVALID, std::string(who) + ": null data pointer");
    const size_t half = fm_bytes(g, mmax, prec, nmaps);
    if ((rc = check_ws(ws, wsb, 2 * half, who))) return rc;
    char *QF = (char *)ws, *UF = (char *)ws + half;
    if ((rc = launch_ring_analysis(g->d, prec, nmaps, Q, g->d.npix, w, QF, mmax, flags, false, false, st))) return rc;
    if ((rc = launch_ring_analysis(g->d, prec, nmaps, U, g->d.npix, w, UF, mmax, flags, false, false, st))) return rc;
    return launch_spin_analysis(g->d, prec, nmaps, lmax, mmax, QF, UF, E, B, st);
}

static int alm2map_spin_impl(const hb_geom *g, int lmax, int mmax, int nmaps, const void *E, const void *B, void *Q,
                             void *U, void *ws, size_t wsb, int flags, cudaStream_t st, int prec, const char *who) {
    int rc = check_common(g, lmax, mmax, nmaps, who);
    if (rc) return rc;
    if (!Q || !U || !E || !B) return fail(HB_ERR_INVALID, std::string(who) + ": null data pointer");
    const size_t half = fm_bytes(g, mmax, prec, nmaps);
    if ((rc = check_ws(ws, wsb, 2 * half, who))) return rc;
    char *QG = (char *)ws, *UG = (char *)ws + half;
    if ((rc = launch_spin_synthesis(g->d, prec, nmaps, lmax, mmax, E, B, QG, UG, st))) return rc;
    if ((rc = launch_ring_synthesis(g->d, prec, nmaps, QG, mmax, Q, g->d.npix, nullptr, false, true, flags, st)))
        return rc;
    return launch_ring_synthesis(g->d, prec, nmaps, UG, mmax, U, g->d.npix, nullptr, false, true, flags, st);
}

// transpose of alm2map_spin2: ring analysis of (gQ, gU) with unit weights and c_m = 2, then
// the spin analysis kernel
static int alm2map_spin_adj_impl(const hb_geom *g, int lmax, int mmax, int nmaps, const void *gQ, const void *gU,
                                 void *gE, void *gB, void *ws, size_t wsb, int flags, cudaStream_t st, int prec,
                                 const char *who) {
    int rc = check_common(g, lmax, mmax, nmaps, who);
    if (rc) return rc;
    if (!gQ || !gU || !gE || !gB) return fail(HB_ERR_INVALID, std::string(who) + ": null data pointer");
    const size_t half = fm_bytes(g, mmax, prec, nmaps);
    if ((rc = check_ws(ws, wsb, 2 * half, who))) return rc;
    char *QF = (char *)ws, *UF = (char *)ws + half;
    const int f = flags & ~HB_F_NOFOLD;
    if ((rc = launch_ring_analysis(g->d, prec, nmaps, gQ, g->d.npix, nullptr, QF, mmax, f, true, true, st))) return rc;
    if ((rc = launch_ring_analysis(g->d, prec, nmaps, gU, g->d.npix, nullptr, UF, mmax, f, true, true, st))) return rc;
    return launch_spin_analysis(g->d, prec, nmaps, lmax, mmax, QF, UF, gE, gB, st);
}

// transpose of map2alm_spin2: spin synthesis, then ring synthesis with c_m = 1 and pixel weights
static int map2alm_spin_adj_impl(const hb_geom *g, int lmax, int mmax, int nmaps, const void *gE, const void *gB,
                                 const double *w, void *gQ, void *gU, void *ws, size_t wsb, int flags,
                                 cudaStream_t st, int prec, const char *who) {
    int rc = check_common(g, lmax, mmax, nmaps, who);
    if (rc) return rc;
    if (!gQ || !gU || !gE || !gB) return fail(HB_ERR_INVALID, std::string(who) + ": null data pointer");
    if (flags & HB_F_NOFOLD) return fail(HB_ERR_UNSUPPORTED, std::string(who) + ": HB_F_NOFOLD has no adjoint here");
    const size_t half = fm_bytes(g, mmax, prec, nmaps);
    if ((rc = check_ws(ws, wsb, 2 * half, who))) return rc;
    char *QG = (char *)ws, *UG = (char *)ws + half;
    if ((rc = launch_spin_synthesis(g->d, prec, nmaps, lmax, mmax, gE, gB, QG, UG, st))) return rc;
    if ((rc = launch_ring_synthesis(g->d, prec, nmaps, QG, mmax, gQ, g->d.npix, w, true, false, flags, st))) return rc;
    return launch_ring_synthesis(g->d, prec, nmaps, UG, mmax, gU, g->d.npix, w, true, false, flags, st);
}

// alm2cl (alm_ops.py:19-32): one thread per l, m-loop over the l-contiguous healpy columns,
// FP64 accumulation.
template <typename V>
__global__ void alm2cl_kernel(int lmax, int mmax, const V *__restrict__ a1, const V *__restrict__ a2, int64_t stride,
                              double *__restrict__ cl) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    const int b = blockIdx.y;
    if (l > lmax) return;
    const V *p1 = a1 + b * stride, *p2 = (a2 ? a2 : a1) + b * stride;
    const int mtop = l < mmax ? l : mmax;
    double acc0 = 0.0, acc = 0.0;
    {
        V u = p1[l], v = p2[l];
        acc0 = (double)u.x * (double)v.x + (double)u.y * (double)v.y;
    }
    for (int m = 1; m <= mtop; ++m) {
        const int64_t k = alm_idx(lmax, l, m);
        V u = p1[k], v = p2[k];
        acc += (double)u.x * (double)v.x + (double)u.y * (double)v.y;
    }
    cl[(int64_t)b * (lmax + 1) + l] = (acc0 + 2.0 * acc) / (2.0 * l + 1.0);
}

template <typename V>
static int alm2cl_impl(int lmax, int mmax, int nmaps, const V *a1, const V *a2, double *cl, cudaStream_t st) {
    if (lmax < 0 || mmax < 0 || mmax > lmax || nmaps <= 0 || nmaps > 65535 || !a1 || !cl)
        return fail(HB_ERR_INVALID, "hb_alm2cl: bad arguments");
    dim3 grid((unsigned)((lmax + 256) / 256), (unsigned)nmaps);
    alm2cl_kernel<V><<<grid, 256, 0, st>>>(lmax, mmax, a1, a2, alm_size(lmax, mmax), cl);
    HB_CHECK_LAUNCH();
    return HB_OK;
}

}  // namespace hb

using namespace hb;

extern "C" {

size_t hb_sht_workspace_size(const hb_geom *g, int lmax, int mmax, int precision, int nmaps) {
    if (!g || mmax < 0 || nmaps <= 0 || (precision != 32 && precision != 64) || mmax > lmax) return 0;
    return fm_bytes(g, mmax, precision, nmaps);
}

size_t hb_spin2_workspace_size(const hb_geom *g, int lmax, int mmax, int precision, int nmaps) {
    return 2 * hb_sht_workspace_size(g, lmax, mmax, precision, nmaps);
}

int hb_map2alm_f32(const hb_geom *g, int lmax, int mmax, int nmaps, const float *maps, const double *weights,
                   float *alm, void *ws, size_t wsb, int flags, hb_stream_t st) {
    return map2alm_impl(g, lmax, mmax, nmaps, maps, weights, alm, ws, wsb, flags, (cudaStream_t)st, 32,
                        "hb_map2alm_f32");
}
int hb_map2alm_f64(const hb_geom *g, int lmax, int mmax, int nmaps, const double *maps, const double *weights,
                   double *alm, void *ws, size_t wsb, int flags, hb_stream_t st) {
    return map2alm_impl(g, lmax, mmax, nmaps, maps, weights, alm, ws, wsb, flags, (cudaStream_t)st, 64,
                        "hb_map2alm_f64");
}
int hb_alm2map_f32(const hb_geom *g, int lmax, int mmax, int nmaps, const float *alm, float *maps, void *ws,
                   size_t wsb, int flags, hb_stream_t st) {
    return alm2map_impl(g, lmax, mmax, nmaps, alm, maps, ws, wsb, flags, (cudaStream_t)st, 32, "hb_alm2map_f32");
}
int hb_alm2map_f64(const hb_geom *g, int lmax, int mmax, int nmaps, const double *alm, double *maps, void *ws,
                   size_t wsb, int flags, hb_stream_t st) {
    return alm2map_impl(g, lmax, mmax, nmaps, alm, maps, ws, wsb, flags, (cudaStream_t)st, 64, "hb_alm2map_f64");
}
int hb_alm2map_adjoint_f32(const hb_geom *g, int lmax, int mmax, int nmaps, const float *maps, float *alm, void *ws,
                           size_t wsb, int flags, hb_stream_t st) {
    return alm2map_adj_impl(g, lmax, mmax, nmaps, maps, alm, ws, wsb, flags, (cudaStream_t)st, 32,
                            "hb_alm2map_adjoint_f32");
}
int hb_alm2map_adjoint_f64(const hb_geom *g, int lmax, int mmax, int nmaps, const double *maps, double *alm, void *ws,
                           size_t wsb, int flags, hb_stream_t st) {
    return alm2map_adj_impl(g, lmax, mmax, nmaps, maps, alm, ws, wsb, flags, (cudaStream_t)st, 64,
                            "hb_alm2map_adjoint_f64");
}
int hb_map2alm_adjoint_f32(const hb_geom *g, int lmax, int mmax, int nmaps, const float *alm, const double *weights,
                           float *maps, void *ws, size_t wsb, int flags, hb_stream_t st) {
    return map2alm_adj_impl(g, lmax, mmax, nmaps, alm, weights, maps, ws, wsb, flags, (cudaStream_t)st, 32,
                            "hb_map2alm_adjoint_f32");
}
int hb_map2alm_adjoint_f64(const hb_geom *g, int lmax, int mmax, int nmaps, const double *alm, const double *weights,
                           double *maps, void *ws, size_t wsb, int flags, hb_stream_t st) {
    return map2alm_adj_impl(g, lmax, mmax, nmaps, alm, weights, maps, ws, wsb, flags, (cudaStream_t)st, 64,
                            "hb_map2alm_adjoint_f64");
}

int hb_map2alm_spin2_f32(const hb_geom *g, int lmax, int mmax, int nmaps, const float *Q, const float *U,
                         const double *weights, float *E, float *B, void *ws, size_t wsb, int flags, hb_stream_t st) {
    return map2alm_spin_impl(g, lmax, mmax, nmaps, Q, U, weights, E, B, ws, wsb, flags, (cudaStream_t)st, 32,
                             "hb_map2alm_spin2_f32");
}
int hb_map2alm_spin2_f64(const hb_geom *g, int lmax, int mmax, int nmaps, const double *Q, const double *U,
                         const double *weights, double *E, double *B, void *ws, size_t wsb, int flags,
                         hb_stream_t st) {
    return map2alm_spin_impl(g, lmax, mmax, nmaps, Q, U, weights, E, B, ws, wsb, flags, (cudaStream_t)st, 64,
                             "hb_map2alm_spin2_f64");
}
int hb_alm2map_spin2_f32(const hb_geom *g, int lmax, int mmax, int nmaps, const float *E, const float *B, float *Q,
                         float *U, void *ws, size_t wsb, int flags, hb_stream_t st) {
    return alm2map_spin_impl(g, lmax, mmax, nmaps, E, B, Q, U, ws, wsb, flags, (cudaStream_t)st, 32,
                             "hb_alm2map_spin2_f32");
}
int hb_alm2map_spin2_f64(const hb_geom *g, int lmax, int mmax, int nmaps, const double *E, const double *B,
                         double *Q, double *U, void *ws, size_t wsb, int flags, hb_stream_t st) {
    return alm2map_spin_impl(g, lmax, mmax, nmaps, E, B, Q, U, ws, wsb, flags, (cudaStream_t)st, 64,
                             "hb_alm2map_spin2_f64");
}

int hb_alm2map_spin2_adjoint_f32(const hb_geom *g, int lmax, int mmax, int nmaps, const float *gQ, const float *gU,
                                 float *gE, float *gB, void *ws, size_t wsb, int flags, hb_stream_t st) {
    return alm2map_spin_adj_impl(g, lmax, mmax, nmaps, gQ, gU, gE, gB, ws, wsb, flags, (cudaStream_t)st, 32,
                                 "hb_alm2map_spin2_adjoint_f32");
}
int hb_alm2map_spin2_adjoint_f64(const hb_geom *g, int lmax, int mmax, int nmaps, const double *gQ,
                                 const double *gU, double *gE, double *gB, void *ws, size_t wsb, int flags,
                                 hb_stream_t st) {
    return alm2map_spin_adj_impl(g, lmax, mmax, nmaps, gQ, gU, gE, gB, ws, wsb, flags, (cudaStream_t)st, 64,
                                 "hb_alm2map_spin2_adjoint_f64");
}
int hb_map2alm_spin2_adjoint_f32(const hb_geom *g, int lmax, int mmax, int nmaps, const float *gE, const float *gB,
                                 const double *weights, float *gQ, float *gU, void *ws, size_t wsb, int flags,
                                 hb_stream_t st) {
    return map2alm_spin_adj_impl(g, lmax, mmax, nmaps, gE, gB, weights, gQ, gU, ws, wsb, flags, (cudaStream_t)st, 32,
                                 "hb_map2alm_spin2_adjoint_f32");
}
int hb_map2alm_spin2_adjoint_f64(const hb_geom *g, int lmax, int mmax, int nmaps, const double *gE,
                                 const double *gB, const double *weights, double *gQ, double *gU, void *ws,
                                 size_t wsb, int flags, hb_stream_t st) {
    return map2alm_spin_adj_impl(g, lmax, mmax, nmaps, gE, gB, weights, gQ, gU, ws, wsb, flags, (cudaStream_t)st, 64,
                                 "hb_map2alm_spin2_adjoint_f64");
}

// ---- pipeline stages (the pieces the transforms above are made of), for callers that
// keep F/G resident or time the stages separately.  F/G layout: [nmaps][mmax+1][npairs][2].
int hb_ring_analysis(const hb_geom *g, int precision, int mmax, int nmaps, const void *maps, const double *weights,
                     void *F, int flags, hb_stream_t st) {
    int rc = check_common(g, mmax, mmax, nmaps, "hb_ring_analysis");
    if (rc) return rc;
    if ((precision != 32 && precision != 64) || !maps || !F) return fail(HB_ERR_INVALID, "hb_ring_analysis: bad args");
    return launch_ring_analysis(g->d, precision, nmaps, maps, g->d.npix, weights, F, mmax, flags, false, false,
                                (cudaStream_t)st);
}
int hb_ring_synthesis(const hb_geom *g, int precision, int mmax, int nmaps, const void *G, void *maps, int flags,
                      hb_stream_t st) {
    int rc = check_common(g, mmax, mmax, nmaps, "hb_ring_synthesis");
    if (rc) return rc;
    if ((precision != 32 && precision != 64) || !maps || !G) return fail(HB_ERR_INVALID, "hb_ring_synthesis: bad args");
    return launch_ring_synthesis(g->d, precision, nmaps, G, mmax, maps, g->d.npix, nullptr, false, true, flags,
                                 (cudaStream_t)st);
}
int hb_legendre_analysis(const hb_geom *g, int precision, int lmax, int mmax, int nmaps, const void *F, void *alm,
                         hb_stream_t st) {
    int rc = check_common(g, lmax, mmax, nmaps, "hb_legendre_analysis");
    if (rc) return rc;
    if ((precision != 32 && precision != 64) || !F || !alm) return fail(HB_ERR_INVALID, "hb_legendre_analysis: bad args");
    return launch_leg_analysis(g->d, precision, nmaps, lmax, mmax, F, alm, (cudaStream_t)st);
}
int hb_legendre_synthesis(const hb_geom *g, int precision, int lmax, int mmax, int nmaps, const void *alm, void *G,
                          hb_stream_t st) {
    int rc = check_common(g, lmax, mmax, nmaps, "hb_legendre_synthesis");
    if (rc) return rc;
    if ((precision != 32 && precision != 64) || !G || !alm) return fail(HB_ERR_INVALID, "hb_legendre_synthesis: bad args");
    return launch_leg_synthesis(g->d, precision, nmaps, lmax, mmax, alm, G, (cudaStream_t)st);
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

int hb_probe_fp32(int blocks, int threads, int iters, float *out, hb_stream_t st) {
    if (blocks <= 0 || threads <= 0 || threads > 1024 || iters <= 0 || !out)
        return fail(HB_ERR_INVALID, "hb_probe_fp32: bad args");
    fp32_probe_kernel<<<blocks, threads, 0, (cudaStream_t)st>>>(iters, out);
    HB_CHECK_LAUNCH();
    return HB_OK;
}

int hb_alm2cl_f32(int lmax, int mmax, int nmaps, const float *alm1, const float *alm2, double *cl, hb_stream_t st) {
    return alm2cl_impl<float2>(lmax, mmax, nmaps, (const float2 *)alm1, (const float2 *)alm2, cl, (cudaStream_t)st);
}
int hb_alm2cl_f64(int lmax, int mmax, int nmaps, const double *alm1, const double *alm2, double *cl,
                  hb_stream_t st) {
    return alm2cl_impl<double2>(lmax, mmax, nmaps, (const double2 *)alm1, (const double2 *)alm2, cl,
                                (cudaStream_t)st);
}

}  // extern "C"
