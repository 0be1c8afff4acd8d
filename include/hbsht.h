/*
 * hbsht: B200-native (sm_100a) HEALPix spherical-harmonic transforms -- public C ABI.
 *
 * Drop-in boundary for the SHT hot path of hellblast.  Every entry point:
 *   - returns int (HB_OK = 0, negative = error; hb_last_error_string() explains),
 *   - takes device pointers plus explicit sizes and an explicit cudaStream_t,
 *   - allocates nothing on the hot path: transforms take a caller-provided device workspace
 *     whose size the matching *_workspace_size() query returns.
 * Geometry handles (hb_geom) are created once (this allocates) and are immutable afterwards,
 * so one handle may be shared by several host threads and streams.
 *
 * alm layout: healpy m-major, idx(l,m) = m*(2*lmax+1-m)/2 + l, size hb_alm_size(lmax,mmax),
 * complex interleaved (re, im) in the transform's precision.  Maps: RING-ordered flat arrays.
 * Batches: nmaps maps back to back ([nmaps][npix]) and nmaps alm vectors ([nmaps][nalm]).
 *
 * Reference interfaces replaced (file:line within Luce-Morningstar/hellblast):
 *   hb_ring_tables            HealpixRingTables.__init__ + build_ring_tables
 *                             (ring_tables.py:17-37, ring_tables_healpix.cu:5-52);
 *                             weights_dz (ring_tables.py:39-40)
 *   hb_geom_create*           the (thetas, nphi_per_ring, weights_dz) arguments of
 *                             map2alm_gpu / alm2map_gpu (sht_raw.py:30, isht.py:5)
 *   hb_map2alm_{f32,f64}      map2alm_gpu (sht.py:1-4 -> sht_raw.py:30-57, sht_fallback.py:36-65)
 *   hb_alm2map_{f32,f64}      alm2map_gpu (isht.py:5-26)
 *   hb_map2alm_spin2_{f32,f64} map2alm_spin_gpu + eb_from_qu_gpu (spin.py:32-78)
 *   hb_alm2map_spin2_{f32,f64} qu_from_eb_gpu (spin.py:80-115)
 *   hb_alm2cl_{f32,f64}       alm2cl (alm_ops.py:19-32), the reduction inside anafast_ring
 *                             (anafast.py:5-7)
 *   hb_map2alm_adjoint_*, hb_alm2map_adjoint_*, hb_*_spin2_adjoint_*
 *                             no reference counterpart (the reference has no gradients);
 *                             exact transposes used by the autograd wrappers
 *   hb_map2alm_f32_noalloc    no reference counterpart: hb_map2alm_f32 with a static scratch
 *                             for callers that cannot allocate or pass a workspace
 */
#ifndef HBSHT_H
#define HBSHT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define HB_API __attribute__((visibility("default")))
#else
#define HB_API
#endif

typedef struct CUstream_st *hb_stream_t; /* same handle as cudaStream_t */
typedef struct hb_geom hb_geom;

enum {
    HB_OK = 0,
    HB_ERR_INVALID = -1,     /* bad argument (size, nside, lmax, null pointer, ...) */
    HB_ERR_UNSUPPORTED = -2, /* valid request outside what this build implements */
    HB_ERR_CUDA = -3,        /* a CUDA runtime call failed */
    HB_ERR_WORKSPACE = -4,   /* workspace pointer null or smaller than the size query */
    HB_ERR_ALLOC = -5        /* allocation failed while creating a handle */
};

/* phi0 convention of a HEALPix geometry */
enum { HB_PHI0_HEALPIX = 0, HB_PHI0_REFERENCE = 1 };
/* default ring weights of a HEALPix geometry */
enum { HB_WEIGHTS_DZ = 0, HB_WEIGHTS_UNIFORM = 1 };

/* flags of the forward transforms (reference-compatibility switches, all off by default) */
enum {
    HB_F_NOPHASE = 1, /* drop exp(-i m phi0): the reference omits it (sht_raw.py:41) */
    HB_F_NOFOLD = 2,  /* zero for m >= nphi instead of folding m mod nphi (sht_raw.py:51) */
    HB_F_NO2PI = 4    /* omit the 2*pi factor, like sht_raw.py:53 (sht_fallback.py:63 has it) */
};

/* Last error message of the calling thread ("" if none). */
HB_API const char *hb_last_error_string(void);
/* Library version string. */
HB_API const char *hb_version(void);

/* alm vector length for (lmax, mmax), healpy layout. */
HB_API int64_t hb_alm_size(int lmax, int mmax);

/* HEALPix ring tables on the device, nside a power of two (ring_tables.py:19).
 * Outputs (device, any may be NULL): z[Nr], theta[Nr], nphi[Nr], phi0[Nr],
 * ring_start[Nr+1], z_edges[Nr+1], weights_dz[Nr], Nr = 4*nside-1.
 * Integer outputs are bit-exact with the reference; phi0_mode selects HB_PHI0_*. */
HB_API int hb_ring_tables(int64_t nside, int phi0_mode, double *z, double *theta, int32_t *nphi, double *phi0,
                   int64_t *ring_start, double *z_edges, double *weights_dz, hb_stream_t stream);

/* Geometry of a HEALPix RING grid.  weights_mode selects HB_WEIGHTS_*. */
HB_API int hb_geom_create_healpix(int64_t nside, int phi0_mode, int weights_mode, hb_geom **out);
/* Geometry of arbitrary iso-latitude rings (host arrays, length nr).  weights are the
 * reference's per-ring weights (sum 2 for a full sphere): pixel weight = 2*pi*w_r/nphi_r.
 * phi0 may be NULL (all zero).  Ring r's pixels start at the running sum of nphi.
 * nphi_r must be a positive multiple of 2. */
HB_API int hb_geom_create(int64_t nr, const double *theta, const int32_t *nphi, const double *phi0,
                   const double *weights, hb_geom **out);
HB_API int hb_geom_destroy(hb_geom *g);
/* nr, npix, ring pairs used by the Legendre kernels, nside (0 if not HEALPix) */
HB_API int hb_geom_info(const hb_geom *g, int64_t *nr, int64_t *npix, int64_t *npairs, int64_t *nside);
/* Kernel launches one ring-FFT stage of the geometry makes per direction in the given
 * precision (one per transform-length class; no reference counterpart: its FFT is one cuFFT
 * call per ring, sht_raw.py:38-43). */
HB_API int hb_geom_fft_launches(const hb_geom *g, int precision, int *n);

/* Transform plans: a geometry plus (lmax, mmax) plus the FP64-computed checkpoints that
 * re-anchor the FP32 Legendre recursions every 256 l (FP32 transforms need them to stay within
 * 1e-5 of FP64 at lmax ~ 4000; FP64 transforms do not use them).  Creating a plan allocates
 * (about 16 bytes per (m, 256-block of l, ring pair) per table) and runs one FP64 pass; plans
 * are immutable afterwards and may be shared across threads and streams.  The geometry must
 * outlive the plan. */
typedef struct hb_plan hb_plan;
enum { HB_PLAN_FP32 = 1, HB_PLAN_SPIN2_FP32 = 2 };
HB_API int hb_plan_create(const hb_geom *g, int lmax, int mmax, int flags, hb_plan **out);
HB_API int hb_plan_destroy(hb_plan *p);
HB_API size_t hb_plan_bytes(const hb_plan *p);

/* Workspace bytes for one call of the transform family; precision 32 or 64. */
HB_API size_t hb_sht_workspace_size(const hb_plan *p, int precision, int nmaps);
HB_API size_t hb_spin2_workspace_size(const hb_plan *p, int precision, int nmaps);

/* map2alm: alm = sum_pix (2 pi w_r / nphi_r) f(pix) conj(Y_lm(pix)).  maps [nmaps][npix],
 * alm [nmaps][nalm] complex.  weights: device [nr] per-ring weights or NULL (geometry's).
 * FP32 needs a plan made with HB_PLAN_FP32. */
HB_API int hb_map2alm_f32(const hb_plan *p, int nmaps, const float *maps, const double *weights, float *alm,
                          void *ws, size_t ws_bytes, int flags, hb_stream_t stream);
HB_API int hb_map2alm_f64(const hb_plan *p, int nmaps, const double *maps, const double *weights, double *alm,
                          void *ws, size_t ws_bytes, int flags, hb_stream_t stream);
/* hb_map2alm_f32 without a workspace and without allocating: its F(m, ring pair) scratch is a
 * fixed static device array of HB_NOALLOC_SCRATCH_BYTES that every GPU loading this library
 * holds until the process exits.  For callers that may not allocate device memory per call
 * and have no way to pass a workspace (an allocator owned by the host runtime, a plugin ABI
 * without a workspace argument).  No counterpart in the reference.
 * - Calls needing more than the scratch (nmaps * (mmax+1) * npairs * 16 bytes; 64 MiB holds
 *   one map at nside 1024, lmax 2047) return HB_ERR_INVALID.
 * - The first call with a given device current looks up the array's device address (and may
 *   load the module onto that device); make that first call before any stream capture.
 * - All calls share the one array per device: calls that overlap in time on the same device
 *   (two streams, two threads) race on it and give wrong results.  Each call overwrites every
 *   scratch entry it reads, so the leftover contents of an earlier call do not matter. */
#define HB_NOALLOC_SCRATCH_BYTES (64u << 20)
HB_API int hb_map2alm_f32_noalloc(const hb_plan *p, int nmaps, const float *maps, const double *weights,
                                  float *alm, int flags, hb_stream_t stream);

/* alm2map: f(pix) = sum_lm a_lm Y_lm(pix) (real field: m>0 counted twice). */
HB_API int hb_alm2map_f32(const hb_plan *p, int nmaps, const float *alm, float *maps, void *ws, size_t ws_bytes,
                          int flags, hb_stream_t stream);
HB_API int hb_alm2map_f64(const hb_plan *p, int nmaps, const double *alm, double *maps, void *ws, size_t ws_bytes,
                          int flags, hb_stream_t stream);

/* Exact adjoints (transposes, Re and Im of alm as independent real coordinates):
 *   hb_alm2map_adjoint: map-space vector -> alm-space vector, includes the m>0 doubling;
 *   hb_map2alm_adjoint: alm-space vector -> map-space vector, includes the pixel weights. */
HB_API int hb_alm2map_adjoint_f32(const hb_plan *p, int nmaps, const float *maps, float *alm, void *ws,
                                  size_t ws_bytes, int flags, hb_stream_t stream);
HB_API int hb_alm2map_adjoint_f64(const hb_plan *p, int nmaps, const double *maps, double *alm, void *ws,
                                  size_t ws_bytes, int flags, hb_stream_t stream);
HB_API int hb_map2alm_adjoint_f32(const hb_plan *p, int nmaps, const float *alm, const double *weights, float *maps,
                                  void *ws, size_t ws_bytes, int flags, hb_stream_t stream);
HB_API int hb_map2alm_adjoint_f64(const hb_plan *p, int nmaps, const double *alm, const double *weights,
                                  double *maps, void *ws, size_t ws_bytes, int flags, hb_stream_t stream);

/* Spin-2: Q/U maps -> E/B alm (E = -(a2+a-2)/2, B = i(a2-a-2)/2, healpy convention) and back.
 * FP32 needs a plan made with HB_PLAN_SPIN2_FP32. */
HB_API int hb_map2alm_spin2_f32(const hb_plan *p, int nmaps, const float *Q, const float *U, const double *weights,
                                float *E, float *B, void *ws, size_t ws_bytes, int flags, hb_stream_t stream);
HB_API int hb_map2alm_spin2_f64(const hb_plan *p, int nmaps, const double *Q, const double *U,
                                const double *weights, double *E, double *B, void *ws, size_t ws_bytes, int flags,
                                hb_stream_t stream);
HB_API int hb_alm2map_spin2_f32(const hb_plan *p, int nmaps, const float *E, const float *B, float *Q, float *U,
                                void *ws, size_t ws_bytes, int flags, hb_stream_t stream);
HB_API int hb_alm2map_spin2_f64(const hb_plan *p, int nmaps, const double *E, const double *B, double *Q, double *U,
                                void *ws, size_t ws_bytes, int flags, hb_stream_t stream);

/* Exact adjoints of the spin-2 pair (transposes over Re/Im of E and B):
 *   hb_alm2map_spin2_adjoint: (gQ, gU) -> (gE, gB), includes the m>0 doubling;
 *   hb_map2alm_spin2_adjoint: (gE, gB) -> (gQ, gU), includes the pixel weights. */
HB_API int hb_alm2map_spin2_adjoint_f32(const hb_plan *p, int nmaps, const float *gQ, const float *gU, float *gE,
                                        float *gB, void *ws, size_t ws_bytes, int flags, hb_stream_t stream);
HB_API int hb_alm2map_spin2_adjoint_f64(const hb_plan *p, int nmaps, const double *gQ, const double *gU,
                                        double *gE, double *gB, void *ws, size_t ws_bytes, int flags,
                                        hb_stream_t stream);
HB_API int hb_map2alm_spin2_adjoint_f32(const hb_plan *p, int nmaps, const float *gE, const float *gB,
                                        const double *weights, float *gQ, float *gU, void *ws, size_t ws_bytes,
                                        int flags, hb_stream_t stream);
HB_API int hb_map2alm_spin2_adjoint_f64(const hb_plan *p, int nmaps, const double *gE, const double *gB,
                                        const double *weights, double *gQ, double *gU, void *ws, size_t ws_bytes,
                                        int flags, hb_stream_t stream);

/* alm2cl: cl[l] = (Re a_l0 b_l0* + 2 sum_{m>0} Re a_lm b_lm*) / (2l+1); alm2 may be NULL
 * (auto spectrum).  cl is always double [nmaps][lmax+1]. */
HB_API int hb_alm2cl_f32(int lmax, int mmax, int nmaps, const float *alm1, const float *alm2, double *cl,
                  hb_stream_t stream);
HB_API int hb_alm2cl_f64(int lmax, int mmax, int nmaps, const double *alm1, const double *alm2, double *cl,
                  hb_stream_t stream);

/* Batched split-precision transforms on the tcgen05 tensor cores (FP32 data, 16-bit hi+lo
 * three-pass products, FP32 accumulation in TMEM).  One batched plan covers nplans plans (each a
 * geometry + lmax, made with HB_PLAN_FP32) with nmaps[i] maps each; all maps of all plans run
 * in one persistent launch per direction, driven by a (plan, m, ring-block or l-block) work list
 * sorted by decreasing work.  Creating it allocates the operand staging buffers.
 * Buffers: alm = concatenation over plans of [nmaps_i][nalm_i] complex64, maps = concatenation
 * over plans of [nmaps_i][npix_i] float32.  map2alm uses each geometry's default ring weights.
 * hb_batched_status returns the kernels' error word (0 = fine; nonzero = a pipeline wait timed
 * out and the results are invalid); it synchronises with the device.
 * (Replaces, for batches, the per-map loops of sht_raw.py:30-57 and isht.py:5-26.) */
typedef struct hb_batched_plan hb_batched_plan;
/* flags: HB_BATCHED_BF16 splits into BF16 hi+lo (8-bit significands) instead of the default
 * IEEE-half hi+lo with exact power-of-two per-m scaling (11-bit significands); both run at the
 * same tcgen05 kind::f16 rate.
 * The maps run in groups of 32 (MMA N = 64) with four TMEM accumulator sets per output tile:
 * the hi*hi products and the cross products accumulate separately, and successive chunks of the
 * l (or ring-pair) contraction alternate between two such pairs; the sets are summed in FP32 at
 * the end (the tensor core's FP32 accumulation error grows with the number of accumulate steps
 * into one set).  HB_BATCHED_WIDE uses groups of 64 (N = 128) with one (hi, cross) pair: one
 * recursion pass serves twice as many maps, at about twice the accumulation error.
 * Measured relative error of a map2alm+alm2map pair against FP64 at nside 2048, lmax 4095:
 * default 4.9e-6, BF16 6.2e-6, WIDE 8.7e-6. */
enum { HB_BATCHED_BF16 = 1, HB_BATCHED_WIDE = 2 };
HB_API int hb_batched_plan_create(const hb_plan *const *plans, const int *nmaps, int nplans, int flags,
                                  hb_batched_plan **out);
HB_API int hb_batched_plan_destroy(hb_batched_plan *bp);
HB_API size_t hb_batched_plan_bytes(const hb_batched_plan *bp);
HB_API int hb_batched_alm2map(hb_batched_plan *bp, const float *alm, float *maps, hb_stream_t stream);
HB_API int hb_batched_map2alm(hb_batched_plan *bp, const float *maps, float *alm, hb_stream_t stream);
/* hb_batched_map2alm with a per-l filter fused into the alm store: alm(l, m) *= fl[l] (device
 * float array, at least max lmax + 1 entries over the plans; null = none).  The beam / pixel-window
 * step of the smoothing pipeline (almxfl after map2alm; beams.py:38-47, smoothing.py:5-14). */
HB_API int hb_batched_map2alm_fl(hb_batched_plan *bp, const float *maps, float *alm, const float *fl,
                                 hb_stream_t stream);
HB_API int hb_batched_status(hb_batched_plan *bp, int *code);
/* Failure-detection test hook (no reference counterpart): every mbarrier wait of the plan's
 * tensor-core kernels gives up after wait_ns (default 2 s) and records an error code that
 * hb_batched_status returns; with withhold_copy = 1 the synthesis kernel's loader in CTA 0
 * skips its first batch-tile copy, so the waits on that stage run out, the kernel records the
 * error and returns (the CUDA context stays usable).  hb_batched_reset_status clears the code. */
HB_API int hb_batched_fault_test(hb_batched_plan *bp, uint64_t wait_ns, int withhold_copy);
HB_API int hb_batched_reset_status(hb_batched_plan *bp);
/* Work the tensor-core kernels execute per call after the evanescent skip: chunks[0] synthesis
 * chunks (64 l x 128 ring pairs each), chunks[1] analysis chunks (32 ring pairs x 256 l each);
 * every chunk is the work of 12 MMAs of 128 x mma_n x 16.  (No counterpart in the reference.) */
HB_API int hb_batched_work(const hb_batched_plan *bp, int64_t *chunks, int *mma_n);
/* CUDA graph of a batched step: hb_batched_graph_capture records hb_batched_alm2map(alm -> maps)
 * then hb_batched_map2alm(maps -> alm_out) (alm or alm_out may be null to keep one direction)
 * on a private stream into an executable graph owned by the plan, replacing an earlier one; the
 * buffer pointers are part of the graph.  hb_batched_graph_launch replays it on `stream`: one
 * launch for the whole step, no host work per kernel.  (No counterpart in the reference, whose
 * per-ring host loops cannot be captured.) */
HB_API int hb_batched_graph_capture(hb_batched_plan *bp, const float *alm, float *maps, float *alm_out);
HB_API int hb_batched_graph_launch(hb_batched_plan *bp, hb_stream_t stream);
/* Profiling: with enable != 0 every exec records CUDA events between its kernels (do not enable
 * while capturing a CUDA graph); hb_batched_stage_ms then returns the last calls' stage times in
 * ms: [alm tile prep, tensor synthesis, ring synthesis, ring analysis, F tile prep, tensor
 * analysis] (synchronises). */
HB_API int hb_batched_profile(hb_batched_plan *bp, int enable);
HB_API int hb_batched_stage_ms(hb_batched_plan *bp, float *ms);

/* Pipeline stages (what the transforms are made of), for callers that keep the per-ring
 * Fourier coefficients resident or time the stages.  F / G: complex, precision 32 or 64,
 * layout [nmaps][mmax+1][npairs][2] (north, south ring of each pair), npairs from hb_geom_info.
 *   hb_ring_analysis:      maps -> F (weights, phi0 phase, alias fold; flags as map2alm)
 *   hb_legendre_analysis:  F -> alm
 *   hb_legendre_synthesis: alm -> G
 *   hb_ring_synthesis:     G -> maps
 * (sht_raw.py:38-43 / 46-56 and isht.py:11-25 are the reference's versions of these steps.) */
HB_API int hb_ring_analysis(const hb_plan *p, int precision, int nmaps, const void *maps, const double *weights,
                            void *F, int flags, hb_stream_t stream);
HB_API int hb_ring_synthesis(const hb_plan *p, int precision, int nmaps, const void *G, void *maps, int flags,
                             hb_stream_t stream);
HB_API int hb_legendre_analysis(const hb_plan *p, int precision, int nmaps, const void *F, void *alm,
                                hb_stream_t stream);
/* The Legendre stages restricted to a list of orders, for a transform split over several GPUs by
 * m (each rank transforms its own orders after the all-to-all exchange of the ring-FFT output).
 * mlist: device array of nm orders (an order outside [0, mmax] is skipped); F / G hold one row
 * [npairs][2] per listed order, in list order; alm is the full healpy-layout array of which only
 * the listed orders' entries are written (the analysis may clear the others).  The reference
 * has no multi-GPU path; these split sht_raw.py:46-56 (analysis) and isht.py:11-24 (synthesis)
 * by order. */
HB_API int hb_legendre_analysis_ms(const hb_plan *p, int precision, int nmaps, int nm, const int32_t *mlist,
                                   const void *F, void *alm, hb_stream_t stream);
HB_API int hb_legendre_synthesis_ms(const hb_plan *p, int precision, int nmaps, int nm, const int32_t *mlist,
                                    const void *alm, void *G, hb_stream_t stream);
HB_API int hb_legendre_synthesis(const hb_plan *p, int precision, int nmaps, const void *alm, void *G,
                                 hb_stream_t stream);

/* HEALPix pixel indexing (Gorski et al. 2005): every array is device memory, n points; bad is one
 * device int that a kernel sets to 1 when an input is out of range (that output becomes -1 /
 * NaN).  nside: a power of 2.
 *   hb_ring2nest / hb_nest2ring: index conversion (replace order_convert.py:8-34, which goes
 *     through angles; Ring2NestLUT in nested.py:19-41 needs healpy);
 *   hb_pix2ang: pixel centres; HB_PIX_NEST for NESTED input (replaces nested_pix2ang.cu:16-85),
 *     else RING (coords_ring.cu:30-54); HB_PIX_REFERENCE (RING only) uses the reference's phi0
 *     table phi0_ref (nr entries, from hb_ring_tables with HB_PHI0_REFERENCE) and its wrap;
 *   hb_ang2pix: the pixel holding (theta, phi): NESTED (what nested_gpu.cu:27-95 sets out to do)
 *     or RING; HB_PIX_REFERENCE (RING only) reproduces coords_ring.py:18-24 + coords_ring.cu:9-29
 *     (ring from the z_edges table, nr + 1 entries, then the nearest phi centre);
 *   hb_reorder: map reordering RING -> NESTED (to_nest = 1) or back, nmaps maps of 12 nside^2
 *     float (precision 32) or double (64) values, out of place. */
enum { HB_PIX_NEST = 1, HB_PIX_REFERENCE = 2 };
HB_API int hb_ring2nest(int64_t nside, int64_t n, const int64_t *ring, int64_t *nest, int *bad, hb_stream_t stream);
HB_API int hb_nest2ring(int64_t nside, int64_t n, const int64_t *nest, int64_t *ring, int *bad, hb_stream_t stream);
HB_API int hb_pix2ang(int64_t nside, int flags, const double *phi0_ref, int64_t n, const int64_t *pix, double *theta,
                      double *phi, int *bad, hb_stream_t stream);
HB_API int hb_ang2pix(int64_t nside, int flags, const double *z_edges, const double *phi0_ref, int64_t n,
                      const double *theta, const double *phi, int64_t *pix, int *bad, hb_stream_t stream);
HB_API int hb_reorder(int64_t nside, int to_nest, int precision, int nmaps, const void *in, void *out,
                      hb_stream_t stream);

/* Wigner d and alm rotation (FP64; device arrays).
 *   hb_wigner_d: d^l_{m m'}(beta_b) for m, m' = -l..l into out[b][m + l][m' + l] (what
 *     wigner_d_fast.cu:8-52 and wigner_full.py:12-40 compute by the closed-form sum; here by the
 *     three-term recursion in l, stable to l = 16383);
 *   hb_rotate_alm: a'_{lm} = sum_m' exp(-i m alpha) d^l_{mm'}(beta) exp(-i m' gamma) a_{lm'}
 *     (Euler ZYZ, rotate_alm_euler.py:5-14 / wigner_full.py:79-96) for nmaps healpy-layout
 *     complex128 alm vectors with mmax = lmax, out of place. */
HB_API int hb_wigner_d(int l, int nbeta, const double *beta, double *out, hb_stream_t stream);
HB_API int hb_rotate_alm(int lmax, int nmaps, const void *alm_in, void *alm_out, double alpha, double beta,
                         double gamma, hb_stream_t stream);

/* Diagnostics (no reference counterpart): FP32 FMA throughput probe, blocks*threads threads
 * each running iters*8 FMAs; out holds blocks*threads floats.  Used by bench.py to measure the
 * FP32-pipe roofline on the running GPU. */
HB_API int hb_probe_fp32(int blocks, int threads, int iters, float *out, hb_stream_t stream);

#ifdef __cplusplus
}
#endif
#endif /* HBSHT_H */
