// Ring geometry: the HEALPix ring-table kernel and the device-resident geometry handle.
//
// hb_ring_tables restates HealpixRingTables (ring_tables.py:17-40) and its kernel
// build_ring_tables (ring_tables_healpix.cu:5-52): the same double expressions for z and the
// same integer nphi, so z, theta, nphi, ring_start and z_edges are bit-identical to the
// reference.  Differences by design: one thread per ring with ring_start in closed form
// (no serial scan by thread 0), and phi0 in either the HEALPix convention (default) or the
// reference's, which sits +1/2 pixel off on the equatorial belt (ring_tables_healpix.cu:25-27).
#include <algorithm>
#include <cstdlib>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "hb_internal.cuh"

namespace hb {

static thread_local std::string g_last_error;
void set_error(const std::string &msg) { g_last_error = msg; }
int fail(int code, const std::string &msg) {
    g_last_error = msg;
    return code;
}

// z of 1-based ring i, the exact double expressions of ring_tables_healpix.cu:17,23,30
__host__ __device__ __forceinline__ double ring_z(int64_t nside, int64_t i) {
    if (i < nside) return 1.0 - (double)(i * i) / (3.0 * (double)(nside * nside));
    if (i <= 3 * nside) return (double)(2 * nside - i) * (2.0 / (3.0 * (double)nside));
    int64_t ip = 4 * nside - i;
    return -(1.0 - (double)(ip * ip) / (3.0 * (double)(nside * nside)));
}
__host__ __device__ __forceinline__ int ring_nphi(int64_t nside, int64_t i) {
    if (i < nside) return 4 * (int)i;
    if (i <= 3 * nside) return 4 * (int)nside;
    return 4 * (int)(4 * nside - i);
}
// first pixel of 1-based ring i (closed form of the prefix sum, ring_tables_healpix.cu:42-45)
__host__ __device__ __forceinline__ int64_t ring_first(int64_t nside, int64_t i) {
    int64_t ncap = 2 * nside * (nside - 1), npix = 12 * nside * nside;
    if (i <= nside) return 2 * i * (i - 1);
    if (i <= 3 * nside) return ncap + (i - nside) * 4 * nside;
    int64_t ip = 4 * nside - i;  // this ring and the ip-1 rings south of it hold 2 ip (ip+1) pixels
    return npix - 2 * ip * (ip + 1);
}
__host__ __device__ __forceinline__ double ring_phi0(int64_t nside, int64_t i, int healpix) {
    const double pi = 3.141592653589793238462643383279502884;
    int npr = ring_nphi(nside, i);
    double dphi = 2.0 * pi / (double)npr;
    if (i < nside || i > 3 * nside) return 0.5 * dphi;
    int s = (int)((i - nside) & 1);
    if (healpix) return s ? 0.0 : 0.5 * dphi;
    return (1.0 - 0.5 * (double)s) * dphi;
}

__global__ void ring_tables_kernel(int64_t nside, int healpix, double *z, double *theta, int32_t *nphi,
                                   double *phi0, int64_t *ring_start, double *z_edges, double *wdz) {
    int64_t nr = 4 * nside - 1;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x + 1; i <= nr + 1;
         i += (int64_t)gridDim.x * blockDim.x) {
        if (i <= nr) {
            double zz = ring_z(nside, i);
            if (z) z[i - 1] = zz;
            if (theta) theta[i - 1] = acos(fmax(-1.0, fmin(1.0, zz)));
            if (nphi) nphi[i - 1] = ring_nphi(nside, i);
            if (phi0) phi0[i - 1] = ring_phi0(nside, i, healpix);
            if (ring_start) ring_start[i - 1] = ring_first(nside, i);
            // z_edges[i-1] = midpoint of rings i-1 and i (ring_tables_healpix.cu:46-50)
            double ehi = (i == 1) ? 1.0 : 0.5 * (ring_z(nside, i - 1) + zz);
            double elo = (i == nr) ? -1.0 : 0.5 * (zz + ring_z(nside, i + 1));
            if (z_edges) z_edges[i - 1] = ehi;
            if (wdz) wdz[i - 1] = ehi - elo;
        } else {
            if (ring_start) ring_start[nr] = 12 * nside * nside;
            if (z_edges) z_edges[nr] = -1.0;
        }
    }
}

static bool is_pow2(int64_t v) { return v > 0 && (v & (v - 1)) == 0; }
static int64_t next_pow2(int64_t v) {
    int64_t p = 1;
    while (p < v) p <<= 1;
    return p;
}

// log2 tables of the sectoral start constants (long double on the host)
static void fill_log2_tables(std::vector<double> &cm, std::vector<double> &spin) {
    const long double fpi = 4.0L * 3.141592653589793238462643383279502884L;
    cm.resize(HB_MAX_L + 1);
    spin.resize(HB_MAX_L + 1);
    long double acc = 0.5L * log2l(1.0L / fpi);
    cm[0] = (double)acc;
    for (int m = 1; m <= HB_MAX_L; ++m) {
        acc += 0.5L * log2l((long double)(2 * m + 1) / (long double)(2 * m));
        cm[m] = (double)acc;
    }
    const long double ln2 = logl(2.0L);
    auto lf = [&](int n) { return lgammal((long double)n + 1.0L) / ln2; };
    for (int m = 0; m <= HB_MAX_L; ++m) {
        if (m >= 2)  // sqrt((2m)!/((m+2)!(m-2)!)) * N_m
            spin[m] = (double)(0.5L * (lf(2 * m) - lf(m + 2) - lf(m - 2)) + 0.5L * log2l((2 * m + 1) / fpi));
        else  // sqrt(24/((2+m)!(2-m)!)) * N_2
            spin[m] = (double)(0.5L * (lf(4) - lf(2 + m) - lf(2 - m)) + 0.5L * log2l(5.0L / fpi));
    }
}

struct HostGeom {
    std::vector<int32_t> nphi, ring_pair, ring_side, pair_ring, fft_len, blu_owner;
    std::vector<int64_t> ofs, blu_ofs;
    std::vector<double> phi0_pi, w, pair_x, pair_log2sin, pair_log2ch, pair_log2sh;
    std::vector<float> pair_xhi, pair_xlo;
    int64_t npix = 0, blu_total = 0;
    int max_fft_len = 1, max_nphi = 0;
};

// x, sin theta, cos(theta/2), sin(theta/2) of each pair are passed in from the caller in the
// most accurate form available (exact rationals on the HEALPix grid).
static int finish_geom(HostGeom &h, int64_t nside, const std::vector<double> &xn, const std::vector<double> &sn,
                       const std::vector<double> &chn, const std::vector<double> &shn, hb_geom **out) {
    const int64_t nr = (int64_t)h.nphi.size(), np = (int64_t)h.pair_x.size();
    (void)xn; (void)sn; (void)chn; (void)shn;
    // ragged FFT plan
    h.fft_len.resize(nr);
    h.blu_ofs.resize(nr);
    std::map<int64_t, int64_t> blu_of_N;
    for (int64_t r = 0; r < nr; ++r) {
        int64_t N = h.nphi[r] / 2;
        if (is_pow2(N)) {
            h.fft_len[r] = (int32_t)N;
            h.blu_ofs[r] = -1;
        } else {
            int64_t L = next_pow2(2 * N - 1);
            h.fft_len[r] = (int32_t)L;
            auto it = blu_of_N.find(N);
            if (it == blu_of_N.end()) {
                blu_of_N[N] = h.blu_total;
                h.blu_ofs[r] = h.blu_total;
                h.blu_owner.push_back((int32_t)r);
                h.blu_total += L + N;  // chirp spectrum (L entries), then the chirp itself (N entries)
            } else {
                h.blu_ofs[r] = it->second;
            }
        }
        h.max_fft_len = std::max<int>(h.max_fft_len, h.fft_len[r]);
        h.max_nphi = std::max<int>(h.max_nphi, h.nphi[r]);
    }
    std::vector<double> cm, spin;
    fill_log2_tables(cm, spin);
    int log_tw = 1;
    while ((1 << log_tw) < h.max_fft_len) ++log_tw;
    // pair classes by convolution length
    std::vector<std::pair<int32_t, int32_t>> pl;
    for (int64_t p = 0; p < np; ++p) {
        const int32_t rn = h.pair_ring[2 * p], rs = h.pair_ring[2 * p + 1];
        pl.push_back({std::max(h.fft_len[rn], rs >= 0 ? h.fft_len[rs] : 0), (int32_t)p});
    }
    std::sort(pl.begin(), pl.end());
    std::vector<int32_t> cls_pairs(np), cls_L;
    std::vector<int64_t> cls_first;
    for (int64_t i = 0; i < np; ++i) {
        cls_pairs[i] = pl[i].second;
        if (i == 0 || pl[i].first != pl[i - 1].first) {
            cls_L.push_back(pl[i].first);
            cls_first.push_back(i);
        }
    }
    cls_first.push_back(np);
    if (cls_L.size() > 32) return fail(HB_ERR_UNSUPPORTED, "hb_geom: more than 32 FFT length classes");
    // FP32: the pairs of the pair-packed kernels by (log2 L, Bluestein), the rest as above
    // (HB_NO_PAIR_PACK set in the environment keeps every pair on the general kernels,
    // HB_NO_PAIR_PACK_BLU the Bluestein pairs)
    const bool pack = std::getenv("HB_NO_PAIR_PACK") == nullptr;
    const bool pack_blu = std::getenv("HB_NO_PAIR_PACK_BLU") == nullptr;
    const bool quad_ok = std::getenv("HB_NO_QUAD_SPLIT") == nullptr;  // HB_NO_QUAD_SPLIT: whole-ring Bluestein
    std::vector<std::pair<int32_t, int32_t>> pk, rest;
    std::vector<int64_t> pkb_ofs(np, -1);
    std::map<int, int64_t> bt_of_n;  // ring length -> offset of its chirp spectrum
    std::vector<int32_t> bt_n, bt_rn, bt_logL;  // chirp length, ring length, log2 chirp transform length
    std::vector<int64_t> bt_ofs;
    int64_t bt_total = 0;
    int pk_max_log = 0;
    for (int64_t i = 0; i < np; ++i) {
        const int32_t p = pl[i].second, rn = h.pair_ring[2 * p], rs = h.pair_ring[2 * p + 1];
        int lg = 0;
        bool blu = false;
        if (pack && pk_pair_ok(h.nphi[rn], rs >= 0 ? h.nphi[rs] : -1, h.phi0_pi[rn], rs >= 0 ? h.phi0_pi[rs] : 0.0, &lg,
                               &blu) && (pack_blu || !blu)) {
            const int lq = (blu && quad_ok) ? pk_quad_log(h.nphi[rn], lg) : 0;  // quad split: 4 x length n/4
            const int lc = lq ? lq : lg;                                          // chirp transform length
            pk.push_back({lc | (blu ? 256 : 0) | (lq ? 512 : 0), p});
            pk_max_log = std::max(pk_max_log, lc);
            if (blu) {
                auto it = bt_of_n.find(h.nphi[rn]);
                if (it == bt_of_n.end()) {
                    it = bt_of_n.emplace(h.nphi[rn], bt_total).first;
                    bt_n.push_back(lq ? h.nphi[rn] / 4 : h.nphi[rn]);
                    bt_rn.push_back(h.nphi[rn]);
                    bt_logL.push_back(lc);
                    bt_ofs.push_back(bt_total);
                    bt_total += pk_bt_entries(lc, lq != 0);  // chirp spectrum, chirp, phase block
                }
                pkb_ofs[p] = it->second;
            }
        } else {
            rest.push_back(pl[i]);
        }
    }
    if (pk_max_log > log_tw) log_tw = pk_max_log;  // the FP64 chirp-spectrum transforms use the table
    std::sort(pk.begin(), pk.end());
    std::vector<int32_t> pk_pairs(np, 0), rest_pairs(np, 0), pk_logn, rest_L;
    std::vector<int64_t> pk_first, rest_first;
    for (size_t i = 0; i < pk.size(); ++i) {
        pk_pairs[i] = pk[i].second;
        if (i == 0 || pk[i].first != pk[i - 1].first) {
            pk_logn.push_back(pk[i].first);
            pk_first.push_back((int64_t)i);
        }
    }
    pk_first.push_back((int64_t)pk.size());
    if (pk_logn.size() > 16) return fail(HB_ERR_UNSUPPORTED, "hb_geom: more than 16 pair-packed classes");
    for (size_t i = 0; i < rest.size(); ++i) {
        rest_pairs[i] = rest[i].second;
        if (i == 0 || rest[i].first != rest[i - 1].first) {
            rest_L.push_back(rest[i].first);
            rest_first.push_back((int64_t)i);
        }
    }
    rest_first.push_back((int64_t)rest.size());

    // one device allocation carved into 256-byte aligned pieces
    size_t total = 0;
    auto carve = [&](size_t bytes) {
        size_t o = total;
        total += (bytes + 255) & ~(size_t)255;
        return o;
    };
    size_t o_nphi = carve(4 * nr), o_ofs = carve(8 * nr), o_phi0 = carve(8 * nr), o_w = carve(8 * nr),
           o_rp = carve(4 * nr), o_rs = carve(4 * nr), o_pr = carve(8 * np), o_px = carve(8 * np),
           o_pxh = carve(4 * np), o_pxl = carve(4 * np), o_pls = carve(8 * np), o_plc = carve(8 * np),
           o_plh = carve(8 * np), o_fl = carve(4 * nr), o_bo = carve(8 * nr), o_b64 = carve(16 * (h.blu_total + 1)),
           o_b32 = carve(8 * (h.blu_total + 1)), o_bw = carve(4 * (h.blu_owner.size() + 1)), o_cm = carve(8 * (HB_MAX_L + 1)), o_sp = carve(8 * (HB_MAX_L + 1)),
           o_t64 = carve(16 * ((size_t)1 << (log_tw - 1))), o_t32 = carve(8 * ((size_t)1 << (log_tw - 1))),
           o_cp = carve(4 * (size_t)np), o_pk = carve(4 * (size_t)np), o_rest = carve(4 * (size_t)np),
           o_pkbo = carve(8 * (size_t)np), o_bt = carve(8 * (size_t)(bt_total + 1)),
           o_btn = carve(4 * (bt_n.size() + 1)), o_btl = carve(4 * (bt_n.size() + 1)), o_bto = carve(8 * (bt_n.size() + 1)),
           o_btr = carve(4 * (bt_n.size() + 1));
    int64_t tw_ofs[PK_MAX_LOG + 1] = {}, tw_total = 0;  // pair-packed table blocks per length class
    for (int lg = PK_MIN_LOG; lg <= PK_MAX_LOG; ++lg) {
        tw_ofs[lg] = tw_total;
        tw_total += (pk_tab_entries(lg) + 1) & ~int64_t(1);
    }
    const size_t o_ptw = carve(8 * (size_t)tw_total);
    char *base = nullptr;
    if (cudaMalloc(&base, total) != cudaSuccess) {
        cudaGetLastError();
        return fail(HB_ERR_ALLOC, "hb_geom: cudaMalloc of " + std::to_string(total) + " bytes failed");
    }
    hb_geom *g = new hb_geom();
    g->alloc_base = base;
    g->nside = nside;
    GeomDev &d = g->d;
    d.nr = nr; d.npix = h.npix; d.npairs = np;
    d.nphi = (int32_t *)(base + o_nphi); d.ofs = (int64_t *)(base + o_ofs); d.phi0_pi = (double *)(base + o_phi0);
    d.w = (double *)(base + o_w); d.ring_pair = (int32_t *)(base + o_rp); d.ring_side = (int32_t *)(base + o_rs);
    d.pair_ring = (int32_t *)(base + o_pr); d.pair_x = (double *)(base + o_px); d.pair_xhi = (float *)(base + o_pxh);
    d.pair_xlo = (float *)(base + o_pxl); d.pair_log2sin = (double *)(base + o_pls);
    d.pair_log2ch = (double *)(base + o_plc); d.pair_log2sh = (double *)(base + o_plh);
    d.fft_len = (int32_t *)(base + o_fl); d.blu_ofs = (int64_t *)(base + o_bo);
    d.blu_f64 = (double2 *)(base + o_b64); d.blu_f32 = (float2 *)(base + o_b32);
    d.blu_owner = (int32_t *)(base + o_bw); d.n_blu = (int64_t)h.blu_owner.size();
    d.log2cm = (double *)(base + o_cm); d.log2spin = (double *)(base + o_sp);
    d.max_fft_len = h.max_fft_len; d.max_nphi = h.max_nphi;
    d.tw64 = (double2 *)(base + o_t64); d.tw32 = (float2 *)(base + o_t32); d.log_tw = log_tw;
    d.cls_pairs = (int32_t *)(base + o_cp); d.n_cls = (int)cls_L.size();
    for (size_t c = 0; c < cls_L.size(); ++c) { d.cls_L[c] = cls_L[c]; d.cls_first[c] = cls_first[c]; }
    d.cls_first[cls_L.size()] = np;
    d.pk_pairs = (int32_t *)(base + o_pk); d.pk_n_cls = (int)pk_logn.size();
    for (size_t c = 0; c < pk_logn.size(); ++c) { d.pk_logn[c] = pk_logn[c]; d.pk_first[c] = pk_first[c]; }
    d.pk_first[pk_logn.size()] = pk_first.back();
    d.pkb_bt = (float2 *)(base + o_bt); d.pkb_bt_ofs = (int64_t *)(base + o_pkbo);
    d.pk_tw = (float2 *)(base + o_ptw);
    for (int lg = 0; lg <= PK_MAX_LOG; ++lg) d.pk_tw_ofs[lg] = tw_ofs[lg];
    d.rest_pairs = (int32_t *)(base + o_rest); d.rest_n_cls = (int)rest_L.size();
    for (size_t c = 0; c < rest_L.size(); ++c) { d.rest_L[c] = rest_L[c]; d.rest_first[c] = rest_first[c]; }
    d.rest_first[rest_L.size()] = rest_first.back();
    struct Up { void *dst; const void *src; size_t n; } ups[] = {
        {d.nphi, h.nphi.data(), 4 * (size_t)nr}, {d.ofs, h.ofs.data(), 8 * (size_t)nr},
        {d.phi0_pi, h.phi0_pi.data(), 8 * (size_t)nr}, {d.w, h.w.data(), 8 * (size_t)nr},
        {d.ring_pair, h.ring_pair.data(), 4 * (size_t)nr}, {d.ring_side, h.ring_side.data(), 4 * (size_t)nr},
        {d.pair_ring, h.pair_ring.data(), 8 * (size_t)np}, {d.pair_x, h.pair_x.data(), 8 * (size_t)np},
        {d.pair_xhi, h.pair_xhi.data(), 4 * (size_t)np}, {d.pair_xlo, h.pair_xlo.data(), 4 * (size_t)np},
        {d.pair_log2sin, h.pair_log2sin.data(), 8 * (size_t)np}, {d.pair_log2ch, h.pair_log2ch.data(), 8 * (size_t)np},
        {d.pair_log2sh, h.pair_log2sh.data(), 8 * (size_t)np}, {d.fft_len, h.fft_len.data(), 4 * (size_t)nr},
        {d.blu_ofs, h.blu_ofs.data(), 8 * (size_t)nr},
        {d.blu_owner, h.blu_owner.data(), 4 * h.blu_owner.size()}, {d.log2cm, cm.data(), 8 * (size_t)(HB_MAX_L + 1)},
        {d.log2spin, spin.data(), 8 * (size_t)(HB_MAX_L + 1)}, {d.cls_pairs, cls_pairs.data(), 4 * (size_t)np},
        {d.pk_pairs, pk_pairs.data(), 4 * (size_t)np}, {d.rest_pairs, rest_pairs.data(), 4 * (size_t)np},
        {d.pkb_bt_ofs, pkb_ofs.data(), 8 * (size_t)np}, {base + o_btn, bt_n.data(), 4 * bt_n.size()},
        {base + o_btl, bt_logL.data(), 4 * bt_n.size()}, {base + o_bto, bt_ofs.data(), 8 * bt_n.size()},
        {base + o_btr, bt_rn.data(), 4 * bt_n.size()}};
    for (auto &u : ups) {
        if (cudaMemcpy(u.dst, u.src, u.n, cudaMemcpyHostToDevice) != cudaSuccess) {
            cudaGetLastError();
            cudaFree(base);
            delete g;
            return fail(HB_ERR_CUDA, "hb_geom: upload failed");
        }
    }
    int rc = build_fft_tables(d, 0);
    if (rc == HB_OK && !bt_n.empty())
        rc = build_pk_chirp_tables(d, (int)bt_n.size(), (const int32_t *)(base + o_btn), (const int32_t *)(base + o_btl),
                                   (const int64_t *)(base + o_bto), pk_max_log, d.pkb_bt, 0);
    if (rc == HB_OK)
        rc = build_pk_tables(d, (int)bt_n.size(), (const int32_t *)(base + o_btn), (const int32_t *)(base + o_btr),
                             (const int32_t *)(base + o_btl), (const int64_t *)(base + o_bto), 0);
    if (rc == HB_OK && cudaStreamSynchronize(0) != cudaSuccess) rc = fail(HB_ERR_CUDA, "hb_geom: table build failed");
    if (rc != HB_OK) {
        cudaFree(base);
        delete g;
        return rc;
    }
    *out = g;
    return HB_OK;
}

// Pair rings r and nr-1-r when they mirror each other; the rest stay unpaired.
static void make_pairs(HostGeom &h, const std::vector<double> &theta, const std::vector<double> &x,
                       const std::vector<double> &s, const std::vector<double> &ch, const std::vector<double> &sh) {
    const double pi = 3.141592653589793238462643383279502884;
    int64_t nr = (int64_t)theta.size();
    h.ring_pair.assign(nr, -1);
    h.ring_side.assign(nr, 0);
    for (int64_t r = 0; r < nr; ++r) {
        if (h.ring_pair[r] >= 0) continue;
        int64_t q = nr - 1 - r;
        bool mirror = q > r && std::fabs(theta[r] + theta[q] - pi) <= 1e-12 * pi && theta[r] < 0.5 * pi;
        int64_t p = (int64_t)h.pair_x.size();
        h.pair_ring.push_back((int32_t)r);
        h.pair_ring.push_back(mirror ? (int32_t)q : -1);
        h.ring_pair[r] = (int32_t)p;
        if (mirror) {
            h.ring_pair[q] = (int32_t)p;
            h.ring_side[q] = 1;
        }
        h.pair_x.push_back(x[r]);
        float xh = (float)x[r];
        h.pair_xhi.push_back(xh);
        h.pair_xlo.push_back((float)(x[r] - (double)xh));
        h.pair_log2sin.push_back(std::log2(s[r]));
        h.pair_log2ch.push_back(std::log2(ch[r]));
        h.pair_log2sh.push_back(std::log2(sh[r]));
    }
}

}  // namespace hb

using namespace hb;

extern "C" {

const char *hb_last_error_string(void) { return g_last_error.c_str(); }
const char *hb_version(void) { return "hbsht 0.2.0 (sm_100a)"; }
int64_t hb_alm_size(int lmax, int mmax) {
    if (lmax < 0 || mmax < 0 || mmax > lmax) return -1;
    return alm_size(lmax, mmax);
}

int hb_ring_tables(int64_t nside, int phi0_mode, double *z, double *theta, int32_t *nphi, double *phi0,
                   int64_t *ring_start, double *z_edges, double *weights_dz, hb_stream_t stream) {
    if (!is_pow2(nside) || nside > (1 << 20))
        return fail(HB_ERR_INVALID, "hb_ring_tables: nside must be a power of 2 (ring_tables.py:19)");
    if (phi0_mode != HB_PHI0_HEALPIX && phi0_mode != HB_PHI0_REFERENCE)
        return fail(HB_ERR_INVALID, "hb_ring_tables: bad phi0_mode");
    int64_t nr = 4 * nside - 1;
    int threads = 256;
    int blocks = (int)std::min<int64_t>((nr + 1 + threads - 1) / threads, 148 * 8);
    ring_tables_kernel<<<blocks, threads, 0, (cudaStream_t)stream>>>(nside, phi0_mode == HB_PHI0_HEALPIX ? 1 : 0, z,
                                                                      theta, nphi, phi0, ring_start, z_edges,
                                                                      weights_dz);
    HB_CHECK_LAUNCH();
    return HB_OK;
}

int hb_geom_create_healpix(int64_t nside, int phi0_mode, int weights_mode, hb_geom **out) {
    if (!out) return fail(HB_ERR_INVALID, "hb_geom_create_healpix: out is NULL");
    if (!is_pow2(nside) || nside > 8192)
        return fail(HB_ERR_INVALID, "hb_geom_create_healpix: nside must be a power of 2 <= 8192");
    if (phi0_mode != HB_PHI0_HEALPIX && phi0_mode != HB_PHI0_REFERENCE)
        return fail(HB_ERR_INVALID, "hb_geom_create_healpix: bad phi0_mode");
    if (weights_mode != HB_WEIGHTS_DZ && weights_mode != HB_WEIGHTS_UNIFORM)
        return fail(HB_ERR_INVALID, "hb_geom_create_healpix: bad weights_mode");
    const double pi = 3.141592653589793238462643383279502884;
    const int64_t nr = 4 * nside - 1, npix = 12 * nside * nside;
    HostGeom h;
    h.npix = npix;
    std::vector<double> theta(nr), x(nr), s(nr), ch(nr), sh(nr);
    for (int64_t i = 1; i <= nr; ++i) {
        int64_t r = i - 1;
        h.nphi.push_back(ring_nphi(nside, i));
        h.ofs.push_back(ring_first(nside, i));
        h.phi0_pi.push_back(ring_phi0(nside, i, phi0_mode == HB_PHI0_HEALPIX) / pi);
        double zz = ring_z(nside, i);
        double ehi = (i == 1) ? 1.0 : 0.5 * (ring_z(nside, i - 1) + zz);
        double elo = (i == nr) ? -1.0 : 0.5 * (zz + ring_z(nside, i + 1));
        h.w.push_back(weights_mode == HB_WEIGHTS_DZ ? ehi - elo : 2.0 * (double)ring_nphi(nside, i) / (double)npix);
        // accurate x, sin(theta), half angles: on the caps 1-|z| = ip^2/(3 nside^2) exactly
        int64_t ip = std::min<int64_t>(i, 4 * nside - i);
        long double t, zl;
        if (ip < nside) {
            t = (long double)(ip * ip) / (3.0L * (long double)(nside * nside));
            zl = (i < nside) ? 1.0L - t : -(1.0L - t);
        } else {
            zl = (long double)(2 * nside - i) * 2.0L / (3.0L * (long double)nside);
            t = 1.0L - fabsl(zl);
        }
        x[r] = (double)zl;
        s[r] = (double)sqrtl(t * (2.0L - t));
        theta[r] = (double)acosl(zl);
        ch[r] = (double)sqrtl((1.0L + zl) / 2.0L);
        sh[r] = (double)sqrtl((1.0L - zl) / 2.0L);
    }
    make_pairs(h, theta, x, s, ch, sh);
    return finish_geom(h, nside, x, s, ch, sh, out);
}

int hb_geom_create(int64_t nr, const double *theta, const int32_t *nphi, const double *phi0, const double *weights,
                   hb_geom **out) {
    if (!out || !theta || !nphi || !weights || nr <= 0)
        return fail(HB_ERR_INVALID, "hb_geom_create: null argument or nr <= 0");
    const double pi = 3.141592653589793238462643383279502884;
    HostGeom h;
    std::vector<double> th(nr), x(nr), s(nr), ch(nr), sh(nr);
    int64_t acc = 0;
    for (int64_t r = 0; r < nr; ++r) {
        if (nphi[r] <= 0 || (nphi[r] & 1) || nphi[r] > (1 << 16))
            return fail(HB_ERR_INVALID, "hb_geom_create: nphi must be even, positive and <= 65536");
        if (!(theta[r] > 0.0 && theta[r] < pi))
            return fail(HB_ERR_INVALID, "hb_geom_create: theta must lie strictly inside (0, pi)");
        h.nphi.push_back(nphi[r]);
        h.ofs.push_back(acc);
        acc += nphi[r];
        h.phi0_pi.push_back(phi0 ? phi0[r] / pi : 0.0);
        h.w.push_back(weights[r]);
        th[r] = theta[r];
        x[r] = std::cos(theta[r]);
        s[r] = std::sin(theta[r]);
        ch[r] = std::cos(0.5 * theta[r]);
        sh[r] = std::sin(0.5 * theta[r]);
    }
    h.npix = acc;
    make_pairs(h, th, x, s, ch, sh);
    return finish_geom(h, 0, x, s, ch, sh, out);
}

int hb_geom_destroy(hb_geom *g) {
    if (!g) return HB_OK;
    cudaFree(g->alloc_base);
    delete g;
    return HB_OK;
}

int hb_geom_info(const hb_geom *g, int64_t *nr, int64_t *npix, int64_t *npairs, int64_t *nside) {
    if (!g) return fail(HB_ERR_INVALID, "hb_geom_info: null geometry");
    if (nr) *nr = g->d.nr;
    if (npix) *npix = g->d.npix;
    if (npairs) *npairs = g->d.npairs;
    if (nside) *nside = g->nside;
    return HB_OK;
}

int hb_geom_fft_launches(const hb_geom *g, int precision, int *n) {
    if (!g || !n || (precision != 32 && precision != 64))
        return fail(HB_ERR_INVALID, "hb_geom_fft_launches: bad arguments");
    *n = precision == 32 ? g->d.pk_n_cls + g->d.rest_n_cls : g->d.n_cls;
    return HB_OK;
}

}  // extern "C"
