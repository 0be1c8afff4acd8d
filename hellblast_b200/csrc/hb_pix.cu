// HEALPix pixel indexing on the GPU: RING <-> NESTED index conversion, pixel centres, the pixel
// containing a direction, and map reordering between the two schemes.
//
// Replaces the reference's coordinate kernels and their drivers (coords_ring.cu:9-54 with
// coords_ring.py:18-54, nested_gpu.cu:27-95, nested_pix2ang.cu:16-85, order_convert.py:8-34).
// The HEALPix pixelisation (Gorski et al. 2005, ApJ 622, 759): 12 base faces, face f with corner
// ring jrll[f] nside and corner longitude index jpll[f]; NESTED index f nside^2 + (ix, iy)
// bit-interleaved (ix in the even bits); RING index counted ring by ring from the north pole.
// Index conversions go through (ix, iy, f) in integer arithmetic only (bit-exact); angles are
// FP64.  One thread per point, grid-stride loops over 148 x 16 CTAs at most; every kernel reads
// and writes each point once (HBM-bound: 16 bytes per index conversion).
//
// The reference's own conventions are available for parity (HB_PIX_REFERENCE):
//   * pix2ang RING: phi = phi0_r + j 2 pi / nphi_r with the reference's phi0 table
//     (ring_tables_healpix.cu:22-27, half a pixel off HEALPix on some rings) and its wrap
//     (coords_ring.cu:49-51);
//   * ang2pix RING: the ring whose z-edge interval holds cos(theta) (coords_ring.py:18-24), then
//     the nearest pixel centre in phi, llround((phi - phi0) / dphi) mod nphi (coords_ring.cu:21-28).
// The reference's NESTED ang2pix (nested_gpu.cu:27-95) is not the HEALPix map (it misnumbers the
// faces and uses a linear polar-cap coordinate): it has no compatibility mode here.
#include <cmath>

#include "hb_internal.cuh"

namespace hb {
namespace {

__constant__ int kJrll[12] = {2, 2, 2, 2, 3, 3, 3, 3, 4, 4, 4, 4};
__constant__ int kJpll[12] = {1, 3, 5, 7, 0, 2, 4, 6, 1, 3, 5, 7};

// bit i -> bit 2i for the low 32 bits, and its inverse
__device__ __forceinline__ uint64_t spread2(uint64_t x) {
    x &= 0xFFFFFFFFull;
    x = (x | (x << 16)) & 0x0000FFFF0000FFFFull;
    x = (x | (x << 8)) & 0x00FF00FF00FF00FFull;
    x = (x | (x << 4)) & 0x0F0F0F0F0F0F0F0Full;
    x = (x | (x << 2)) & 0x3333333333333333ull;
    x = (x | (x << 1)) & 0x5555555555555555ull;
    return x;
}
__device__ __forceinline__ uint64_t gather2(uint64_t x) {
    x &= 0x5555555555555555ull;
    x = (x | (x >> 1)) & 0x3333333333333333ull;
    x = (x | (x >> 2)) & 0x0F0F0F0F0F0F0F0Full;
    x = (x | (x >> 4)) & 0x00FF00FF00FF00FFull;
    x = (x | (x >> 8)) & 0x0000FFFF0000FFFFull;
    x = (x | (x >> 16)) & 0x00000000FFFFFFFFull;
    return x;
}

// floor(sqrt(v)) for v < 2^53, exact
__device__ __forceinline__ int64_t isqrt64(int64_t v) {
    int64_t r = (int64_t)sqrt((double)v);
    r -= (r * r > v) ? 1 : 0;
    r += ((r + 1) * (r + 1) <= v) ? 1 : 0;
    return r;
}

struct Xyf {
    int64_t ix, iy;
    int f;
};

__device__ __forceinline__ Xyf nest2xyf(int64_t nside, int log2n, int64_t p) {
    Xyf x;
    x.f = (int)(p >> (2 * log2n));
    const uint64_t q = (uint64_t)(p & ((int64_t(1) << (2 * log2n)) - 1));
    x.ix = (int64_t)gather2(q);
    x.iy = (int64_t)gather2(q >> 1);
    (void)nside;
    return x;
}
__device__ __forceinline__ int64_t xyf2nest(int log2n, const Xyf &x) {
    return ((int64_t)x.f << (2 * log2n)) + (int64_t)(spread2((uint64_t)x.ix) | (spread2((uint64_t)x.iy) << 1));
}

// ring number jr (1 .. 4 nside - 1), pixels before it, pixels in it / 4 and the half-pixel shift
struct RingInfo {
    int64_t nbefore, nr;
    int kshift;
};
__device__ __forceinline__ RingInfo ring_info(int64_t nside, int64_t jr) {
    const int64_t npix = 12 * nside * nside, ncap = 2 * nside * (nside - 1);
    RingInfo r;
    if (jr < nside) {
        r.nr = jr; r.nbefore = 2 * jr * (jr - 1); r.kshift = 0;
    } else if (jr > 3 * nside) {
        r.nr = 4 * nside - jr; r.nbefore = npix - 2 * (r.nr + 1) * r.nr; r.kshift = 0;
    } else {
        r.nr = nside; r.nbefore = ncap + (jr - nside) * 4 * nside; r.kshift = (int)((jr - nside) & 1);
    }
    return r;
}

__device__ __forceinline__ int64_t xyf2ring(int64_t nside, const Xyf &x) {
    const int64_t jr = (int64_t)kJrll[x.f] * nside - x.ix - x.iy - 1;
    const RingInfo ri = ring_info(nside, jr);
    int64_t jp = ((int64_t)kJpll[x.f] * ri.nr + x.ix - x.iy + 1 + ri.kshift) / 2;
    jp += (jp < 1) ? 4 * ri.nr : 0;
    jp -= (jp > 4 * ri.nr) ? 4 * ri.nr : 0;
    return ri.nbefore + jp - 1;
}

// RING pixel -> ring number (1 .. 4 nside - 1) and 1-based position in the ring
__device__ __forceinline__ void ring_pos(int64_t nside, int64_t p, int64_t &iring, int64_t &iphi) {
    const int64_t npix = 12 * nside * nside, ncap = 2 * nside * (nside - 1);
    if (p < ncap) {
        iring = (1 + isqrt64(1 + 2 * p)) >> 1;
        iphi = p + 1 - 2 * iring * (iring - 1);
    } else if (p < npix - ncap) {
        const int64_t ip = p - ncap, t = ip / (4 * nside);
        iring = t + nside;
        iphi = ip - t * 4 * nside + 1;
    } else {
        const int64_t ip = npix - p, ir = (1 + isqrt64(2 * ip - 1)) >> 1;
        iphi = 4 * ir + 1 - (ip - 2 * ir * (ir - 1));
        iring = 4 * nside - ir;
    }
}

__device__ __forceinline__ Xyf ring2xyf(int64_t nside, int64_t p) {
    int64_t iring, iphi;
    ring_pos(nside, p, iring, iphi);
    int64_t nr;
    int kshift, face;
    if (iring < nside) {
        nr = iring; kshift = 0;
        face = (int)((iphi - 1) / nr);
    } else if (iring <= 3 * nside) {
        nr = nside; kshift = (int)((iring + nside) & 1);
        const int64_t ire = iring - nside + 1, irm = 2 * nside + 2 - ire;
        const int64_t ifm = (iphi - ire / 2 + nside - 1) / nside, ifp = (iphi - irm / 2 + nside - 1) / nside;
        face = (ifp == ifm) ? (int)(ifp | 4) : ((ifp < ifm) ? (int)ifp : (int)(ifm + 8));
    } else {
        nr = 4 * nside - iring; kshift = 0;
        face = 8 + (int)((iphi - 1) / nr);
    }
    const int64_t irt = iring - (int64_t)kJrll[face] * nside + 1;
    int64_t ipt = 2 * iphi - (int64_t)kJpll[face] * nr - kshift - 1;
    ipt -= (ipt >= 2 * nside) ? 8 * nside : 0;
    Xyf x;
    x.ix = (ipt - irt) >> 1;
    x.iy = (-ipt - irt) >> 1;
    x.f = face;
    return x;
}

// centre of RING pixel p: z = cos theta and phi (HEALPix convention)
__device__ __forceinline__ void ring_center(int64_t nside, int64_t p, double &z, double &phi) {
    const double pi = 3.141592653589793238462643383279502884;
    int64_t iring, iphi;
    ring_pos(nside, p, iring, iphi);
    const double fact2 = 4.0 / (double)(12 * nside * nside);
    if (iring < nside) {
        z = 1.0 - (double)(iring * iring) * fact2;
        phi = ((double)iphi - 0.5) * (pi / (2.0 * (double)iring));
    } else if (iring <= 3 * nside) {
        const double fodd = ((iring + nside) & 1) ? 1.0 : 0.5;
        z = (double)(2 * nside - iring) * (2.0 / (3.0 * (double)nside));
        phi = ((double)iphi - fodd) * (pi / (2.0 * (double)nside));
    } else {
        const int64_t ir = 4 * nside - iring;
        z = -1.0 + (double)(ir * ir) * fact2;
        phi = ((double)iphi - 0.5) * (pi / (2.0 * (double)ir));
    }
}

// the pixel holding direction (z, phi): RING index, or (ix, iy, f)
__device__ __forceinline__ double turns4(double phi) {  // phi / (pi/2) reduced to [0, 4)
    const double twopi = 6.283185307179586476925286766559;
    double t = fmod(phi, twopi);
    t += (t < 0.0) ? twopi : 0.0;
    t *= 0.63661977236758134307553505349006;  // 2 / pi
    return t >= 4.0 ? 0.0 : t;
}
__device__ __forceinline__ int64_t zphi2ring(int64_t nside, double z, double phi) {
    const double za = fabs(z), tt = turns4(phi);
    const int64_t npix = 12 * nside * nside, ncap = 2 * nside * (nside - 1);
    if (za <= 2.0 / 3.0) {
        const double t1 = (double)nside * (0.5 + tt), t2 = (double)nside * z * 0.75;
        const int64_t jp = (int64_t)(t1 - t2), jm = (int64_t)(t1 + t2);
        const int64_t ir = nside + 1 + jp - jm, kshift = 1 - (ir & 1);
        int64_t ip = (jp + jm - nside + kshift + 1) / 2;
        ip %= 4 * nside;
        ip += (ip < 0) ? 4 * nside : 0;
        return ncap + (ir - 1) * 4 * nside + ip;
    }
    const double tp = tt - floor(tt), tmp = (double)nside * sqrt(3.0 * (1.0 - za));
    const int64_t jp = (int64_t)(tp * tmp), jm = (int64_t)((1.0 - tp) * tmp);
    const int64_t ir = jp + jm + 1;
    int64_t ip = (int64_t)(tt * (double)ir);
    ip %= 4 * ir;
    ip += (ip < 0) ? 4 * ir : 0;
    return (z > 0.0) ? 2 * ir * (ir - 1) + ip : npix - 2 * ir * (ir + 1) + ip;
}
__device__ __forceinline__ Xyf zphi2xyf(int64_t nside, double z, double phi) {
    const double za = fabs(z), tt = turns4(phi);
    Xyf x;
    if (za <= 2.0 / 3.0) {
        const double t1 = (double)nside * (0.5 + tt), t2 = (double)nside * z * 0.75;
        const int64_t jp = (int64_t)(t1 - t2), jm = (int64_t)(t1 + t2);
        const int64_t ifp = jp / nside, ifm = jm / nside;
        x.f = (ifp == ifm) ? (int)(ifp | 4) : ((ifp < ifm) ? (int)ifp : (int)(ifm + 8));
        x.ix = jm & (nside - 1);
        x.iy = nside - (jp & (nside - 1)) - 1;
    } else {
        int ntt = (int)tt;
        ntt = ntt >= 4 ? 3 : ntt;
        const double tp = tt - (double)ntt, tmp = (double)nside * sqrt(3.0 * (1.0 - za));
        int64_t jp = (int64_t)(tp * tmp), jm = (int64_t)((1.0 - tp) * tmp);
        jp = jp > nside - 1 ? nside - 1 : jp;
        jm = jm > nside - 1 ? nside - 1 : jm;
        if (z >= 0.0) {
            x.f = ntt; x.ix = nside - jm - 1; x.iy = nside - jp - 1;
        } else {
            x.f = ntt + 8; x.ix = jp; x.iy = jm;
        }
    }
    return x;
}

// ------------------------------------------------------------------------------ kernels
#define HB_GRID_STRIDE(i, n) for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

__global__ void ring2nest_kernel(int64_t nside, int log2n, int64_t n, const int64_t *__restrict__ in,
                                 int64_t *__restrict__ out, int *bad) {
    const int64_t npix = 12 * nside * nside;
    HB_GRID_STRIDE(i, n) {
        const int64_t p = in[i];
        if (p < 0 || p >= npix) { out[i] = -1; atomicOr(bad, 1); continue; }
        out[i] = xyf2nest(log2n, ring2xyf(nside, p));
    }
}
__global__ void nest2ring_kernel(int64_t nside, int log2n, int64_t n, const int64_t *__restrict__ in,
                                 int64_t *__restrict__ out, int *bad) {
    const int64_t npix = 12 * nside * nside;
    HB_GRID_STRIDE(i, n) {
        const int64_t p = in[i];
        if (p < 0 || p >= npix) { out[i] = -1; atomicOr(bad, 1); continue; }
        out[i] = xyf2ring(nside, nest2xyf(nside, log2n, p));
    }
}
// ref: the reference's RING convention (phi0 table of ring_tables_healpix.cu, coords_ring.cu:47-53)
__global__ void pix2ang_kernel(int64_t nside, int log2n, int nest, int ref, const double *__restrict__ phi0_ref,
                               int64_t n, const int64_t *__restrict__ pix, double *__restrict__ theta,
                               double *__restrict__ phi, int *bad) {
    const int64_t npix = 12 * nside * nside;
    const double twopi = 6.283185307179586476925286766559;
    HB_GRID_STRIDE(i, n) {
        int64_t p = pix[i];
        if (p < 0 || p >= npix) { theta[i] = phi[i] = nan(""); atomicOr(bad, 1); continue; }
        if (nest) p = xyf2ring(nside, nest2xyf(nside, log2n, p));
        double z, ph;
        ring_center(nside, p, z, ph);
        if (ref) {  // phi0_r + j dphi, wrapped as coords_ring.cu:50-51
            int64_t iring, iphi;
            ring_pos(nside, p, iring, iphi);
            const int64_t nphi = iring < nside ? 4 * iring : (iring <= 3 * nside ? 4 * nside : 4 * (4 * nside - iring));
            // separate rounded multiply and add (no FMA contraction), as the reference's host-side
            // arithmetic rounds them
            ph = __dadd_rn(phi0_ref[iring - 1], __dmul_rn((double)(iphi - 1), twopi / (double)nphi));
            if (ph >= twopi) ph = __dsub_rn(ph, __dmul_rn(twopi, floor(ph / twopi)));
        }
        theta[i] = acos(z);
        phi[i] = ph;
    }
}
__global__ void ang2pix_kernel(int64_t nside, int log2n, int nest, int64_t n, const double *__restrict__ theta,
                               const double *__restrict__ phi, int64_t *__restrict__ pix, int *bad) {
    const double pi = 3.141592653589793238462643383279502884;
    HB_GRID_STRIDE(i, n) {
        const double th = theta[i];
        if (!(th >= 0.0 && th <= pi) || !isfinite(phi[i])) { pix[i] = -1; atomicOr(bad, 1); continue; }
        const double z = cos(th);
        pix[i] = nest ? xyf2nest(log2n, zphi2xyf(nside, z, phi[i])) : zphi2ring(nside, z, phi[i]);
    }
}
// The reference's RING ang2pix (coords_ring.py:18-24, coords_ring.cu:19-28): ring r with
// z_edges[r] >= z > z_edges[r+1] (clamped to the rings), then llround(((phi - phi0_r) mod 2 pi)
// / dphi) mod nphi.  z_edges: the reference's midpoint table (nr + 1 entries, descending).
__global__ void ang2pix_ring_ref_kernel(int64_t nside, const double *__restrict__ z_edges,
                                        const double *__restrict__ phi0_ref, int64_t n,
                                        const double *__restrict__ theta, const double *__restrict__ phi,
                                        int64_t *__restrict__ pix, int *bad) {
    const double twopi = 6.283185307179586476925286766559;
    const int nr = (int)(4 * nside - 1);
    HB_GRID_STRIDE(i, n) {
        const double th = theta[i];
        if (!isfinite(th) || !isfinite(phi[i])) { pix[i] = -1; atomicOr(bad, 1); continue; }
        const double z = cos(th);
        // searchsorted(-z_edges, -z, side='right') - 1: the last r with -z_edges[r] <= -z
        int lo = 0, hi = nr + 1;  // count of edges e with -e <= -z
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (-z_edges[mid] <= -z) lo = mid + 1; else hi = mid;
        }
        int r = lo - 1;
        r = r < 0 ? 0 : (r > nr - 1 ? nr - 1 : r);
        const int64_t iring = r + 1;
        const int64_t nphi = iring < nside ? 4 * iring : (iring <= 3 * nside ? 4 * nside : 4 * (4 * nside - iring));
        const double dphi = twopi / (double)nphi;
        double d = fmod(phi[i] - phi0_ref[r], twopi);
        d += (d < 0.0) ? twopi : 0.0;
        int64_t j = llround(d / dphi);
        j -= (j >= nphi) ? nphi : 0;
        int64_t first;
        if (iring < nside) first = 2 * iring * (iring - 1);
        else if (iring <= 3 * nside) first = 2 * nside * (nside - 1) + (iring - nside) * 4 * nside;
        else { const int64_t ir = 4 * nside - iring; first = 12 * nside * nside - 2 * ir * (ir + 1); }
        pix[i] = first + j;
    }
}
// map reordering: out[perm(p)] = in[p] (RING -> NESTED with ring2nest, NESTED -> RING with
// nest2ring); each map read and written once
template <typename T>
__global__ void reorder_kernel(int64_t nside, int log2n, int to_nest, int nmaps, const T *__restrict__ in,
                               T *__restrict__ out) {
    const int64_t npix = 12 * nside * nside;
    HB_GRID_STRIDE(i, npix * nmaps) {
        const int64_t b = i / npix, p = i - b * npix;
        const int64_t q = to_nest ? xyf2nest(log2n, ring2xyf(nside, p)) : xyf2ring(nside, nest2xyf(nside, log2n, p));
        out[b * npix + q] = in[i];
    }
}

int pix_grid(int64_t n) {
    int64_t b = (n + 255) / 256;
    return (int)(b < 148 * 16 ? (b > 0 ? b : 1) : 148 * 16);
}

int check_nside(int64_t nside, const char *who, int *log2n) {
    if (nside < 1 || nside > (int64_t(1) << 29) || (nside & (nside - 1)))
        return fail(HB_ERR_INVALID, std::string(who) + ": nside must be a power of 2 in [1, 2^29]");
    int l = 0;
    while ((int64_t(1) << l) < nside) ++l;
    *log2n = l;
    return HB_OK;
}

}  // namespace
}  // namespace hb

using namespace hb;

extern "C" {

int hb_ring2nest(int64_t nside, int64_t n, const int64_t *ring, int64_t *nest, int *bad, hb_stream_t s) {
    int lg, rc = check_nside(nside, "hb_ring2nest", &lg);
    if (rc) return rc;
    if (n < 0 || (n > 0 && (!ring || !nest || !bad))) return fail(HB_ERR_INVALID, "hb_ring2nest: bad arguments");
    if (n == 0) return HB_OK;
    ring2nest_kernel<<<pix_grid(n), 256, 0, (cudaStream_t)s>>>(nside, lg, n, ring, nest, bad);
    HB_CHECK_LAUNCH();
    return HB_OK;
}

int hb_nest2ring(int64_t nside, int64_t n, const int64_t *nest, int64_t *ring, int *bad, hb_stream_t s) {
    int lg, rc = check_nside(nside, "hb_nest2ring", &lg);
    if (rc) return rc;
    if (n < 0 || (n > 0 && (!ring || !nest || !bad))) return fail(HB_ERR_INVALID, "hb_nest2ring: bad arguments");
    if (n == 0) return HB_OK;
    nest2ring_kernel<<<pix_grid(n), 256, 0, (cudaStream_t)s>>>(nside, lg, n, nest, ring, bad);
    HB_CHECK_LAUNCH();
    return HB_OK;
}

int hb_pix2ang(int64_t nside, int flags, const double *phi0_ref, int64_t n, const int64_t *pix, double *theta,
               double *phi, int *bad, hb_stream_t s) {
    int lg, rc = check_nside(nside, "hb_pix2ang", &lg);
    if (rc) return rc;
    const int nest = (flags & HB_PIX_NEST) ? 1 : 0, ref = (flags & HB_PIX_REFERENCE) ? 1 : 0;
    if (n < 0 || (n > 0 && (!pix || !theta || !phi || !bad)) || (ref && (nest || !phi0_ref)))
        return fail(HB_ERR_INVALID, "hb_pix2ang: bad arguments (HB_PIX_REFERENCE is RING only and needs phi0_ref)");
    if (n == 0) return HB_OK;
    pix2ang_kernel<<<pix_grid(n), 256, 0, (cudaStream_t)s>>>(nside, lg, nest, ref, phi0_ref, n, pix, theta, phi, bad);
    HB_CHECK_LAUNCH();
    return HB_OK;
}

int hb_ang2pix(int64_t nside, int flags, const double *z_edges, const double *phi0_ref, int64_t n,
               const double *theta, const double *phi, int64_t *pix, int *bad, hb_stream_t s) {
    int lg, rc = check_nside(nside, "hb_ang2pix", &lg);
    if (rc) return rc;
    const int nest = (flags & HB_PIX_NEST) ? 1 : 0, ref = (flags & HB_PIX_REFERENCE) ? 1 : 0;
    if (n < 0 || (n > 0 && (!pix || !theta || !phi || !bad)) || (ref && (nest || !phi0_ref || !z_edges)))
        return fail(HB_ERR_INVALID,
                    "hb_ang2pix: bad arguments (HB_PIX_REFERENCE is RING only and needs z_edges and phi0_ref)");
    if (n == 0) return HB_OK;
    if (ref)
        ang2pix_ring_ref_kernel<<<pix_grid(n), 256, 0, (cudaStream_t)s>>>(nside, z_edges, phi0_ref, n, theta, phi, pix,
                                                                          bad);
    else
        ang2pix_kernel<<<pix_grid(n), 256, 0, (cudaStream_t)s>>>(nside, lg, nest, n, theta, phi, pix, bad);
    HB_CHECK_LAUNCH();
    return HB_OK;
}

int hb_reorder(int64_t nside, int to_nest, int precision, int nmaps, const void *in, void *out, hb_stream_t s) {
    int lg, rc = check_nside(nside, "hb_reorder", &lg);
    if (rc) return rc;
    if (nmaps < 1 || !in || !out || in == out || (precision != 32 && precision != 64))
        return fail(HB_ERR_INVALID, "hb_reorder: bad arguments (out of place, precision 32 or 64)");
    const int64_t n = 12 * nside * nside * (int64_t)nmaps;
    if (precision == 32)
        reorder_kernel<float><<<pix_grid(n), 256, 0, (cudaStream_t)s>>>(nside, lg, to_nest ? 1 : 0, nmaps,
                                                                         (const float *)in, (float *)out);
    else
        reorder_kernel<double><<<pix_grid(n), 256, 0, (cudaStream_t)s>>>(nside, lg, to_nest ? 1 : 0, nmaps,
                                                                          (const double *)in, (double *)out);
    HB_CHECK_LAUNCH();
    return HB_OK;
}

}  // extern "C"
