// Wigner-d matrices and the rotation of alm by Euler angles (ZYZ), FP64.
//
// Replaces the reference's rotation path (rotate_alm_euler.py:5-14 with wigner_router.py,
// wigner_fast.py and wigner_d_fast.cu:8-52; wigner_full.py:12-96; wigner_delta.py:19-56), which
// builds each d^l_{mm'}(beta) from the closed-form alternating sum.  That sum is numerically
// unusable at large l (cancellation, exp overflow), and the reference's version of it raises
// cos(beta/2) and sin(beta/2) to powers other than the textbook ones (wigner_full.py:28-37), so
// its d^l is not a rotation matrix.  Here d^l_{mm'}(beta) (d^j_{m'm} of the usual convention
// with first index m) comes from the three-term recursion in l at fixed (m, m'),
//   l R_{l+1} d_{l+1} = (2l+1) (l(l+1) cos beta - m m') d_l - (l+1) R_l d_{l-1},
//   R_l = sqrt((l^2 - m^2)(l^2 - m'^2)),
// started at l0 = max(|m|, |m'|) from the closed form of the edge element, kept as a mantissa
// and a power-of-two exponent (steps of 2^256) while it is below FP64 range.
//
// Rotation (the reference's convention, rotate_alm_euler.py / wigner_full.py:79-96):
//   a'_{lm} = sum_{m'=-l..l} exp(-i m alpha) d^l_{mm'}(beta) exp(-i m' gamma) a_{lm'},
// a_{l,-m'} = (-1)^{m'} conj(a_{lm'}) for the real field; healpy m-major layout, m >= 0 stored.
// One CTA per output order m; its threads take input orders m', each running the recursion over
// l and adding its term to the CTA's shared accumulator row a'_{l m} (warp reduction, then one
// shared-memory atomic per warp and l).
#include <algorithm>
#include <cmath>

#include "hb_internal.cuh"

namespace hb {
namespace {

constexpr int ROT_NT = 256;
constexpr double TWO256 = 1.157920892373161954235709850086879078532699846656405640394575840079131296e77;  // 2^256

// d^{l0}_{m,m'}(beta), l0 = max(|m|, |m'|), for beta in [0, pi], as mantissa * 2^(256 e), from
//   d^j_{j,k} = sqrt((2j)! / ((j+k)! (j-k)!)) cos(b/2)^{j+k} (-sin(b/2))^{j-k}
// and d_{a,b} = (-1)^{a-b} d_{b,a} = d_{-b,-a}.  lc, ls: log2 cos(b/2), log2 sin(b/2) (-inf at the
// ends of the range, where the edge element is 0 or a power of 0).
__device__ __forceinline__ void d_edge(int m, int mp, double lc, double ls, double &mant, int &e) {
    int j, k, sh;
    if (abs(m) >= abs(mp)) {
        if (m >= 0) { j = m; k = mp; sh = 0; }                 // d_{l0,k}
        else { j = -m; k = -mp; sh = (mp + j) & 1; }           // d_{m,m'} = d_{-m',l0} = (-1)^{..} d_{l0,-m'}
    } else {
        if (mp > 0) { j = mp; k = m; sh = (m - j) & 1; }       // d_{m,l0} = (-1)^{m-l0} d_{l0,m}
        else { j = -mp; k = -m; sh = 0; }                      // d_{m,-l0} = d_{l0,-m}
    }
    const double l2e = 1.4426950408889634073599246810018921;  // log2 e
    double L2 = 0.5 * (lgamma(2.0 * j + 1.0) - lgamma((double)(j + k) + 1.0) - lgamma((double)(j - k) + 1.0)) * l2e;
    if (j + k > 0) L2 += (double)(j + k) * lc;
    if (j - k > 0) L2 += (double)(j - k) * ls;
    const int sign = (((j - k) & 1) ^ sh) ? -1 : 1;
    if (!(L2 > -1.0e300)) {  // -inf: an exact zero that the recursion keeps
        mant = 0.0;
        e = 0;
        return;
    }
    e = (int)floor((L2 + 128.0) / 256.0);
    mant = exp2(L2 - 256.0 * (double)e) * (double)sign;
}

// one step of the l-recursion at fixed (m, m'): (d0, d1) = (d_{l-1}, d_l) -> (d_l, d_{l+1}),
// keeping the scale exponent e (values with e < 0 are below 2^-128 of the FP64 range's middle)
__device__ __forceinline__ void d_step(int l, int m, int mp, double x, double &d0, double &d1, int &e) {
    double v;
    if (l == 0) {  // m = m' = 0: P_1 = x P_0
        v = x * d1;
    } else {
        const double dl = (double)l, m2 = (double)m * m, p2 = (double)mp * mp;
        const double R1 = sqrt(((dl + 1.0) * (dl + 1.0) - m2) * ((dl + 1.0) * (dl + 1.0) - p2));
        const double R0 = sqrt((dl * dl - m2) * (dl * dl - p2));
        v = ((2.0 * dl + 1.0) * (dl * (dl + 1.0) * x - (double)m * mp) * d1 - (dl + 1.0) * R0 * d0) / (dl * R1);
    }
    d0 = d1;
    d1 = v;
    if (e < 0 && fabs(d1) > 3.402823669209385e38) {  // 2^128: bring the scale up by 2^256
        d1 /= TWO256;
        d0 /= TWO256;
        ++e;
    }
}

// beta reduced to [0, pi]: d(beta) = d(-beta') (-1)^{m-m'} for beta = 2 pi - beta'
struct BetaRed {
    double x, lc, ls;
    bool flip;
};
__host__ __device__ __forceinline__ BetaRed beta_reduce(double beta) {
    const double twopi = 6.283185307179586476925286766559, pi = 3.141592653589793238462643383279502884;
    double b = fmod(beta, twopi);
    if (b < 0.0) b += twopi;
    BetaRed r;
    r.flip = b > pi;
    if (r.flip) b = twopi - b;
    r.x = cos(b);
    r.lc = log2(cos(0.5 * b));
    r.ls = log2(sin(0.5 * b));
    return r;
}

__global__ void __launch_bounds__(ROT_NT) wigner_d_kernel(int l, int nbeta, const double *__restrict__ beta,
                                                         double *__restrict__ out) {
    const int dim = 2 * l + 1;
    const int64_t total = (int64_t)nbeta * dim * dim;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int b = (int)(i / ((int64_t)dim * dim));
        const int r = (int)(i - (int64_t)b * dim * dim);
        const int m = r / dim - l, mp = r % dim - l;
        const BetaRed br = beta_reduce(beta[b]);
        double d0 = 0.0, d1;
        int e;
        d_edge(m, mp, br.lc, br.ls, d1, e);
        for (int ll = max(abs(m), abs(mp)); ll < l; ++ll) d_step(ll, m, mp, br.x, d0, d1, e);
        double v = e == 0 ? d1 : 0.0;
        if (br.flip && ((m - mp) & 1)) v = -v;
        out[i] = v;
    }
}

// a'_{lm} for one output order m per CTA (see the file comment)
__global__ void __launch_bounds__(ROT_NT) rotate_alm_kernel(int lmax, const double2 *__restrict__ ain,
                                                           double2 *__restrict__ aout, double alpha, double x,
                                                           double lc, double ls, int flip, double gamma) {
    extern __shared__ double2 acc[];  // [lmax + 1]
    const int m = blockIdx.x, b = blockIdx.y;
    const int64_t nalm = alm_idx(lmax, lmax, lmax) + 1;
    const double2 *a = ain + b * nalm;
    for (int l = threadIdx.x; l <= lmax; l += blockDim.x) acc[l] = make_double2(0.0, 0.0);
    __syncthreads();
    const int lane = threadIdx.x & 31;
    // input orders m' in [-lmax, lmax], one per thread per pass (every warp makes the same passes)
    for (int base = -lmax; base <= lmax; base += ROT_NT) {
        const int mp = base + (int)threadIdx.x;
        const bool act = mp <= lmax;
        const int amp = abs(mp);
        const int l0 = act ? max(m, amp) : lmax + 1;
        // exp(-i m' gamma); a_{l,-m'} = (-1)^{m'} conj a_{l m'}; the (-1)^{m-m'} of a reduced beta
        double gs, gc;
        sincos(-(double)mp * gamma, &gs, &gc);
        double sg = (mp < 0 && (amp & 1)) ? -1.0 : 1.0;
        if (flip && ((m - mp) & 1)) sg = -sg;
        int lw = l0;  // the warp walks l from its smallest l0; lanes before their own l0 add zero
        for (int o = 16; o > 0; o >>= 1) lw = min(lw, __shfl_xor_sync(0xffffffffu, lw, o));
        if (lw > lmax) continue;
        double d0 = 0.0, d1 = 0.0;
        int e = -1;
        if (act && l0 <= lmax) d_edge(m, mp, lc, ls, d1, e);
        for (int l = lw; l <= lmax; ++l) {
            if (act && l > l0) d_step(l - 1, m, mp, x, d0, d1, e);
            double tr = 0.0, ti = 0.0;
            if (act && l >= l0 && e == 0) {
                const double2 v = a[alm_idx(lmax, l, amp)];
                const double vi = mp < 0 ? -v.y : v.y;
                const double dv = sg * d1;
                tr = dv * (v.x * gc - vi * gs);
                ti = dv * (v.x * gs + vi * gc);
            }
            for (int o = 16; o > 0; o >>= 1) {
                tr += __shfl_xor_sync(0xffffffffu, tr, o);
                ti += __shfl_xor_sync(0xffffffffu, ti, o);
            }
            if (lane == 0 && (tr != 0.0 || ti != 0.0)) {
                atomicAdd(&acc[l].x, tr);
                atomicAdd(&acc[l].y, ti);
            }
        }
    }
    __syncthreads();
    double as, ac;
    sincos(-(double)m * alpha, &as, &ac);
    for (int l = m + (int)threadIdx.x; l <= lmax; l += blockDim.x) {
        const double2 v = acc[l];
        aout[b * nalm + alm_idx(lmax, l, m)] = make_double2(v.x * ac - v.y * as, v.x * as + v.y * ac);
    }
}

}  // namespace
}  // namespace hb

using namespace hb;

extern "C" {

int hb_wigner_d(int l, int nbeta, const double *beta, double *out, hb_stream_t s) {
    if (l < 0 || l > HB_MAX_L || nbeta < 0 || (nbeta > 0 && (!beta || !out)))
        return fail(HB_ERR_INVALID, "hb_wigner_d: bad arguments");
    if (nbeta == 0) return HB_OK;
    const int64_t total = (int64_t)nbeta * (2 * l + 1) * (2 * l + 1);
    const int blocks = (int)std::min<int64_t>((total + ROT_NT - 1) / ROT_NT, 148 * 16);
    wigner_d_kernel<<<blocks, ROT_NT, 0, (cudaStream_t)s>>>(l, nbeta, beta, out);
    HB_CHECK_LAUNCH();
    return HB_OK;
}

int hb_rotate_alm(int lmax, int nmaps, const void *alm_in, void *alm_out, double alpha, double beta, double gamma,
                  hb_stream_t s) {
    if (lmax < 0 || lmax > HB_MAX_L || nmaps < 1 || nmaps > 65535 || !alm_in || !alm_out || alm_in == alm_out)
        return fail(HB_ERR_INVALID, "hb_rotate_alm: bad arguments (lmax <= 16383, out of place)");
    const size_t smem = sizeof(double2) * (size_t)(lmax + 1);
    HB_CUDA_TRY(cudaFuncSetAttribute(rotate_alm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const BetaRed br = beta_reduce(beta);
    rotate_alm_kernel<<<dim3((unsigned)(lmax + 1), (unsigned)nmaps), ROT_NT, smem, (cudaStream_t)s>>>(
        lmax, (const double2 *)alm_in, (double2 *)alm_out, alpha, br.x, br.lc, br.ls, br.flip ? 1 : 0, gamma);
    HB_CHECK_LAUNCH();
    return HB_OK;
}

}  // extern "C"
