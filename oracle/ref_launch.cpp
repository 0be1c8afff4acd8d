/* Serial host "launcher" for the reference kernels compiled by build_ref.sh (test
 * infrastructure only).  Each entry point runs the kernel body once per emulated thread. */
#include <cstdint>
#include "ref_prelude.h"
hb_dim3 blockIdx{0, 0, 0}, threadIdx{0, 0, 0}, blockDim{1, 1, 1}, gridDim{1, 1, 1};

extern "C" void build_ring_tables(long long nside, double *z_centers, double *theta_centers, int *nphi,
                                  double *phi_center0, long long *ring_start, double *z_edges);
extern "C" void plm_recurrence(const double *x, int Ntheta, int lmax, int m, double *Plm);
extern "C" void wigner_d_ms_sum(const double *theta, int Ntheta, int lmax, int m, int s, double *out);
extern "C" void ang2pix_ring_with_rings(const double *theta, const double *phi, const int *ring_idx, int N,
                                        const long long *ring_start, const int *nphi, const double *phi_center0,
                                        long long *out_ipix);
extern "C" void pix2ang_ring_batch(const long long *ipix, int N, const double *theta_centers,
                                   const long long *ring_start, const int *nphi, const double *phi_center0,
                                   double *out_theta, double *out_phi);
extern "C" void vec2pix_nest_batch(const double *theta, const double *phi, int N, int nside,
                                   unsigned long long *out_ipix);
extern "C" void pix2ang_nest_batch(const unsigned long long *ipnest, int N, int nside, double *out_theta,
                                   double *out_phi);

/* One emulated thread with a one-thread grid: it strides over every ring and then, as tid 0,
 * does the serial prefix sums (ring_tables_healpix.cu:14,40). */
extern "C" void ref_build_ring_tables(long long nside, double *z, double *theta, int *nphi, double *phi0,
                                      long long *ring_start, double *z_edges) {
    blockIdx = {0, 0, 0}; threadIdx = {0, 0, 0}; blockDim = {1, 1, 1}; gridDim = {1, 1, 1};
    build_ring_tables(nside, z, theta, nphi, phi0, ring_start, z_edges);
}

/* One emulated thread per theta (legendre.cu:9-10). */
extern "C" void ref_plm_recurrence(const double *x, int Ntheta, int lmax, int m, double *Plm) {
    blockDim = {1, 1, 1}; gridDim = {Ntheta, 1, 1}; threadIdx = {0, 0, 0};
    for (long long b = 0; b < Ntheta; ++b) {
        blockIdx = {b, 0, 0};
        plm_recurrence(x, Ntheta, lmax, m, Plm);
    }
}

/* One emulated thread per theta (wigner_d_ms.cu:25-26). */
extern "C" void ref_wigner_d_ms_sum(const double *theta, int Ntheta, int lmax, int m, int s, double *out) {
    blockDim = {1, 1, 1}; gridDim = {Ntheta, 1, 1}; threadIdx = {0, 0, 0};
    for (long long b = 0; b < Ntheta; ++b) {
        blockIdx = {b, 0, 0};
        wigner_d_ms_sum(theta, Ntheta, lmax, m, s, out);
    }
}

/* One emulated thread per point (coords_ring.cu:19-20,40-41, nested_gpu.cu:34-35). */
extern "C" void ref_ang2pix_ring_with_rings(const double *theta, const double *phi, const int *ring_idx, int N,
                                            const long long *ring_start, const int *nphi, const double *phi0,
                                            long long *out) {
    blockDim = {1, 1, 1}; gridDim = {N, 1, 1}; threadIdx = {0, 0, 0};
    for (long long b = 0; b < N; ++b) {
        blockIdx = {b, 0, 0};
        ang2pix_ring_with_rings(theta, phi, ring_idx, N, ring_start, nphi, phi0, out);
    }
}
extern "C" void ref_pix2ang_ring_batch(const long long *ipix, int N, const double *theta_c, const long long *ring_start,
                                       const int *nphi, const double *phi0, double *th, double *ph) {
    blockDim = {1, 1, 1}; gridDim = {N, 1, 1}; threadIdx = {0, 0, 0};
    for (long long b = 0; b < N; ++b) {
        blockIdx = {b, 0, 0};
        pix2ang_ring_batch(ipix, N, theta_c, ring_start, nphi, phi0, th, ph);
    }
}
extern "C" void ref_vec2pix_nest_batch(const double *theta, const double *phi, int N, int nside,
                                       unsigned long long *out) {
    blockDim = {1, 1, 1}; gridDim = {N, 1, 1}; threadIdx = {0, 0, 0};
    for (long long b = 0; b < N; ++b) {
        blockIdx = {b, 0, 0};
        vec2pix_nest_batch(theta, phi, N, nside, out);
    }
}
/* pix2ang_nest_batch fills its face tables with threads 0..11 before a barrier
 * (nested_pix2ang.cu:24-32): emulated as a 12-thread block per point group. */
extern "C" void ref_pix2ang_nest_batch(const unsigned long long *ipnest, int N, int nside, double *th, double *ph) {
    /* threads 0..11 of a block past the end: they fill the face tables and return */
    blockDim = {12, 1, 1}; gridDim = {N, 1, 1};
    blockIdx = {N, 0, 0};
    for (long long t = 0; t < 12; ++t) {
        threadIdx = {t, 0, 0};
        pix2ang_nest_batch(ipnest, N, nside, th, ph);
    }
    blockDim = {1, 1, 1}; threadIdx = {0, 0, 0};
    for (long long b = 0; b < N; ++b) {
        blockIdx = {b, 0, 0};
        pix2ang_nest_batch(ipnest, N, nside, th, ph);
    }
}
