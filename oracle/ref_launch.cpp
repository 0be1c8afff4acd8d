/* Serial host "launcher" for the reference kernels compiled by build_ref.sh (test
 * infrastructure only).  Each entry point runs the kernel body once per emulated thread. */
#include <cstdint>
#include "ref_prelude.h"
hb_dim3 blockIdx{0, 0, 0}, threadIdx{0, 0, 0}, blockDim{1, 1, 1}, gridDim{1, 1, 1};

extern "C" void build_ring_tables(long long nside, double *z_centers, double *theta_centers, int *nphi,
                                  double *phi_center0, long long *ring_start, double *z_edges);
extern "C" void plm_recurrence(const double *x, int Ntheta, int lmax, int m, double *Plm);
extern "C" void wigner_d_ms_sum(const double *theta, int Ntheta, int lmax, int m, int s, double *out);

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
