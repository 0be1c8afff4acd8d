/*
 * FP64 CPU oracle for the HEALPix spherical-harmonic transform hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the arbiter that the CUDA kernels in
 * hellblast_b200/csrc are checked against.  Only tests/, __graft_entry__.smoke()
 * and bench.py's cpu_baseline leg may load it; the product path never does.
 *
 * It restates, in plain C with OpenMP, the algorithm of the reference's SHT path:
 *   - ring geometry            ring_tables_healpix.cu:14-51, ring_tables.py:39-40
 *   - Legendre functions       legendre.cu:2-35 times sht_raw.py:26-28 (normalised
 *                              lambda_lm with the Condon-Shortley phase), computed here by
 *                              the overflow-free normalised three-term recursion with a
 *                              log-scaled sectoral start (Gorski et al. 2005, ApJ 622, 759;
 *                              Reinecke & Seljebotn 2013, A&A 554, A112)
 *   - analysis contraction     sht_raw.py:46-56 / sht_fallback.py:59-64
 *                              a_lm = sum_r lambda_lm(x_r) F_r(m)
 *   - synthesis                isht.py:15-25   G_r(m) = sum_l a_lm lambda_lm(x_r)
 *   - spin-2 (E/B)             spin.py:32-115 with one consistent convention:
 *                              _sY_lm = sqrt((2l+1)/4pi) d^l_{m,-s}(theta) e^{i m phi},
 *                              E = -(a2 + a-2)/2, B = i (a2 - a-2)/2, a(+-2) = -(E +- iB)
 *   - alm2cl                   alm_ops.py:19-32
 * The per-ring FFT with the phi0 phase and the m-aliasing fold lives in the Python half
 * of the oracle (oracle/sht_oracle.py), which uses numpy's pocketfft.
 *
 * alm layout: healpy m-major, idx(l,m) = m*(2*lmax+1-m)/2 + l, complex interleaved.
 * F / G layout: [m][ring] complex interleaved.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_SCALE 256          /* exponent step of the running scale */
#define ORC_HUGE 0x1p128       /* rescale while |lambda| > ORC_HUGE and the scale is negative */

static inline int64_t alm_idx(int64_t lmax, int64_t l, int64_t m) {
    return m * (2 * lmax + 1 - m) / 2 + l;
}

/* ------------------------------------------------------------------ ring tables */
/* Follows ring_tables_healpix.cu:14-51 (same double expressions for z, the same integer
 * nphi and ring_start), with phi0 either the reference's formula (healpix_phi0 == 0,
 * ring_tables_healpix.cu:21,27,34) or the HEALPix convention (healpix_phi0 != 0). */
void orc_ring_tables(int64_t nside, int healpix_phi0, double *z, double *theta, int32_t *nphi,
                     double *phi0, int64_t *ring_start, double *z_edges) {
    const double pi = 3.141592653589793238462643383279502884;
    int64_t nr = 4 * nside - 1;
    for (int64_t i = 1; i <= nr; ++i) {
        double zz, dphi, p0;
        int npr;
        if (i < nside) {
            zz = 1.0 - (double)(i * i) / (3.0 * (double)(nside * nside));
            npr = 4 * (int)i;
            dphi = 2.0 * pi / (double)npr;
            p0 = 0.5 * dphi;
        } else if (i <= 3 * nside) {
            zz = (double)(2 * nside - i) * (2.0 / (3.0 * (double)nside));
            npr = 4 * (int)nside;
            dphi = 2.0 * pi / (double)npr;
            int s = (int)((i - nside) & 1);
            if (healpix_phi0)
                p0 = s ? 0.0 : 0.5 * dphi;
            else
                p0 = (1.0 - 0.5 * (double)s) * dphi;
        } else {
            int64_t ip = 4 * nside - i;
            zz = -(1.0 - (double)(ip * ip) / (3.0 * (double)(nside * nside)));
            npr = 4 * (int)ip;
            dphi = 2.0 * pi / (double)npr;
            p0 = 0.5 * dphi;
        }
        z[i - 1] = zz;
        theta[i - 1] = acos(fmax(-1.0, fmin(1.0, zz)));
        nphi[i - 1] = npr;
        phi0[i - 1] = p0;
    }
    ring_start[0] = 0;
    for (int64_t i = 0; i < nr; ++i) ring_start[i + 1] = ring_start[i] + (int64_t)nphi[i];
    z_edges[0] = 1.0;
    for (int64_t i = 0; i < nr - 1; ++i) z_edges[i + 1] = 0.5 * (z[i] + z[i + 1]);
    z_edges[nr] = -1.0;
}

/* ------------------------------------------------------------------ scalar lambda_lm */
/* log2 of sqrt((2m+1)!! / ((2m)!! 4 pi)) for m = 0..mmax */
static void log2_sectoral_norm(int mmax, long double *out) {
    long double acc = 0.5L * log2l(1.0L / (4.0L * 3.141592653589793238462643383279502884L));
    out[0] = acc;
    for (int m = 1; m <= mmax; ++m) {
        acc += 0.5L * log2l((long double)(2 * m + 1) / (long double)(2 * m));
        out[m] = acc;
    }
}

/* Recursion coefficients for fixed m: lambda_l = A_l x lambda_{l-1} + B_l lambda_{l-2}. */
static void scalar_coefs(int lmax, int m, double *A, double *B) {
    for (int l = m + 1; l <= lmax; ++l) {
        long double ll = l, mm = m;
        long double a = sqrtl((4.0L * ll * ll - 1.0L) / (ll * ll - mm * mm));
        long double b = (l - 1 > m) ? sqrtl(((ll - 1) * (ll - 1) - mm * mm) / (4.0L * (ll - 1) * (ll - 1) - 1.0L)) : 0.0L;
        A[l] = (double)a;
        B[l] = (double)(-a * b);
    }
}

/* lambda_lm(x) for l = m..lmax at one point; out[l] (entries l < m untouched). */
static void scalar_lambda_point(int lmax, int m, double x, long double log2_sin, long double log2_cm,
                                const double *A, const double *B, double *out) {
    long double L = log2_cm + (long double)m * log2_sin;
    int e = (int)floorl((L + 128.0L) / (long double)ORC_SCALE);
    double l1 = (double)exp2l(L - (long double)ORC_SCALE * e);
    if (m & 1) l1 = -l1;
    double l2 = 0.0;
    out[m] = (e == 0) ? l1 : (e > 0 ? ldexp(l1, ORC_SCALE * e) : 0.0);
    for (int l = m + 1; l <= lmax; ++l) {
        double v = A[l] * x * l1 + B[l] * l2;
        l2 = l1;
        l1 = v;
        if (e < 0 && fabs(l1) > ORC_HUGE) {
            l1 = ldexp(l1, -ORC_SCALE);
            l2 = ldexp(l2, -ORC_SCALE);
            ++e;
        }
        out[l] = (e == 0) ? l1 : 0.0;
    }
}

/* Public: normalised lambda_lm(x_i) for l=m..lmax at n points -> out[i*(lmax+1)+l]. */
void orc_lambda_lm(int lmax, int m, int64_t n, const double *x, const double *sin_theta, double *out) {
    long double *lc = (long double *)malloc(sizeof(long double) * (size_t)(m + 1));
    double *A = (double *)calloc((size_t)lmax + 2, sizeof(double));
    double *B = (double *)calloc((size_t)lmax + 2, sizeof(double));
    log2_sectoral_norm(m, lc);
    scalar_coefs(lmax, m, A, B);
    for (int64_t i = 0; i < n; ++i) {
        double *o = out + i * (lmax + 1);
        for (int l = 0; l < m; ++l) o[l] = 0.0;
        scalar_lambda_point(lmax, m, x[i], log2l((long double)sin_theta[i]), lc[m], A, B, o);
    }
    free(lc); free(A); free(B);
}

/* Analysis: alm[idx(l,m)] = sum_r lambda_lm(x_r) * F[m][r]  (complex, healpy layout). */
void orc_legendre_analysis(int lmax, int mmax, int64_t nr, const double *x, const double *sin_theta,
                           const double *F, double *alm) {
    long double *lc = (long double *)malloc(sizeof(long double) * (size_t)(mmax + 1));
    log2_sectoral_norm(mmax, lc);
    long double *ls = (long double *)malloc(sizeof(long double) * (size_t)nr);
    for (int64_t r = 0; r < nr; ++r) ls[r] = log2l((long double)sin_theta[r]);
#pragma omp parallel
    {
        double *A = (double *)calloc((size_t)lmax + 2, sizeof(double));
        double *B = (double *)calloc((size_t)lmax + 2, sizeof(double));
        double *lam = (double *)malloc(sizeof(double) * ((size_t)lmax + 1));
        double *acc = (double *)malloc(sizeof(double) * 2 * ((size_t)lmax + 1));
#pragma omp for schedule(dynamic, 1)
        for (int m = 0; m <= mmax; ++m) {
            scalar_coefs(lmax, m, A, B);
            memset(acc, 0, sizeof(double) * 2 * ((size_t)lmax + 1));
            for (int64_t r = 0; r < nr; ++r) {
                const double fr = F[2 * ((int64_t)m * nr + r)], fi = F[2 * ((int64_t)m * nr + r) + 1];
                scalar_lambda_point(lmax, m, x[r], ls[r], lc[m], A, B, lam);
                for (int l = m; l <= lmax; ++l) {
                    acc[2 * l] += lam[l] * fr;
                    acc[2 * l + 1] += lam[l] * fi;
                }
            }
            for (int l = m; l <= lmax; ++l) {
                int64_t k = alm_idx(lmax, l, m);
                alm[2 * k] = acc[2 * l];
                alm[2 * k + 1] = acc[2 * l + 1];
            }
        }
        free(A); free(B); free(lam); free(acc);
    }
    free(lc); free(ls);
}

/* Synthesis: G[m][r] = sum_l a_lm lambda_lm(x_r). */
void orc_legendre_synthesis(int lmax, int mmax, int64_t nr, const double *x, const double *sin_theta,
                            const double *alm, double *G) {
    long double *lc = (long double *)malloc(sizeof(long double) * (size_t)(mmax + 1));
    log2_sectoral_norm(mmax, lc);
    long double *ls = (long double *)malloc(sizeof(long double) * (size_t)nr);
    for (int64_t r = 0; r < nr; ++r) ls[r] = log2l((long double)sin_theta[r]);
#pragma omp parallel
    {
        double *A = (double *)calloc((size_t)lmax + 2, sizeof(double));
        double *B = (double *)calloc((size_t)lmax + 2, sizeof(double));
        double *lam = (double *)malloc(sizeof(double) * ((size_t)lmax + 1));
#pragma omp for schedule(dynamic, 1)
        for (int m = 0; m <= mmax; ++m) {
            scalar_coefs(lmax, m, A, B);
            for (int64_t r = 0; r < nr; ++r) {
                scalar_lambda_point(lmax, m, x[r], ls[r], lc[m], A, B, lam);
                double gr = 0.0, gi = 0.0;
                for (int l = m; l <= lmax; ++l) {
                    int64_t k = alm_idx(lmax, l, m);
                    gr += lam[l] * alm[2 * k];
                    gi += lam[l] * alm[2 * k + 1];
                }
                G[2 * ((int64_t)m * nr + r)] = gr;
                G[2 * ((int64_t)m * nr + r) + 1] = gi;
            }
        }
        free(A); free(B); free(lam);
    }
    free(lc); free(ls);
}

/* Analysis restricted to the nms orders ms[j]: F [j][r] complex -> out [j][l] complex (l < ms[j]
 * zero), for spot checks of transforms too large to run in full here. */
void orc_legendre_analysis_ms(int lmax, int nms, const int *ms, int64_t nr, const double *x,
                              const double *sin_theta, const double *F, double *out) {
    int mx = 0;
    for (int j = 0; j < nms; ++j) mx = ms[j] > mx ? ms[j] : mx;
    long double *lc = (long double *)malloc(sizeof(long double) * (size_t)(mx + 1));
    log2_sectoral_norm(mx, lc);
    long double *ls = (long double *)malloc(sizeof(long double) * (size_t)nr);
    for (int64_t r = 0; r < nr; ++r) ls[r] = log2l((long double)sin_theta[r]);
    memset(out, 0, sizeof(double) * 2 * (size_t)nms * ((size_t)lmax + 1));
#pragma omp parallel
    {
        double *A = (double *)calloc((size_t)lmax + 2, sizeof(double));
        double *B = (double *)calloc((size_t)lmax + 2, sizeof(double));
        double *lam = (double *)malloc(sizeof(double) * ((size_t)lmax + 1));
#pragma omp for schedule(dynamic, 1)
        for (int j = 0; j < nms; ++j) {
            const int m = ms[j];
            double *acc = out + 2 * (size_t)j * ((size_t)lmax + 1);
            scalar_coefs(lmax, m, A, B);
            for (int64_t r = 0; r < nr; ++r) {
                const double fr = F[2 * ((int64_t)j * nr + r)], fi = F[2 * ((int64_t)j * nr + r) + 1];
                scalar_lambda_point(lmax, m, x[r], ls[r], lc[m], A, B, lam);
                for (int l = m; l <= lmax; ++l) {
                    acc[2 * l] += lam[l] * fr;
                    acc[2 * l + 1] += lam[l] * fi;
                }
            }
        }
        free(A); free(B); free(lam);
    }
    free(lc); free(ls);
}

/* Synthesis restricted to the nms orders ms[j]: a [j][l] complex -> G [j][r] complex. */
void orc_legendre_synthesis_ms(int lmax, int nms, const int *ms, int64_t nr, const double *x,
                               const double *sin_theta, const double *a, double *G) {
    int mx = 0;
    for (int j = 0; j < nms; ++j) mx = ms[j] > mx ? ms[j] : mx;
    long double *lc = (long double *)malloc(sizeof(long double) * (size_t)(mx + 1));
    log2_sectoral_norm(mx, lc);
    long double *ls = (long double *)malloc(sizeof(long double) * (size_t)nr);
    for (int64_t r = 0; r < nr; ++r) ls[r] = log2l((long double)sin_theta[r]);
#pragma omp parallel
    {
        double *A = (double *)calloc((size_t)lmax + 2, sizeof(double));
        double *B = (double *)calloc((size_t)lmax + 2, sizeof(double));
        double *lam = (double *)malloc(sizeof(double) * ((size_t)lmax + 1));
#pragma omp for schedule(dynamic, 1)
        for (int j = 0; j < nms; ++j) {
            const int m = ms[j];
            const double *aj = a + 2 * (size_t)j * ((size_t)lmax + 1);
            scalar_coefs(lmax, m, A, B);
            for (int64_t r = 0; r < nr; ++r) {
                scalar_lambda_point(lmax, m, x[r], ls[r], lc[m], A, B, lam);
                double gr = 0.0, gi = 0.0;
                for (int l = m; l <= lmax; ++l) {
                    gr += lam[l] * aj[2 * l];
                    gi += lam[l] * aj[2 * l + 1];
                }
                G[2 * ((int64_t)j * nr + r)] = gr;
                G[2 * ((int64_t)j * nr + r) + 1] = gi;
            }
        }
        free(A); free(B); free(lam);
    }
    free(lc); free(ls);
}

/* ------------------------------------------------------------------ spin-2 */
/* Normalised spin functions N_l d^l_{m,s}(theta), N_l = sqrt((2l+1)/4pi), for l = l0..lmax,
 * l0 = max(m, 2), s = +2 or -2, by the three-term Wigner-d recursion in l
 *   l R_{l+1} d_{l+1} = (2l+1)(l(l+1) x - m s) d_l - (l+1) R_l d_{l-1},
 *   R_l = sqrt((l^2-m^2)(l^2-s^2)),
 * started from the closed-form d^{l0}_{m,s} (log-scaled). */
static void spin_coefs(int lmax, int m, int s, double *a, double *b, double *c) {
    const long double fpi = 4.0L * 3.141592653589793238462643383279502884L;
    int l0 = m > 2 ? m : 2;
    for (int l = l0; l < lmax; ++l) {
        long double ll = l, mm = m, ss = s;
        long double R1 = sqrtl(((ll + 1) * (ll + 1) - mm * mm) * ((ll + 1) * (ll + 1) - ss * ss));
        long double R0 = sqrtl((ll * ll - mm * mm) * (ll * ll - ss * ss));
        long double N1 = sqrtl((2 * ll + 3) / fpi), N0 = sqrtl((2 * ll + 1) / fpi), Nm = sqrtl((2 * ll - 1) / fpi);
        a[l] = (double)((N1 / N0) * (2 * ll + 1) * (ll + 1) / R1);
        b[l] = (double)((N1 / N0) * (2 * ll + 1) * mm * ss / (ll * R1));
        c[l] = (double)((N1 / Nm) * (ll + 1) * R0 / (ll * R1));
    }
}

static long double lfac2(int n) { return lgammal((long double)n + 1.0L) / logl(2.0L); }

/* log2 |N_l0 d^{l0}_{m,s}(theta)| and its sign, from log2 cos(theta/2) and log2 sin(theta/2). */
static void spin_start(int m, int s, long double lc, long double lsn, long double *log2v, int *sign) {
    const long double fpi = 4.0L * 3.141592653589793238462643383279502884L;
    if (m >= 2) {
        /* d^m_{m,s} = sqrt((2m)!/((m+s)!(m-s)!)) cos^{m+s} (-sin)^{m-s} */
        *log2v = 0.5L * (lfac2(2 * m) - lfac2(m + s) - lfac2(m - s)) + (m + s) * lc + (m - s) * lsn
                 + 0.5L * log2l((2 * m + 1) / fpi);
        *sign = ((m - s) & 1) ? -1 : 1;
    } else if (s == 2) {
        /* d^2_{m,2} = sqrt(24/((2+m)!(2-m)!)) cos^{2+m} sin^{2-m} */
        *log2v = 0.5L * (lfac2(4) - lfac2(2 + m) - lfac2(2 - m)) + (2 + m) * lc + (2 - m) * lsn
                 + 0.5L * log2l(5.0L / fpi);
        *sign = 1;
    } else {
        /* d^2_{m,-2} = (-1)^m sqrt(24/((2-m)!(2+m)!)) cos^{2-m} sin^{2+m} */
        *log2v = 0.5L * (lfac2(4) - lfac2(2 + m) - lfac2(2 - m)) + (2 - m) * lc + (2 + m) * lsn
                 + 0.5L * log2l(5.0L / fpi);
        *sign = (m & 1) ? -1 : 1;
    }
}

static void spin_lambda_point(int lmax, int m, int s, double x, long double lc, long double lsn,
                              const double *a, const double *b, const double *c, double *out) {
    int l0 = m > 2 ? m : 2;
    long double L;
    int sg;
    spin_start(m, s, lc, lsn, &L, &sg);
    int e = (int)floorl((L + 128.0L) / (long double)ORC_SCALE);
    double l1 = (double)exp2l(L - (long double)ORC_SCALE * e) * sg, l2 = 0.0;
    out[l0] = (e == 0) ? l1 : (e > 0 ? ldexp(l1, ORC_SCALE * e) : 0.0);
    for (int l = l0; l < lmax; ++l) {
        double v = (a[l] * x - b[l]) * l1 - c[l] * l2;
        l2 = l1;
        l1 = v;
        if (e < 0 && fabs(l1) > ORC_HUGE) {
            l1 = ldexp(l1, -ORC_SCALE);
            l2 = ldexp(l2, -ORC_SCALE);
            ++e;
        }
        out[l + 1] = (e == 0) ? l1 : 0.0;
    }
}

/* Public: spin-weighted lambda.  out_p2[i*(lmax+1)+l] = _{+2}lambda_lm(theta_i) = N_l d^l_{m,-2},
 * out_m2[...] = _{-2}lambda_lm = N_l d^l_{m,+2}; entries l < max(m,2) are zero. */
void orc_spin2_lambda(int lmax, int m, int64_t n, const double *x, const double *theta, double *out_p2,
                      double *out_m2) {
    double *a = (double *)calloc((size_t)lmax + 2, sizeof(double));
    double *b = (double *)calloc((size_t)lmax + 2, sizeof(double));
    double *c = (double *)calloc((size_t)lmax + 2, sizeof(double));
    double *a2 = (double *)calloc((size_t)lmax + 2, sizeof(double));
    double *b2 = (double *)calloc((size_t)lmax + 2, sizeof(double));
    double *c2 = (double *)calloc((size_t)lmax + 2, sizeof(double));
    spin_coefs(lmax, m, -2, a, b, c);
    spin_coefs(lmax, m, 2, a2, b2, c2);
    for (int64_t i = 0; i < n; ++i) {
        double *op = out_p2 + i * (lmax + 1), *om = out_m2 + i * (lmax + 1);
        for (int l = 0; l <= lmax; ++l) op[l] = om[l] = 0.0;
        long double th = theta[i];
        long double lc = log2l(cosl(0.5L * th)), lsn = log2l(sinl(0.5L * th));
        if (m <= lmax && lmax >= 2) {
            spin_lambda_point(lmax, m, -2, x[i], lc, lsn, a, b, c, op);
            spin_lambda_point(lmax, m, 2, x[i], lc, lsn, a2, b2, c2, om);
        }
    }
    free(a); free(b); free(c); free(a2); free(b2); free(c2);
}

/* Spin-2 analysis.  Qf, Uf: [m][r] weighted Fourier coefficients of Q and U.
 * E_lm = -sum_r (lp Q + i lm U),  B_lm = -sum_r (lp U - i lm Q),
 * lp = (_2lambda + _-2lambda)/2, lm = (_2lambda - _-2lambda)/2.  E, B zero for l < 2. */
void orc_spin2_analysis(int lmax, int mmax, int64_t nr, const double *x, const double *theta,
                        const double *Qf, const double *Uf, double *E, double *B) {
    int64_t nalm = alm_idx(lmax, lmax, mmax) + 1;
    memset(E, 0, sizeof(double) * 2 * nalm);
    memset(B, 0, sizeof(double) * 2 * nalm);
    if (lmax < 2) return;
#pragma omp parallel
    {
        double *a = (double *)calloc((size_t)lmax + 2, sizeof(double)), *b = (double *)calloc((size_t)lmax + 2, sizeof(double)),
               *c = (double *)calloc((size_t)lmax + 2, sizeof(double)), *a2 = (double *)calloc((size_t)lmax + 2, sizeof(double)),
               *b2 = (double *)calloc((size_t)lmax + 2, sizeof(double)), *c2 = (double *)calloc((size_t)lmax + 2, sizeof(double));
        double *lp2 = (double *)calloc((size_t)lmax + 1, sizeof(double)), *lm2 = (double *)calloc((size_t)lmax + 1, sizeof(double));
        double *acc = (double *)malloc(sizeof(double) * 4 * ((size_t)lmax + 1));
#pragma omp for schedule(dynamic, 1)
        for (int m = 0; m <= mmax; ++m) {
            int l0 = m > 2 ? m : 2;
            spin_coefs(lmax, m, -2, a, b, c);
            spin_coefs(lmax, m, 2, a2, b2, c2);
            memset(acc, 0, sizeof(double) * 4 * ((size_t)lmax + 1));
            for (int64_t r = 0; r < nr; ++r) {
                long double th = theta[r];
                long double lc = log2l(cosl(0.5L * th)), lsn = log2l(sinl(0.5L * th));
                spin_lambda_point(lmax, m, -2, x[r], lc, lsn, a, b, c, lp2);
                spin_lambda_point(lmax, m, 2, x[r], lc, lsn, a2, b2, c2, lm2);
                const double qr = Qf[2 * ((int64_t)m * nr + r)], qi = Qf[2 * ((int64_t)m * nr + r) + 1];
                const double ur = Uf[2 * ((int64_t)m * nr + r)], ui = Uf[2 * ((int64_t)m * nr + r) + 1];
                for (int l = l0; l <= lmax; ++l) {
                    double lp = 0.5 * (lp2[l] + lm2[l]), lm = 0.5 * (lp2[l] - lm2[l]);
                    /* E = -(lp Q + i lm U) */
                    acc[4 * l + 0] -= lp * qr - lm * ui;
                    acc[4 * l + 1] -= lp * qi + lm * ur;
                    /* B = -(lp U - i lm Q) */
                    acc[4 * l + 2] -= lp * ur + lm * qi;
                    acc[4 * l + 3] -= lp * ui - lm * qr;
                }
            }
            for (int l = l0; l <= lmax; ++l) {
                int64_t k = alm_idx(lmax, l, m);
                E[2 * k] = acc[4 * l]; E[2 * k + 1] = acc[4 * l + 1];
                B[2 * k] = acc[4 * l + 2]; B[2 * k + 1] = acc[4 * l + 3];
            }
        }
        free(a); free(b); free(c); free(a2); free(b2); free(c2); free(lp2); free(lm2); free(acc);
    }
}

/* Spin-2 analysis restricted to the nms harmonic orders ms[j]: Qf, Uf [j][r] weighted Fourier
 * coefficients of those m; E, B [j][lmax + 1] complex (zero below max(m, 2)).  Same sums as
 * orc_spin2_analysis, for spot checks of transforms too large to run in full here. */
void orc_spin2_analysis_ms(int lmax, int nms, const int *ms, int64_t nr, const double *x, const double *theta,
                           const double *Qf, const double *Uf, double *E, double *B) {
    memset(E, 0, sizeof(double) * 2 * (size_t)nms * (lmax + 1));
    memset(B, 0, sizeof(double) * 2 * (size_t)nms * (lmax + 1));
    if (lmax < 2) return;
#pragma omp parallel
    {
        double *a = (double *)calloc((size_t)lmax + 2, sizeof(double)), *b = (double *)calloc((size_t)lmax + 2, sizeof(double)),
               *c = (double *)calloc((size_t)lmax + 2, sizeof(double)), *a2 = (double *)calloc((size_t)lmax + 2, sizeof(double)),
               *b2 = (double *)calloc((size_t)lmax + 2, sizeof(double)), *c2 = (double *)calloc((size_t)lmax + 2, sizeof(double));
        double *lp2 = (double *)calloc((size_t)lmax + 1, sizeof(double)), *lm2 = (double *)calloc((size_t)lmax + 1, sizeof(double));
#pragma omp for schedule(dynamic, 1)
        for (int j = 0; j < nms; ++j) {
            const int m = ms[j], l0 = m > 2 ? m : 2;
            double *e = E + 2 * (size_t)j * (lmax + 1), *bb = B + 2 * (size_t)j * (lmax + 1);
            spin_coefs(lmax, m, -2, a, b, c);
            spin_coefs(lmax, m, 2, a2, b2, c2);
            for (int64_t r = 0; r < nr; ++r) {
                long double th = theta[r];
                long double lc = log2l(cosl(0.5L * th)), lsn = log2l(sinl(0.5L * th));
                spin_lambda_point(lmax, m, -2, x[r], lc, lsn, a, b, c, lp2);
                spin_lambda_point(lmax, m, 2, x[r], lc, lsn, a2, b2, c2, lm2);
                const double qr = Qf[2 * ((int64_t)j * nr + r)], qi = Qf[2 * ((int64_t)j * nr + r) + 1];
                const double ur = Uf[2 * ((int64_t)j * nr + r)], ui = Uf[2 * ((int64_t)j * nr + r) + 1];
                for (int l = l0; l <= lmax; ++l) {
                    double lp = 0.5 * (lp2[l] + lm2[l]), lm = 0.5 * (lp2[l] - lm2[l]);
                    e[2 * l] -= lp * qr - lm * ui;
                    e[2 * l + 1] -= lp * qi + lm * ur;
                    bb[2 * l] -= lp * ur + lm * qi;
                    bb[2 * l + 1] -= lp * ui - lm * qr;
                }
            }
        }
        free(a); free(b); free(c); free(a2); free(b2); free(c2); free(lp2); free(lm2);
    }
}

/* Spin-2 synthesis.  Qg[m][r] = -sum_l (E lp + i B lm), Ug[m][r] = -sum_l (B lp - i E lm). */
void orc_spin2_synthesis(int lmax, int mmax, int64_t nr, const double *x, const double *theta,
                         const double *E, const double *B, double *Qg, double *Ug) {
    memset(Qg, 0, sizeof(double) * 2 * (size_t)(mmax + 1) * nr);
    memset(Ug, 0, sizeof(double) * 2 * (size_t)(mmax + 1) * nr);
    if (lmax < 2) return;
#pragma omp parallel
    {
        double *a = (double *)calloc((size_t)lmax + 2, sizeof(double)), *b = (double *)calloc((size_t)lmax + 2, sizeof(double)),
               *c = (double *)calloc((size_t)lmax + 2, sizeof(double)), *a2 = (double *)calloc((size_t)lmax + 2, sizeof(double)),
               *b2 = (double *)calloc((size_t)lmax + 2, sizeof(double)), *c2 = (double *)calloc((size_t)lmax + 2, sizeof(double));
        double *lp2 = (double *)calloc((size_t)lmax + 1, sizeof(double)), *lm2 = (double *)calloc((size_t)lmax + 1, sizeof(double));
#pragma omp for schedule(dynamic, 1)
        for (int m = 0; m <= mmax; ++m) {
            int l0 = m > 2 ? m : 2;
            spin_coefs(lmax, m, -2, a, b, c);
            spin_coefs(lmax, m, 2, a2, b2, c2);
            for (int64_t r = 0; r < nr; ++r) {
                long double th = theta[r];
                long double lc = log2l(cosl(0.5L * th)), lsn = log2l(sinl(0.5L * th));
                spin_lambda_point(lmax, m, -2, x[r], lc, lsn, a, b, c, lp2);
                spin_lambda_point(lmax, m, 2, x[r], lc, lsn, a2, b2, c2, lm2);
                double q0 = 0, q1 = 0, u0 = 0, u1 = 0;
                for (int l = l0; l <= lmax; ++l) {
                    int64_t k = alm_idx(lmax, l, m);
                    double er = E[2 * k], ei = E[2 * k + 1], br = B[2 * k], bi = B[2 * k + 1];
                    double lp = 0.5 * (lp2[l] + lm2[l]), lm = 0.5 * (lp2[l] - lm2[l]);
                    q0 -= er * lp - bi * lm;
                    q1 -= ei * lp + br * lm;
                    u0 -= br * lp + ei * lm;
                    u1 -= bi * lp - er * lm;
                }
                Qg[2 * ((int64_t)m * nr + r)] = q0; Qg[2 * ((int64_t)m * nr + r) + 1] = q1;
                Ug[2 * ((int64_t)m * nr + r)] = u0; Ug[2 * ((int64_t)m * nr + r) + 1] = u1;
            }
        }
        free(a); free(b); free(c); free(a2); free(b2); free(c2); free(lp2); free(lm2);
    }
}

/* ------------------------------------------------------------------ alm2cl */
/* alm_ops.py:19-32 restated for the healpy layout, with an optional second alm for cross spectra:
 * cl[l] = (Re(a_l0 b_l0*) + 2 sum_{m=1}^{min(l,mmax)} Re(a_lm b_lm*)) / (2l+1). */
void orc_alm2cl(int lmax, int mmax, const double *alm1, const double *alm2, double *cl) {
    if (!alm2) alm2 = alm1;
    for (int l = 0; l <= lmax; ++l) {
        double acc = 0.0;
        int mtop = l < mmax ? l : mmax;
        for (int m = 0; m <= mtop; ++m) {
            int64_t k = alm_idx(lmax, l, m);
            double v = alm1[2 * k] * alm2[2 * k] + alm1[2 * k + 1] * alm2[2 * k + 1];
            acc += (m == 0) ? v : 2.0 * v;
        }
        cl[l] = acc / (2.0 * l + 1.0);
    }
}

/* ------------------------------------------------------------------ pixel indexing */
/* HEALPix pixelisation (Gorski et al. 2005, ApJ 622, 759, sections 4-5): 12 base faces, face f
 * with corner ring jrll[f] * nside and corner longitude index jpll[f]; NESTED index
 * f nside^2 + (ix, iy) bit-interleaved (ix in the even bits); RING index counted ring by ring
 * from the north pole.  Restated for the parity tests of the reference's coordinate kernels
 * (coords_ring.cu:9-54, nested_gpu.cu:27-95, nested_pix2ang.cu:16-85, order_convert.py:8-34). */
static const int ORC_JRLL[12] = {2, 2, 2, 2, 3, 3, 3, 3, 4, 4, 4, 4};
static const int ORC_JPLL[12] = {1, 3, 5, 7, 0, 2, 4, 6, 1, 3, 5, 7};

static int64_t orc_spread(int64_t v) { /* bit i of v -> bit 2i */
    int64_t r = 0;
    for (int b = 0; b < 31; ++b) r |= ((v >> b) & 1LL) << (2 * b);
    return r;
}
static int64_t orc_compress(int64_t v) { /* bit 2i of v -> bit i */
    int64_t r = 0;
    for (int b = 0; b < 31; ++b) r |= ((v >> (2 * b)) & 1LL) << b;
    return r;
}
static int64_t orc_isqrt(int64_t v) {
    int64_t r = (int64_t)sqrt((double)v);
    while (r * r > v) --r;
    while ((r + 1) * (r + 1) <= v) ++r;
    return r;
}

static void orc_nest2xyf(int64_t nside, int64_t p, int64_t *ix, int64_t *iy, int *f) {
    int64_t nn = nside * nside;
    *f = (int)(p / nn);
    p -= (int64_t)(*f) * nn;
    *ix = orc_compress(p);
    *iy = orc_compress(p >> 1);
}
static int64_t orc_xyf2nest(int64_t nside, int64_t ix, int64_t iy, int f) {
    return (int64_t)f * nside * nside + orc_spread(ix) + 2 * orc_spread(iy);
}
static int64_t orc_xyf2ring(int64_t nside, int64_t ix, int64_t iy, int f) {
    int64_t nl4 = 4 * nside, ncap = 2 * nside * (nside - 1), npix = 12 * nside * nside;
    int64_t jr = (int64_t)ORC_JRLL[f] * nside - ix - iy - 1, nr, nbefore;
    int kshift;
    if (jr < nside) { nr = jr; nbefore = 2 * nr * (nr - 1); kshift = 0; }
    else if (jr > 3 * nside) { nr = nl4 - jr; nbefore = npix - 2 * (nr + 1) * nr; kshift = 0; }
    else { nr = nside; nbefore = ncap + (jr - nside) * nl4; kshift = (int)((jr - nside) & 1); }
    int64_t jp = ((int64_t)ORC_JPLL[f] * nr + ix - iy + 1 + kshift) / 2;
    if (jp > 4 * nr) jp -= 4 * nr;
    else if (jp < 1) jp += 4 * nr;
    return nbefore + jp - 1;
}
static void orc_ring2xyf(int64_t nside, int64_t p, int64_t *ix, int64_t *iy, int *f) {
    int64_t nl2 = 2 * nside, ncap = 2 * nside * (nside - 1), npix = 12 * nside * nside;
    int64_t iring, iphi, nr;
    int kshift, face;
    if (p < ncap) {
        iring = (1 + orc_isqrt(1 + 2 * p)) >> 1;
        iphi = p + 1 - 2 * iring * (iring - 1);
        kshift = 0; nr = iring;
        face = (int)((iphi - 1) / nr);
    } else if (p < npix - ncap) {
        int64_t ip = p - ncap, tmp = ip / (4 * nside);
        iring = tmp + nside;
        iphi = ip - tmp * 4 * nside + 1;
        kshift = (int)((iring + nside) & 1);
        nr = nside;
        int64_t ire = tmp + 1, irm = nl2 + 2 - ire;
        int64_t ifm = (iphi - ire / 2 + nside - 1) / nside, ifp = (iphi - irm / 2 + nside - 1) / nside;
        face = (ifp == ifm) ? (int)(ifp | 4) : ((ifp < ifm) ? (int)ifp : (int)(ifm + 8));
    } else {
        int64_t ip = npix - p;
        iring = (1 + orc_isqrt(2 * ip - 1)) >> 1;
        iphi = 4 * iring + 1 - (ip - 2 * iring * (iring - 1));
        kshift = 0; nr = iring;
        iring = 2 * nl2 - iring;
        face = 8 + (int)((iphi - 1) / nr);
    }
    int64_t irt = iring - (int64_t)ORC_JRLL[face] * nside + 1;
    int64_t ipt = 2 * iphi - (int64_t)ORC_JPLL[face] * nr - kshift - 1;
    if (ipt >= nl2) ipt -= 8 * nside;
    *ix = (ipt - irt) >> 1;
    *iy = (-ipt - irt) >> 1;
    *f = face;
}

/* RING <-> NESTED index of n pixels */
void orc_ring2nest(int64_t nside, int64_t n, const int64_t *in, int64_t *out) {
#pragma omp parallel for
    for (int64_t i = 0; i < n; ++i) {
        int64_t ix, iy; int f;
        orc_ring2xyf(nside, in[i], &ix, &iy, &f);
        out[i] = orc_xyf2nest(nside, ix, iy, f);
    }
}
void orc_nest2ring(int64_t nside, int64_t n, const int64_t *in, int64_t *out) {
#pragma omp parallel for
    for (int64_t i = 0; i < n; ++i) {
        int64_t ix, iy; int f;
        orc_nest2xyf(nside, in[i], &ix, &iy, &f);
        out[i] = orc_xyf2ring(nside, ix, iy, f);
    }
}

/* pixel centre (z = cos theta, phi) of RING pixel p */
static void orc_ring_center(int64_t nside, int64_t p, double *z, double *phi) {
    const double pi = 3.141592653589793238462643383279502884;
    int64_t ncap = 2 * nside * (nside - 1), npix = 12 * nside * nside;
    double fact2 = 4.0 / (double)npix;
    if (p < ncap) {
        int64_t iring = (1 + orc_isqrt(1 + 2 * p)) >> 1, iphi = p + 1 - 2 * iring * (iring - 1);
        *z = 1.0 - (double)(iring * iring) * fact2;
        *phi = ((double)iphi - 0.5) * (pi / (2.0 * (double)iring));
    } else if (p < npix - ncap) {
        int64_t ip = p - ncap, tmp = ip / (4 * nside), iring = tmp + nside, iphi = ip - tmp * 4 * nside + 1;
        double fodd = ((iring + nside) & 1) ? 1.0 : 0.5;
        *z = (double)(2 * nside - iring) * (2.0 / (3.0 * (double)nside));
        *phi = ((double)iphi - fodd) * (pi / (2.0 * (double)nside));
    } else {
        int64_t ip = npix - p, iring = (1 + orc_isqrt(2 * ip - 1)) >> 1;
        int64_t iphi = 4 * iring + 1 - (ip - 2 * iring * (iring - 1));
        *z = -1.0 + (double)(iring * iring) * fact2;
        *phi = ((double)iphi - 0.5) * (pi / (2.0 * (double)iring));
    }
}
/* NESTED or RING pixel centres: theta, phi */
void orc_pix2ang(int64_t nside, int nest, int64_t n, const int64_t *pix, double *theta, double *phi) {
#pragma omp parallel for
    for (int64_t i = 0; i < n; ++i) {
        int64_t p = pix[i];
        if (nest) {
            int64_t ix, iy; int f;
            orc_nest2xyf(nside, p, &ix, &iy, &f);
            p = orc_xyf2ring(nside, ix, iy, f);
        }
        double z;
        orc_ring_center(nside, p, &z, &phi[i]);
        theta[i] = acos(z);
    }
}

/* (z, phi) -> RING / NESTED pixel containing it */
static void orc_zphi2xyf_or_ring(int64_t nside, double z, double phi, int nest, int64_t *out) {
    const double pi = 3.141592653589793238462643383279502884;
    double za = fabs(z);
    double tt = fmod(phi, 2.0 * pi);
    if (tt < 0.0) tt += 2.0 * pi;
    tt *= 2.0 / pi; /* [0, 4) */
    if (tt >= 4.0) tt = 0.0;
    int64_t ncap = 2 * nside * (nside - 1), npix = 12 * nside * nside;
    if (!nest) {
        if (za <= 2.0 / 3.0) {
            double t1 = (double)nside * (0.5 + tt), t2 = (double)nside * z * 0.75;
            int64_t jp = (int64_t)(t1 - t2), jm = (int64_t)(t1 + t2);
            int64_t ir = nside + 1 + jp - jm, kshift = 1 - (ir & 1);
            int64_t ip = (jp + jm - nside + kshift + 1) / 2;
            ip %= 4 * nside; if (ip < 0) ip += 4 * nside;
            *out = ncap + (ir - 1) * 4 * nside + ip;
        } else {
            double tp = tt - (double)(int64_t)tt, tmp = (double)nside * sqrt(3.0 * (1.0 - za));
            int64_t jp = (int64_t)(tp * tmp), jm = (int64_t)((1.0 - tp) * tmp);
            int64_t ir = jp + jm + 1, ip = (int64_t)(tt * (double)ir);
            ip %= 4 * ir; if (ip < 0) ip += 4 * ir;
            *out = (z > 0.0) ? 2 * ir * (ir - 1) + ip : npix - 2 * ir * (ir + 1) + ip;
        }
        return;
    }
    int64_t ix, iy; int face;
    if (za <= 2.0 / 3.0) {
        double t1 = (double)nside * (0.5 + tt), t2 = (double)nside * z * 0.75;
        int64_t jp = (int64_t)(t1 - t2), jm = (int64_t)(t1 + t2);
        int64_t ifp = jp / nside, ifm = jm / nside;
        face = (ifp == ifm) ? (int)(ifp | 4) : ((ifp < ifm) ? (int)ifp : (int)(ifm + 8));
        ix = jm & (nside - 1);
        iy = nside - (jp & (nside - 1)) - 1;
    } else {
        int ntt = (int)tt; if (ntt >= 4) ntt = 3;
        double tp = tt - (double)ntt, tmp = (double)nside * sqrt(3.0 * (1.0 - za));
        int64_t jp = (int64_t)(tp * tmp), jm = (int64_t)((1.0 - tp) * tmp);
        if (jp > nside - 1) jp = nside - 1;
        if (jm > nside - 1) jm = nside - 1;
        if (z >= 0.0) { face = ntt; ix = nside - jm - 1; iy = nside - jp - 1; }
        else { face = ntt + 8; ix = jp; iy = jm; }
    }
    *out = orc_xyf2nest(nside, ix, iy, face);
}
void orc_ang2pix(int64_t nside, int nest, int64_t n, const double *theta, const double *phi, int64_t *pix) {
#pragma omp parallel for
    for (int64_t i = 0; i < n; ++i) orc_zphi2xyf_or_ring(nside, cos(theta[i]), phi[i], nest, &pix[i]);
}

/* ------------------------------------------------------------------ Wigner d */
/* d^l_{m,m'}(beta) for m, m' = -l..l into out[(m+l)(2l+1) + m'+l], long double three-term
 * recursion in l at fixed (m, m') from the edge element at l0 = max(|m|,|m'|)
 * (d^j_{j,k} = sqrt((2j)!/((j+k)!(j-k)!)) cos(b/2)^{j+k} (-sin(b/2))^{j-k},
 * d_{a,b} = (-1)^{a-b} d_{b,a} = d_{-b,-a}); beta reduced to [0, pi] first
 * (d(2pi - b) = (-1)^{m-m'} d(b)).  For the parity tests of the alm rotation
 * (rotate_alm_euler.py:5-14, wigner_full.py:12-96). */
void orc_wigner_d(int l, double beta, double *out) {
    const long double pi = 3.141592653589793238462643383279502884L;
    long double b = fmodl((long double)beta, 2.0L * pi);
    if (b < 0) b += 2.0L * pi;
    int flip = b > pi;
    if (flip) b = 2.0L * pi - b;
    long double c = cosl(0.5L * b), s = sinl(0.5L * b), x = cosl(b);
    int dim = 2 * l + 1;
    for (int m = -l; m <= l; ++m) {
        for (int mp = -l; mp <= l; ++mp) {
            int j, k, sh;
            if (abs(m) >= abs(mp)) {
                if (m >= 0) { j = m; k = mp; sh = 0; }
                else { j = -m; k = -mp; sh = (mp + j) & 1; }
            } else {
                if (mp > 0) { j = mp; k = m; sh = (m - j) & 1; }
                else { j = -mp; k = -m; sh = 0; }
            }
            int l0 = j;
            /* edge element, log-scaled like the spin-2 starts above */
            long double L = 0.5L * (lfac2(2 * j) - lfac2(j + k) - lfac2(j - k));
            int zero = 0;
            if (j + k > 0) { if (c == 0) zero = 1; else L += (j + k) * log2l(c); }
            if (j - k > 0) { if (s == 0) zero = 1; else L += (j - k) * log2l(s); }
            int sign = (((j - k) & 1) ^ sh) ? -1 : 1;
            long double d1 = 0, d0 = 0;
            int e = 0;
            if (!zero) {
                e = (int)floorl((L + 128.0L) / 256.0L);
                d1 = exp2l(L - 256.0L * e) * sign;
            }
            for (int ll = l0; ll < l; ++ll) {
                long double v;
                if (ll == 0) v = x * d1;
                else {
                    long double dl = ll, m2 = (long double)m * m, p2 = (long double)mp * mp;
                    long double R1 = sqrtl(((dl + 1) * (dl + 1) - m2) * ((dl + 1) * (dl + 1) - p2));
                    long double R0 = sqrtl((dl * dl - m2) * (dl * dl - p2));
                    v = ((2 * dl + 1) * (dl * (dl + 1) * x - (long double)m * mp) * d1 - (dl + 1) * R0 * d0) / (dl * R1);
                }
                d0 = d1; d1 = v;
                if (e < 0 && fabsl(d1) > 0x1p128L) { d1 = ldexpl(d1, -256); d0 = ldexpl(d0, -256); ++e; }
            }
            double v = (e == 0) ? (double)d1 : 0.0;
            if (flip && ((m - mp) & 1)) v = -v;
            out[(m + l) * dim + (mp + l)] = v;
        }
    }
}
