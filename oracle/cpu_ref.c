/*
 * ORACLE — TEST INFRASTRUCTURE ONLY. Plain-C (OpenMP) restatement of the reference's CPU coupling
 * path, used as the parity reference in tests/ and as the timed CPU baseline in bench.py. The
 * product (yasf_b200/) never links or calls this file.
 *
 * Restated functions (file:line within the reference project):
 *   spherical Bessel / Hankel values      yasfpy/functions/misc.py:183-193 (SciPy spherical_jn/yn)
 *   normalised Legendre P~_p^m            yasfpy/functions/legendre_normalized_trigon.py:12-95
 *   pair geometry and lookup tables       yasfpy/functions/misc.py:117-243 (mutual_lookup)
 *   coupling matvec (R = 1)               yasfpy/functions/cpu_numba.py:22-95
 *                                         (particle_interaction_scalar)
 *   scattering cross-section bilinear     yasfpy/functions/cpu_numba.py:410-457
 *                                         (compute_scattering_cross_section)
 *
 * As in the reference, the lookup tables (plm, sph_h / sph_j, e_j_dm_phi) are materialised before
 * the 4-deep interaction loop; here they are built for the receiving rows actually evaluated
 * (a row sample [s1_begin, s1_end) of the full product), so large aggregates can be sampled.
 * Complex numbers are interleaved (re, im) doubles. translation_ab5 has the reference layout
 * [n_source][n_receiver][p] as read by cpu_numba.py:86.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

/* spherical j_p(x), y_p(x) for p = 0..pmax (SciPy semantics for real x > 0; j_p(0) = delta_p0). */
void oracle_sph_bessel(int pmax, double x, double* jp, double* yp) {
  int p;
  if (x == 0.0) {
    for (p = 0; p <= pmax; ++p) {
      jp[p] = p == 0 ? 1.0 : 0.0;
      yp[p] = -INFINITY;
    }
    return;
  }
  const double s = sin(x), c = cos(x);
  /* y_p: upward recurrence is stable */
  yp[0] = -c / x;
  if (pmax >= 1) yp[1] = -c / (x * x) - s / x;
  for (p = 1; p < pmax; ++p) yp[p + 1] = (2.0 * p + 1.0) / x * yp[p] - yp[p - 1];
  /* j_p: upward while p < x, else Miller's downward recurrence normalised on j_0 / j_1 */
  if (x > (double)pmax + 1.0) {
    jp[0] = s / x;
    if (pmax >= 1) jp[1] = s / (x * x) - c / x;
    for (p = 1; p < pmax; ++p) jp[p + 1] = (2.0 * p + 1.0) / x * jp[p] - jp[p - 1];
    return;
  }
  {
    const int nstart = pmax + 30 + (int)x;
    double fnext = 0.0, f = 1e-250, fprev;
    double* buf = (double*)malloc(sizeof(double) * (size_t)(nstart + 2));
    int q;
    buf[nstart + 1] = 0.0;
    buf[nstart] = f;
    for (q = nstart; q > 0; --q) {
      fprev = (2.0 * q + 1.0) / x * buf[q] - buf[q + 1];
      buf[q - 1] = fprev;
      if (fabs(fprev) > 1e250) {
        int t;
        for (t = q - 1; t <= nstart; ++t) buf[t] *= 1e-250;
      }
    }
    (void)fnext;
    const double j0 = s / x, j1 = s / (x * x) - c / x;
    const double scale = (fabs(j0) >= fabs(j1)) ? j0 / buf[0] : j1 / buf[1];
    for (p = 0; p <= pmax; ++p) jp[p] = buf[p] * scale;
    free(buf);
  }
}

/* P~_l^m(ct, st) for l, m <= lmax, out[l*(lmax+1) + m] (CELES recurrence). */
void oracle_legendre(int lmax, double ct, double st, double* out) {
  const int W = lmax + 1;
  int l, m;
  memset(out, 0, sizeof(double) * (size_t)W * W);
  out[0] = sqrt(0.5);
  if (lmax >= 1) out[1 * W + 0] = sqrt(1.5) * ct;
  for (l = 1; l < lmax; ++l)
    out[(l + 1) * W + 0] = 1.0 / (l + 1) * sqrt((2.0 * l + 1) * (2.0 * l + 3)) * out[l * W] * ct -
                           (double)l / (l + 1) * sqrt((2.0 * l + 3) / (2.0 * l - 1)) * out[(l - 1) * W];
  for (m = 1; m <= lmax; ++m) {
    double fact = 1.0, dfact = 1.0;
    int t;
    for (t = 2; t <= 2 * m; ++t) fact *= t;
    for (t = 1; t <= 2 * m - 1; t += 2) dfact *= t;
    out[m * W + m] = sqrt((2.0 * m + 1) / 2.0 / fact) * dfact * pow(st, m);
    for (l = m; l < lmax; ++l) {
      const double prev = (l - 1 >= 0 && l - 1 >= m) ? out[(l - 1) * W + m] : 0.0;
      out[(l + 1) * W + m] =
          sqrt((2.0 * l + 1) * (2.0 * l + 3) / (l + 1 - m) / (l + 1 + m)) * ct * out[l * W + m] -
          sqrt((2.0 * l + 3) * (l - m) * (l + m) / (2.0 * l - 1) / (l + 1 - m) / (l + 1 + m)) * prev;
    }
  }
}

typedef struct {
  int n;      /* s */
  int tau, l, m;
} mode_desc;

static void modes_of(int lmax, mode_desc* md) {
  int tau, l, m;
  for (tau = 1; tau <= 2; ++tau)
    for (l = 1; l <= lmax; ++l)
      for (m = -l; m <= l; ++m) {
        const int n = (tau - 1) * lmax * (lmax + 2) + (l - 1) * (l + 1) + l + m;
        md[n].n = n;
        md[n].tau = tau;
        md[n].l = l;
        md[n].m = m;
      }
}

/* Lookup tables of mutual_lookup for one receiver s1 against all sources:
 * plm[(p(p+1)/2 + dm) * N + s2], sph[(p * N + s2) * 2 + {re,im}] (h_p, or j_p when regular),
 * eph[(q * N + s2) * 2 + ...] = exp(i (q - 2lmax) phi). */
static void lookups_row(int lmax, int N, const double* pos, double k, int s1, int regular,
                        double* plm, double* sph, double* eph, double* jp, double* yp, double* leg) {
  const int P = 2 * lmax;
  int s2, p, dm, q;
  for (s2 = 0; s2 < N; ++s2) {
    const double dx = pos[3 * s1] - pos[3 * s2], dy = pos[3 * s1 + 1] - pos[3 * s2 + 1],
                 dz = pos[3 * s1 + 2] - pos[3 * s2 + 2];
    const double r = sqrt(dx * dx + dy * dy + dz * dz);
    double ct = r != 0.0 ? dz / r : 0.0;
    if (ct < -1) ct = -1;
    if (ct > 1) ct = 1;
    const double st = sqrt(1.0 - ct * ct);
    const double phi = atan2(dy, dx);
    const double x = k * r;
    oracle_sph_bessel(P, x, jp, yp);
    for (p = 0; p <= P; ++p) {
      if (regular) {
        sph[(p * N + s2) * 2] = jp[p];
        sph[(p * N + s2) * 2 + 1] = 0.0;
      } else if (x != 0.0) {
        sph[(p * N + s2) * 2] = jp[p];
        sph[(p * N + s2) * 2 + 1] = yp[p];
      } else { /* the reference stores 0 where r = 0 (misc.py:189-193, j at 0 is kept) */
        sph[(p * N + s2) * 2] = jp[p];
        sph[(p * N + s2) * 2 + 1] = 0.0;
      }
    }
    oracle_legendre(P, ct, st, leg);
    for (p = 0; p <= P; ++p)
      for (dm = 0; dm <= p; ++dm) plm[(p * (p + 1) / 2 + dm) * N + s2] = leg[p * (P + 1) + dm];
    for (q = 0; q <= 2 * P; ++q) {
      const double a = (q - P) * phi;
      eph[(q * N + s2) * 2] = cos(a);
      eph[(q * N + s2) * 2 + 1] = sin(a);
    }
  }
}

/* wx[(s1 - s1_begin) * nmax + n1] = (W x)[s1, n1] for s1 in [s1_begin, s1_end).
 * The interaction loop follows particle_interaction_scalar: j1 -> s2 != s1 -> j2 -> p.
 * cutoff2 >= 0 keeps only the pairs with |pos[s1] - pos[s2]|^2 <= cutoff2, the near-field pairs of
 * the reference's NearFarCouplingBackend (yasfpy/coupling/backends.py:259-459); < 0 keeps all. */
int oracle_coupling_matvec_cutoff(int lmax, int N, const double* pos, double k, const double* ab5,
                                  const double* x, int s1_begin, int s1_end, double* wx, int threads,
                                  double cutoff2);

int oracle_coupling_matvec(int lmax, int N, const double* pos, double k, const double* ab5,
                           const double* x, int s1_begin, int s1_end, double* wx, int threads) {
  return oracle_coupling_matvec_cutoff(lmax, N, pos, k, ab5, x, s1_begin, s1_end, wx, threads, -1.0);
}

int oracle_coupling_matvec_cutoff(int lmax, int N, const double* pos, double k, const double* ab5,
                                  const double* x, int s1_begin, int s1_end, double* wx, int threads,
                                  double cutoff2) {
  const int nmax = 2 * lmax * (lmax + 2), P = 2 * lmax, NP = P + 1;
  const int nplm = (P + 1) * (P + 2) / 2;
  mode_desc* md = (mode_desc*)malloc(sizeof(mode_desc) * nmax);
  int s1;
  modes_of(lmax, md);
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#endif
  for (s1 = s1_begin; s1 < s1_end; ++s1) {
    double* plm = (double*)malloc(sizeof(double) * (size_t)nplm * N);
    double* sph = (double*)malloc(sizeof(double) * 2 * (size_t)NP * N);
    double* eph = (double*)malloc(sizeof(double) * 2 * (size_t)(2 * P + 1) * N);
    double* jp = (double*)malloc(sizeof(double) * (NP + 1));
    double* yp = (double*)malloc(sizeof(double) * (NP + 1));
    double* leg = (double*)malloc(sizeof(double) * (size_t)(P + 1) * (P + 1));
    int n1;
    lookups_row(lmax, N, pos, k, s1, 0, plm, sph, eph, jp, yp, leg);
#pragma omp parallel for schedule(static)
    for (n1 = 0; n1 < nmax; ++n1) {
      const int tau1 = md[n1].tau, l1 = md[n1].l, m1 = md[n1].m;
      double ar = 0.0, ai = 0.0;
      int s2, n2, p;
      for (s2 = 0; s2 < N; ++s2) {
        if (s2 == s1) continue;
        if (cutoff2 >= 0.0) {
          const double dx = pos[3 * s1] - pos[3 * s2], dy = pos[3 * s1 + 1] - pos[3 * s2 + 1],
                       dz = pos[3 * s1 + 2] - pos[3 * s2 + 2];
          if (dx * dx + dy * dy + dz * dz > cutoff2) continue;
        }
        for (n2 = 0; n2 < nmax; ++n2) {
          const int tau2 = md[n2].tau, l2 = md[n2].l, m2 = md[n2].m;
          const int dtau = abs(tau1 - tau2), dl = abs(l1 - l2), dm = abs(m1 - m2);
          int p_start = dm;
          if (dl + dtau > p_start) p_start = dl + dtau;
          const double* e = eph + ((size_t)(m2 - m1 + P) * N + s2) * 2;
          const double* xv = x + ((size_t)s2 * nmax + n2) * 2;
          const double pxr = e[0] * xv[0] - e[1] * xv[1];
          const double pxi = e[0] * xv[1] + e[1] * xv[0];
          for (p = p_start; p <= l1 + l2; ++p) {
            const double* A = ab5 + (((size_t)n2 * nmax + n1) * NP + p) * 2;
            const double pl = plm[(size_t)(p * (p + 1) / 2 + dm) * N + s2];
            const double* h = sph + ((size_t)p * N + s2) * 2;
            /* A * pl * phase_x * h */
            const double tr = (A[0] * pxr - A[1] * pxi) * pl;
            const double ti = (A[0] * pxi + A[1] * pxr) * pl;
            ar += tr * h[0] - ti * h[1];
            ai += tr * h[1] + ti * h[0];
          }
        }
      }
      wx[((size_t)(s1 - s1_begin) * nmax + n1) * 2] = ar;
      wx[((size_t)(s1 - s1_begin) * nmax + n1) * 2 + 1] = ai;
    }
    free(plm);
    free(sph);
    free(eph);
    free(jp);
    free(yp);
    free(leg);
  }
  free(md);
  return 0;
}

/* out[0..1] = sum_{s1 in [s1_begin, s1_end), n1, s2, n2} conj(b1) e^{i(m2-m1)phi}
 *             b2 sum_{p = |dm|}^{2lmax} A[n2,n1,p] P~_p^{|dm|} j_p   (self pairs included). */
int oracle_scattering_bilinear(int lmax, int N, const double* pos, double k, const double* ab5,
                               const double* b, int s1_begin, int s1_end, double* out, int threads) {
  const int nmax = 2 * lmax * (lmax + 2), P = 2 * lmax, NP = P + 1;
  const int nplm = (P + 1) * (P + 2) / 2;
  mode_desc* md = (mode_desc*)malloc(sizeof(mode_desc) * nmax);
  double tot_r = 0.0, tot_i = 0.0;
  int s1;
  modes_of(lmax, md);
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#endif
  for (s1 = s1_begin; s1 < s1_end; ++s1) {
    double* plm = (double*)malloc(sizeof(double) * (size_t)nplm * N);
    double* sph = (double*)malloc(sizeof(double) * 2 * (size_t)NP * N);
    double* eph = (double*)malloc(sizeof(double) * 2 * (size_t)(2 * P + 1) * N);
    double* jp = (double*)malloc(sizeof(double) * (NP + 1));
    double* yp = (double*)malloc(sizeof(double) * (NP + 1));
    double* leg = (double*)malloc(sizeof(double) * (size_t)(P + 1) * (P + 1));
    double rr = 0.0, ri = 0.0;
    int n1;
    lookups_row(lmax, N, pos, k, s1, 1, plm, sph, eph, jp, yp, leg);
#pragma omp parallel for schedule(static) reduction(+ : rr, ri)
    for (n1 = 0; n1 < nmax; ++n1) {
      const int m1 = md[n1].m;
      const double* b1 = b + ((size_t)s1 * nmax + n1) * 2;
      int s2, n2, p;
      for (s2 = 0; s2 < N; ++s2) {
        for (n2 = 0; n2 < nmax; ++n2) {
          const int m2 = md[n2].m, dm = abs(m1 - m2);
          double vr = 0.0, vi = 0.0;
          for (p = dm; p <= P; ++p) {
            const double* A = ab5 + (((size_t)n2 * nmax + n1) * NP + p) * 2;
            const double pl = plm[(size_t)(p * (p + 1) / 2 + dm) * N + s2];
            const double jv = sph[((size_t)p * N + s2) * 2];
            vr += A[0] * pl * jv;
            vi += A[1] * pl * jv;
          }
          const double* e = eph + ((size_t)(m2 - m1 + P) * N + s2) * 2;
          const double* b2 = b + ((size_t)s2 * nmax + n2) * 2;
          /* conj(b1) * e * b2 */
          const double cr = b1[0] * e[0] + b1[1] * e[1];
          const double ci = b1[0] * e[1] - b1[1] * e[0];
          const double fr = cr * b2[0] - ci * b2[1];
          const double fi = cr * b2[1] + ci * b2[0];
          rr += vr * fr - vi * fi;
          ri += vr * fi + vi * fr;
        }
      }
    }
    tot_r += rr;
    tot_i += ri;
    free(plm);
    free(sph);
    free(eph);
    free(jp);
    free(yp);
    free(leg);
  }
  out[0] = tot_r;
  out[1] = tot_i;
  free(md);
  return 0;
}

int oracle_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
