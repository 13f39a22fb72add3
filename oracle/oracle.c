/*
 * oracle.c -- CPU FP64 restatement of OpenPFC's spectral PFC time step.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
 * calls this file.  It is imported by tests/, by __graft_entry__.smoke() and by
 * bench.py's CPU-baseline / reference arm, always as the checker or as the
 * timed CPU baseline, never as the thing being measured on the GPU.
 *
 * Parity pins (checked in tests/test_oracle.py):
 *   - FFT known answers of tests/unit/kernel/fft/test_fft.cpp:28-70 and
 *     tests/unit/runtime/gpu/test_fft_cuda.cpp:84-189;
 *   - numpy.fft.rfftn / irfftn (pocketfft, float64) at 8^3..64^3;
 *   - Tungsten golden L2^2 norms of apps/tungsten/tests/test_tungsten.cpp:288-300;
 *   - operator tables produced by the reference's own header-only code
 *     (tungsten_spectral.hpp, spectral_exp_coefficients.hpp, tungsten_params.hpp)
 *     compiled by oracle/Makefile into oracle/_ref/ref_ops.
 *
 * Conventions restated (file:line in the reference project):
 *   - real fields x-fastest, idx = i + N0*(j + N1*k)
 *       (include/openpfc/kernel/field/operations.hpp:96-103);
 *   - complex half spectrum (N0/2+1) x N1 x N2, same order
 *       (src/openpfc/runtime/cpu/fft.cpp:58-70);
 *   - forward transform unnormalised, backward scaled by 1/(N0*N1*N2)
 *       (include/openpfc/kernel/fft/detail/fft_heffte_backend.hpp:216,243);
 *   - k_i = i*f for i <= N/2 else (i-N)*f with f = 2*pi/(dx*N)
 *       (include/openpfc/kernel/fft/kspace.hpp:97-103,165-167).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_PI 3.14159265358979323846264338327950288

/* ------------------------------------------------------------------------- */
/* 1D mixed-radix complex FFT (Stockham autosort, out of place, FP64).        */
/* ------------------------------------------------------------------------- */

typedef struct {
  int n;
  int nf;
  int fac[40];
  double *tw; /* exp(-2*pi*i*k/n), k = 0..n-1, interleaved */
} orc_plan;

/* cos/sin of 2*pi*k/n with octant reduction so special angles are exact. */
static void unit_root(long k, long n, double *c, double *s) {
  k %= n;
  if (k < 0) k += n;
  /* reduce to [0, n/8] using symmetries when n divisible by 8 */
  long k8 = 8 * k;
  if (n % 8 == 0) {
    long oct = k8 / n; /* 0..7 */
    long rem = k - oct * (n / 8);
    double a = 2.0 * ORC_PI * (double)rem / (double)n; /* in [0, pi/4) */
    double ca = cos(a), sa = sin(a);
    double cc = 0, ss = 0;
    double r2 = 0.70710678118654752440084436210484903928;
    switch (oct) {
    case 0: cc = ca; ss = sa; break;
    case 1: cc = r2 * (ca - sa); ss = r2 * (ca + sa); break;
    case 2: cc = -sa; ss = ca; break;
    case 3: cc = -r2 * (ca + sa); ss = r2 * (ca - sa); break;
    case 4: cc = -ca; ss = -sa; break;
    case 5: cc = -r2 * (ca - sa); ss = -r2 * (ca + sa); break;
    case 6: cc = sa; ss = -ca; break;
    default: cc = r2 * (ca + sa); ss = -r2 * (ca - sa); break;
    }
    /* the octant-0 branch is exact at rem == 0, so quarter/half turns are exact */
    *c = cc;
    *s = ss;
    return;
  }
  if (4 * k == n) { *c = 0; *s = 1; return; }
  if (2 * k == n) { *c = -1; *s = 0; return; }
  if (4 * k == 3 * n) { *c = 0; *s = -1; return; }
  double a = 2.0 * ORC_PI * (double)k / (double)n;
  *c = cos(a);
  *s = sin(a);
}

static int plan_init(orc_plan *p, int n) {
  p->n = n;
  p->nf = 0;
  int m = n;
  /* prefer radix 4, then 2, 3, 5, then any prime */
  while (m % 4 == 0) { p->fac[p->nf++] = 4; m /= 4; }
  while (m % 2 == 0) { p->fac[p->nf++] = 2; m /= 2; }
  for (int q = 3; m > 1; q += 2) {
    while (m % q == 0) { p->fac[p->nf++] = q; m /= q; }
  }
  p->tw = (double *)malloc(sizeof(double) * 2 * (size_t)(n > 0 ? n : 1));
  if (!p->tw) return -1;
  for (int k = 0; k < n; ++k) {
    double c, s;
    unit_root(k, n, &c, &s);
    p->tw[2 * k] = c;
    p->tw[2 * k + 1] = -s;
  }
  return 0;
}

static void plan_free(orc_plan *p) { free(p->tw); p->tw = NULL; }

/* One Stockham pass: radix R, sub-length Ns, sign -1 forward / +1 inverse.  */
static void stockham_pass(const double *x, double *y, int n, int R, int Ns,
                          const double *tw, int sign) {
  int nb = n / R;
  double vr[64], vi[64];
  double gbuf_r[64], gbuf_i[64];
  for (int j = 0; j < nb; ++j) {
    int k = j % Ns;
    for (int r = 0; r < R; ++r) {
      double ar = x[2 * (j + r * nb)], ai = x[2 * (j + r * nb) + 1];
      long ti = ((long)k * r * (n / (Ns * R))) % n;
      double wr = tw[2 * ti], wi = sign < 0 ? tw[2 * ti + 1] : -tw[2 * ti + 1];
      vr[r] = ar * wr - ai * wi;
      vi[r] = ar * wi + ai * wr;
    }
    if (R == 2) {
      double tr = vr[1], ti2 = vi[1];
      vr[1] = vr[0] - tr; vi[1] = vi[0] - ti2;
      vr[0] = vr[0] + tr; vi[0] = vi[0] + ti2;
    } else if (R == 4) {
      double ar = vr[0] + vr[2], ai = vi[0] + vi[2];
      double br = vr[0] - vr[2], bi = vi[0] - vi[2];
      double cr = vr[1] + vr[3], ci = vi[1] + vi[3];
      double dr = vr[1] - vr[3], di = vi[1] - vi[3];
      /* multiply d by -i (forward) or +i (inverse) */
      double er = sign < 0 ? di : -di, ei = sign < 0 ? -dr : dr;
      vr[0] = ar + cr; vi[0] = ai + ci;
      vr[2] = ar - cr; vi[2] = ai - ci;
      vr[1] = br + er; vi[1] = bi + ei;
      vr[3] = br - er; vi[3] = bi - ei;
    } else {
      /* generic O(R^2) DFT with the length-n table: w_R^{u r} = w_n^{u r n/R} */
      for (int u = 0; u < R; ++u) {
        double sr = 0, si = 0;
        for (int r = 0; r < R; ++r) {
          long ti = ((long)u * r % R) * (n / R);
          double wr = tw[2 * ti], wi = sign < 0 ? tw[2 * ti + 1] : -tw[2 * ti + 1];
          sr += vr[r] * wr - vi[r] * wi;
          si += vr[r] * wi + vi[r] * wr;
        }
        gbuf_r[u] = sr;
        gbuf_i[u] = si;
      }
      for (int u = 0; u < R; ++u) { vr[u] = gbuf_r[u]; vi[u] = gbuf_i[u]; }
    }
    int idxD = (j / Ns) * Ns * R + k;
    for (int r = 0; r < R; ++r) {
      y[2 * (idxD + r * Ns)] = vr[r];
      y[2 * (idxD + r * Ns) + 1] = vi[r];
    }
  }
}

/* In-place 1D FFT of a contiguous interleaved line; work has 2n doubles. */
static void fft1d(const orc_plan *p, double *data, double *work, int sign) {
  double *x = data, *y = work;
  int Ns = 1;
  for (int f = 0; f < p->nf; ++f) {
    int R = p->fac[f];
    stockham_pass(x, y, p->n, R, Ns, p->tw, sign);
    Ns *= R;
    double *t = x; x = y; y = t;
  }
  if (x != data) memcpy(data, x, sizeof(double) * 2 * (size_t)p->n);
}

int orc_fft1d(int n, double *data, int sign) {
  if (n <= 0) return -1;
  orc_plan p;
  if (plan_init(&p, n)) return -2;
  double *w = (double *)malloc(sizeof(double) * 2 * (size_t)n);
  fft1d(&p, data, w, sign);
  free(w);
  plan_free(&p);
  return 0;
}

/* ------------------------------------------------------------------------- */
/* 3D real <-> half-complex transforms in the reference layout.               */
/* ------------------------------------------------------------------------- */

static int g_threads = 0;
void orc_set_threads(int t) { g_threads = t; }
int orc_get_threads(void) {
#ifdef _OPENMP
  return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
  return 1;
#endif
}

/* complex transforms along y and z of a (nx x N1 x N2) interleaved array */
static void fft_yz(double *c, int nx, int n1, int n2, int sign) {
  orc_plan py, pz;
  plan_init(&py, n1);
  plan_init(&pz, n2);
  int nt = orc_get_threads();
  (void)nt;
  if (n1 > 1) {
#pragma omp parallel num_threads(nt)
    {
      double *line = (double *)malloc(sizeof(double) * 2 * (size_t)n1);
      double *work = (double *)malloc(sizeof(double) * 2 * (size_t)n1);
#pragma omp for schedule(static)
      for (long zl = 0; zl < (long)n2 * nx; ++zl) {
        long z = zl / nx, i = zl % nx;
        for (int j = 0; j < n1; ++j) {
          size_t a = (size_t)i + (size_t)nx * ((size_t)j + (size_t)n1 * z);
          line[2 * j] = c[2 * a];
          line[2 * j + 1] = c[2 * a + 1];
        }
        fft1d(&py, line, work, sign);
        for (int j = 0; j < n1; ++j) {
          size_t a = (size_t)i + (size_t)nx * ((size_t)j + (size_t)n1 * z);
          c[2 * a] = line[2 * j];
          c[2 * a + 1] = line[2 * j + 1];
        }
      }
      free(line);
      free(work);
    }
  }
  if (n2 > 1) {
#pragma omp parallel num_threads(nt)
    {
      double *line = (double *)malloc(sizeof(double) * 2 * (size_t)n2);
      double *work = (double *)malloc(sizeof(double) * 2 * (size_t)n2);
#pragma omp for schedule(static)
      for (long yl = 0; yl < (long)n1 * nx; ++yl) {
        long j = yl / nx, i = yl % nx;
        for (int k = 0; k < n2; ++k) {
          size_t a = (size_t)i + (size_t)nx * ((size_t)j + (size_t)n1 * k);
          line[2 * k] = c[2 * a];
          line[2 * k + 1] = c[2 * a + 1];
        }
        fft1d(&pz, line, work, sign);
        for (int k = 0; k < n2; ++k) {
          size_t a = (size_t)i + (size_t)nx * ((size_t)j + (size_t)n1 * k);
          c[2 * a] = line[2 * k];
          c[2 * a + 1] = line[2 * k + 1];
        }
      }
      free(line);
      free(work);
    }
  }
  plan_free(&py);
  plan_free(&pz);
}

/* Forward R2C: in real n0*n1*n2, out interleaved (n0/2+1)*n1*n2, unnormalised. */
int orc_r2c(int n0, int n1, int n2, const double *in, double *out) {
  if (n0 < 1 || n1 < 1 || n2 < 1) return -1;
  int h = n0 / 2 + 1;
  long rows = (long)n1 * n2;
  orc_plan px;
  plan_init(&px, n0);
  int nt = orc_get_threads();
  (void)nt;
#pragma omp parallel num_threads(nt)
  {
    double *line = (double *)malloc(sizeof(double) * 2 * (size_t)n0);
    double *work = (double *)malloc(sizeof(double) * 2 * (size_t)n0);
#pragma omp for schedule(static)
    for (long rp = 0; rp < (rows + 1) / 2; ++rp) {
      long ra = 2 * rp, rb = 2 * rp + 1;
      int two = rb < rows;
      const double *a = in + (size_t)ra * n0;
      const double *b = two ? in + (size_t)rb * n0 : NULL;
      for (int i = 0; i < n0; ++i) {
        line[2 * i] = a[i];
        line[2 * i + 1] = two ? b[i] : 0.0;
      }
      fft1d(&px, line, work, -1);
      double *oa = out + 2 * (size_t)ra * h;
      double *ob = two ? out + 2 * (size_t)rb * h : NULL;
      for (int k = 0; k < h; ++k) {
        int m = (n0 - k) % n0;
        double zr = line[2 * k], zi = line[2 * k + 1];
        double wr = line[2 * m], wi = -line[2 * m + 1]; /* conj(Z[N-k]) */
        oa[2 * k] = 0.5 * (zr + wr);
        oa[2 * k + 1] = 0.5 * (zi + wi);
        if (two) {
          /* (Z - conj(Z[N-k])) / (2i) */
          double dr = zr - wr, di = zi - wi;
          ob[2 * k] = 0.5 * di;
          ob[2 * k + 1] = -0.5 * dr;
        }
      }
    }
    free(line);
    free(work);
  }
  plan_free(&px);
  fft_yz(out, h, n1, n2, -1);
  return 0;
}

/* Backward C2R with 1/(n0*n1*n2) scaling.  `in` is preserved. */
int orc_c2r(int n0, int n1, int n2, const double *in, double *out) {
  if (n0 < 1 || n1 < 1 || n2 < 1) return -1;
  int h = n0 / 2 + 1;
  long rows = (long)n1 * n2;
  size_t nc = (size_t)h * rows;
  double *c = (double *)malloc(sizeof(double) * 2 * nc);
  if (!c) return -2;
  memcpy(c, in, sizeof(double) * 2 * nc);
  fft_yz(c, h, n1, n2, +1);
  double scale = 1.0 / ((double)n0 * (double)n1 * (double)n2);
  orc_plan px;
  plan_init(&px, n0);
  int nt = orc_get_threads();
  (void)nt;
#pragma omp parallel num_threads(nt)
  {
    double *line = (double *)malloc(sizeof(double) * 2 * (size_t)n0);
    double *work = (double *)malloc(sizeof(double) * 2 * (size_t)n0);
#pragma omp for schedule(static)
    for (long rp = 0; rp < (rows + 1) / 2; ++rp) {
      long ra = 2 * rp, rb = 2 * rp + 1;
      int two = rb < rows;
      const double *A = c + 2 * (size_t)ra * h;
      const double *B = two ? c + 2 * (size_t)rb * h : NULL;
      for (int k = 0; k < n0; ++k) {
        double ar, ai, br = 0, bi = 0;
        if (k < h) {
          ar = A[2 * k]; ai = A[2 * k + 1];
          if (two) { br = B[2 * k]; bi = B[2 * k + 1]; }
        } else {
          int m = n0 - k;
          ar = A[2 * m]; ai = -A[2 * m + 1];
          if (two) { br = B[2 * m]; bi = -B[2 * m + 1]; }
        }
        /* C2R ignores the imaginary parts of the DC and Nyquist bins */
        if (k == 0 || 2 * k == n0) { ai = 0; bi = 0; }
        /* Z = A + i B */
        line[2 * k] = ar - bi;
        line[2 * k + 1] = ai + br;
      }
      fft1d(&px, line, work, +1);
      double *oa = out + (size_t)ra * n0;
      double *ob = two ? out + (size_t)rb * n0 : NULL;
      for (int i = 0; i < n0; ++i) {
        oa[i] = line[2 * i] * scale;
        if (two) ob[i] = line[2 * i + 1] * scale;
      }
    }
    free(line);
    free(work);
  }
  plan_free(&px);
  free(c);
  return 0;
}

/* ------------------------------------------------------------------------- */
/* Operator tables.                                                           */
/* ------------------------------------------------------------------------- */

/* include/openpfc/kernel/fft/kspace.hpp:165-167 */
static double k_component(int i, int n, double f) {
  return (i <= n / 2) ? i * f : (i - n) * f;
}

/* docs/api/examples/10_complete_pfc_model.cpp:166-213 (plain conserved PFC).
 * opL = exp(L dt); opN = (opL-1)/L * (-k^2), or dt*(-k^2) when |L| <= 1e-14. */
void orc_ops_plain(const int n[3], const double dx[3], double r, double dt,
                   double *opL, double *opN) {
  double fx = 2.0 * ORC_PI / (dx[0] * n[0]);
  double fy = 2.0 * ORC_PI / (dx[1] * n[1]);
  double fz = 2.0 * ORC_PI / (dx[2] * n[2]);
  int h = n[0] / 2 + 1;
  size_t idx = 0;
  for (int k = 0; k < n[2]; ++k)
    for (int j = 0; j < n[1]; ++j)
      for (int i = 0; i < h; ++i) {
        double kx = k_component(i, n[0], fx);
        double ky = k_component(j, n[1], fy);
        double kz = k_component(k, n[2], fz);
        double k2 = kx * kx + ky * ky + kz * kz;
        double k2_lap = -k2;
        double L = k2_lap * (r + (1.0 - k2) * (1.0 - k2));
        double eL = exp(L * dt);
        opL[idx] = eL;
        opN[idx] = (fabs(L) > 1e-14) ? (eL - 1.0) / L * k2_lap : dt * k2_lap;
        ++idx;
      }
}

/* Gaussian mean-field filter chi = exp(-k^2 / (2 alpha^2)). */
void orc_filter_gauss(const int n[3], const double dx[3], double alpha,
                      double *chi) {
  double fx = 2.0 * ORC_PI / (dx[0] * n[0]);
  double fy = 2.0 * ORC_PI / (dx[1] * n[1]);
  double fz = 2.0 * ORC_PI / (dx[2] * n[2]);
  int h = n[0] / 2 + 1;
  size_t idx = 0;
  for (int k = 0; k < n[2]; ++k)
    for (int j = 0; j < n[1]; ++j)
      for (int i = 0; i < h; ++i) {
        double kx = k_component(i, n[0], fx);
        double ky = k_component(j, n[1], fy);
        double kz = k_component(k, n[2], fz);
        double k2 = kx * kx + ky * ky + kz * kz;
        chi[idx++] = exp(-k2 / (2.0 * alpha * alpha));
      }
}

/* Tungsten parameters, base values (apps/tungsten/include/tungsten/common/
 * tungsten_params.hpp:33-57). */
typedef struct {
  double n0, n_sol, n_vap, T, T0, Bx, alpha, alpha_farTol;
  int alpha_highOrd;
  double lambda, stabP, shift_u, shift_s, p2, p3, p4, q20, q21, q30, q31, q40;
} orc_tungsten_params;

/* Derived coefficients, tungsten_params.hpp:339-411. */
typedef struct {
  double tau, p2b, p3b, p4b, q20b, q21b, q30b, q31b, q40b, q2b, q3b, q4b;
} orc_tungsten_derived;

void orc_tungsten_derive(const orc_tungsten_params *p, orc_tungsten_derived *d) {
  d->tau = p->T / p->T0;
  d->p2b = p->p2 + 2 * p->shift_s * p->p3 + 3 * pow(p->shift_s, 2) * p->p4;
  d->p3b = p->shift_u * (p->p3 + 3 * p->shift_s * p->p4);
  d->p4b = pow(p->shift_u, 2) * p->p4;
  d->q20b = p->q20 + 2.0 * p->shift_s * p->q30 + 3.0 * pow(p->shift_s, 2) * p->q40;
  d->q21b = p->q21 + 2.0 * p->shift_s * p->q31;
  d->q30b = p->shift_u * (p->q30 + 3.0 * p->shift_s * p->q40);
  d->q31b = p->shift_u * p->q31;
  d->q40b = pow(p->shift_u, 2) * p->q40;
  d->q2b = d->q21b * d->tau + d->q20b;
  d->q3b = d->q31b * d->tau + d->q30b;
  d->q4b = d->q40b;
}

/* Mean-field filter and linear peak symbol for one mode
 * (apps/tungsten/include/tungsten/common/tungsten_spectral.hpp:83-104). */
static void tungsten_mode(double kLap, const orc_tungsten_params *p,
                          const orc_tungsten_derived *d, double *fMF_out,
                          double *opCk_out) {
  double alpha2 = 2.0 * p->alpha * p->alpha;
  double lambda2 = 2.0 * p->lambda * p->lambda;
  double fMF = exp(kLap / lambda2);
  double k_val = sqrt(-kLap) - 1.0;
  double k2 = k_val * k_val;
  double rTol = -alpha2 * log(p->alpha_farTol) - 1.0;
  double g1;
  if (p->alpha_highOrd == 0)
    g1 = exp(-k2 / alpha2);
  else
    g1 = exp(-(k2 + rTol * pow(k_val, p->alpha_highOrd)) / alpha2);
  double g2 = 1.0 - 1.0 / alpha2 * k2;
  double gf = (k_val < 0.0) ? g1 : g2;
  double opPeak = p->Bx * exp(-p->T / p->T0) * gf;
  *fMF_out = fMF;
  *opCk_out = p->stabP + d->p2b - opPeak + d->q2b * fMF;
}

/* ETD coefficients (include/openpfc/kernel/integrator/
 * spectral_exp_coefficients.hpp:68-82) and the Tungsten weight n_weight =
 * kLap * phi1 (apps/tungsten/include/tungsten/common/
 * tungsten_etd_workspace.hpp:111-130). */
void orc_ops_tungsten(const int n[3], const double dx[3],
                      const orc_tungsten_params *p, double dt, double *filterMF,
                      double *expL, double *nweight, double *kLap_out,
                      double *opCk_out) {
  orc_tungsten_derived d;
  orc_tungsten_derive(p, &d);
  double fx = 2.0 * ORC_PI / (dx[0] * n[0]);
  double fy = 2.0 * ORC_PI / (dx[1] * n[1]);
  double fz = 2.0 * ORC_PI / (dx[2] * n[2]);
  int h = n[0] / 2 + 1;
  size_t idx = 0;
  for (int k = 0; k < n[2]; ++k)
    for (int j = 0; j < n[1]; ++j)
      for (int i = 0; i < h; ++i) {
        double ki = k_component(i, n[0], fx);
        double kj = k_component(j, n[1], fy);
        double kk = k_component(k, n[2], fz);
        double kLap = -((ki * ki) + (kj * kj) + (kk * kk));
        double fMF, opCk;
        tungsten_mode(kLap, p, &d, &fMF, &opCk);
        double L = kLap * opCk;
        double arg = L * dt;
        double e = exp(arg);
        double phi1 = (fabs(L) < 1e-12) ? dt + 0.5 * L * dt * dt : expm1(arg) / L;
        filterMF[idx] = fMF;
        expL[idx] = e;
        nweight[idx] = kLap * phi1;
        if (kLap_out) kLap_out[idx] = kLap;
        if (opCk_out) opCk_out[idx] = opCk;
        ++idx;
      }
}

/* Scalar form of spectral_exp_coeffs (spectral_exp_coefficients.hpp:68-82). */
void orc_spectral_exp(double L, double dt, double thr, double *exp_Ldt, double *phi1) {
  double arg = L * dt;
  *exp_Ldt = exp(arg);
  *phi1 = (fabs(L) < thr) ? dt + 0.5 * L * dt * dt : expm1(arg) / L;
}

/* ------------------------------------------------------------------------- */
/* Time steps.                                                                */
/* ------------------------------------------------------------------------- */

static double sumsq(const double *a, size_t n) {
  double s = 0;
  for (size_t i = 0; i < n; ++i) s += a[i] * a[i];
  return s;
}

/* Plain conserved PFC, docs/api/examples/10_complete_pfc_model.cpp:121-144:
 * psi_F = F[psi]; N = psi^3; N_F = F[N]; psi_F = opL psi_F + opN N_F;
 * psi = F^-1[psi_F].  norms (optional) receives sum(psi^2) after each step. */
int orc_run_plain(const int n[3], const double dx[3], double r, double dt,
                  double *psi, int nsteps, double *norms) {
  size_t nr = (size_t)n[0] * n[1] * n[2];
  size_t nc = (size_t)(n[0] / 2 + 1) * n[1] * n[2];
  double *opL = malloc(sizeof(double) * nc), *opN = malloc(sizeof(double) * nc);
  double *pF = malloc(sizeof(double) * 2 * nc), *NF = malloc(sizeof(double) * 2 * nc);
  double *Nr = malloc(sizeof(double) * nr);
  if (!opL || !opN || !pF || !NF || !Nr) return -2;
  orc_ops_plain(n, dx, r, dt, opL, opN);
  for (int s = 0; s < nsteps; ++s) {
    orc_r2c(n[0], n[1], n[2], psi, pF);
    for (size_t i = 0; i < nr; ++i) Nr[i] = psi[i] * psi[i] * psi[i];
    orc_r2c(n[0], n[1], n[2], Nr, NF);
    for (size_t i = 0; i < nc; ++i) {
      pF[2 * i] = opL[i] * pF[2 * i] + opN[i] * NF[2 * i];
      pF[2 * i + 1] = opL[i] * pF[2 * i + 1] + opN[i] * NF[2 * i + 1];
    }
    orc_c2r(n[0], n[1], n[2], pF, psi);
    if (norms) norms[s] = sumsq(psi, nr);
  }
  free(opL); free(opN); free(pF); free(NF); free(Nr);
  return 0;
}

/* Timed plain steps for the CPU baseline: tables are built first (untimed),
 * then `nsteps` steps of orc_run_plain's loop body are timed with the OpenMP
 * wall clock.  Returns seconds, or a negative value on allocation failure. */
double orc_time_plain(const int n[3], const double dx[3], double r, double dt,
                      double *psi, int nsteps) {
  size_t nr = (size_t)n[0] * n[1] * n[2];
  size_t nc = (size_t)(n[0] / 2 + 1) * n[1] * n[2];
  double *opL = malloc(sizeof(double) * nc), *opN = malloc(sizeof(double) * nc);
  double *pF = malloc(sizeof(double) * 2 * nc), *NF = malloc(sizeof(double) * 2 * nc);
  double *Nr = malloc(sizeof(double) * nr);
  if (!opL || !opN || !pF || !NF || !Nr) return -1.0;
  orc_ops_plain(n, dx, r, dt, opL, opN);
#ifdef _OPENMP
  double t0 = omp_get_wtime();
#else
  double t0 = 0;
#endif
  for (int s = 0; s < nsteps; ++s) {
    orc_r2c(n[0], n[1], n[2], psi, pF);
#pragma omp parallel for num_threads(orc_get_threads()) schedule(static)
    for (long i = 0; i < (long)nr; ++i) Nr[i] = psi[i] * psi[i] * psi[i];
    orc_r2c(n[0], n[1], n[2], Nr, NF);
#pragma omp parallel for num_threads(orc_get_threads()) schedule(static)
    for (long i = 0; i < (long)nc; ++i) {
      pF[2 * i] = opL[i] * pF[2 * i] + opN[i] * NF[2 * i];
      pF[2 * i + 1] = opL[i] * pF[2 * i + 1] + opN[i] * NF[2 * i + 1];
    }
    orc_c2r(n[0], n[1], n[2], pF, psi);
  }
#ifdef _OPENMP
  double t1 = omp_get_wtime();
#else
  double t1 = 0;
#endif
  free(opL); free(opN); free(pF); free(NF); free(Nr);
  return t1 - t0;
}

/* Tungsten step, apps/tungsten/include/tungsten/cpu/tungsten_model.hpp:306-366. */
int orc_run_tungsten(const int n[3], const double dx[3],
                     const orc_tungsten_params *p, double dt, double *psi,
                     int nsteps, double *norms) {
  size_t nr = (size_t)n[0] * n[1] * n[2];
  size_t nc = (size_t)(n[0] / 2 + 1) * n[1] * n[2];
  orc_tungsten_derived d;
  orc_tungsten_derive(p, &d);
  double *fMF = malloc(sizeof(double) * nc), *eL = malloc(sizeof(double) * nc);
  double *nw = malloc(sizeof(double) * nc);
  double *pF = malloc(sizeof(double) * 2 * nc), *mF = malloc(sizeof(double) * 2 * nc);
  double *NF = malloc(sizeof(double) * 2 * nc);
  double *pMF = malloc(sizeof(double) * nr), *Nr = malloc(sizeof(double) * nr);
  if (!fMF || !eL || !nw || !pF || !mF || !NF || !pMF || !Nr) return -2;
  orc_ops_tungsten(n, dx, p, dt, fMF, eL, nw, NULL, NULL);
  for (int s = 0; s < nsteps; ++s) {
    orc_r2c(n[0], n[1], n[2], psi, pF);
    for (size_t i = 0; i < nc; ++i) {
      mF[2 * i] = fMF[i] * pF[2 * i];
      mF[2 * i + 1] = fMF[i] * pF[2 * i + 1];
    }
    orc_c2r(n[0], n[1], n[2], mF, pMF);
    for (size_t i = 0; i < nr; ++i) {
      double u = psi[i], v = pMF[i];
      double u2 = u * u, u3 = u * u * u, v2 = v * v, v3 = v * v * v;
      Nr[i] = d.p3b * u2 + d.p4b * u3 + d.q3b * v2 + d.q4b * v3;
    }
    if (p->stabP != 0.0)
      for (size_t i = 0; i < nr; ++i) Nr[i] = Nr[i] - p->stabP * psi[i];
    orc_r2c(n[0], n[1], n[2], Nr, NF);
    for (size_t i = 0; i < nc; ++i) {
      pF[2 * i] = eL[i] * pF[2 * i] + nw[i] * NF[2 * i];
      pF[2 * i + 1] = eL[i] * pF[2 * i + 1] + nw[i] * NF[2 * i + 1];
    }
    orc_c2r(n[0], n[1], n[2], pF, psi);
    if (norms) norms[s] = sumsq(psi, nr);
  }
  free(fMF); free(eL); free(nw); free(pF); free(mF); free(NF); free(pMF); free(Nr);
  return 0;
}

/* ------------------------------------------------------------------------- */
/* Aluminum PFC variant, apps/aluminumNew/Aluminum.hpp.                        */
/* ------------------------------------------------------------------------- */

/* Parameter block, names of Aluminum::params (Aluminum.hpp:29-82); the
 * reference test leaves everything it does not set at 0 (T0 at 1). */
typedef struct orc_aluminum_params {
  double n0, n_sol, n_vap, T, T0, Bx, T_const, T_max, T_min, G_grid, V_grid, x_initial, m_xpos, alpha,
      alpha_farTol;
  int alpha_highOrd;
  double tau_const, lambda, stabP, shift_u, shift_s, p2, p3, p4, p2_bar, p3_bar, p4_bar, q20, q21, q30, q31,
      q40, q20_bar, q21_bar, q30_bar, q31_bar, q40_bar, q2_bar, q3_bar, q4_bar, q2_bar_L;
} orc_aluminum_params;

/* Operators per half-spectrum mode, Aluminum.hpp:186-242 (prepare_operators):
 * chi = exp(kLap/(2 lambda^2)); the peak is the larger of the Gaussians around
 * |k| = 1 and |k| = 2/sqrt(3); P_F = Bx exp(-tau_const) peak;
 * opCk = stabP + p2_bar - P_F + q2_bar_L chi; opL = exp(kLap opCk dt);
 * opN = kLap dt if opCk == 0 else (opL - 1)/opCk. */
void orc_ops_aluminum(const int n[3], const double dx[3], const orc_aluminum_params *p, double dt,
                      double *filterMF, double *opL, double *opN, double *P_F) {
  const double fx = 2.0 * ORC_PI / (dx[0] * n[0]);
  const double fy = 2.0 * ORC_PI / (dx[1] * n[1]);
  const double fz = 2.0 * ORC_PI / (dx[2] * n[2]);
  const int h = n[0] / 2 + 1;
  const double alpha2 = 2.0 * p->alpha * p->alpha, lambda2 = 2.0 * p->lambda * p->lambda;
  size_t idx = 0;
  for (int k = 0; k < n[2]; ++k)
    for (int j = 0; j < n[1]; ++j)
      for (int i = 0; i < h; ++i, ++idx) {
        const double ki = k_component(i, n[0], fx), kj = k_component(j, n[1], fy), kk = k_component(k, n[2], fz);
        const double kLap = -(ki * ki + kj * kj + kk * kk);
        const double fMF = exp(kLap / lambda2);
        const double kw = sqrt(-kLap) - 1.0, kp = sqrt(-kLap) - 2.0 / sqrt(3.0);
        const double g1 = exp(-(kw * kw) / alpha2), gp1 = exp(-(kp * kp) / alpha2);
        const double peak = g1 > gp1 ? g1 : gp1;
        const double PF = p->Bx * exp(-p->tau_const) * peak;
        const double opCk = p->stabP + p->p2_bar - PF + p->q2_bar_L * fMF;
        filterMF[idx] = fMF;
        opL[idx] = exp(kLap * opCk * dt);
        opN[idx] = (opCk == 0.0) ? kLap * dt : (opL[idx] - 1.0) / opCk;
        if (P_F) P_F[idx] = PF;
      }
}

/* Aluminum::step(t), Aluminum.hpp:247-326: psi_MF = F^-1[chi psi_F],
 * P*psi = F^-1[P_F psi_F]; with the moving temperature
 * T_var(x, t) = G_grid (dist - x_initial - V_grid t), dist = x + fullruns -
 * (x > steppoint) l, l = N0 dx, fullruns = floor(m_xpos/l) l,
 * steppoint = fmod(m_xpos, l):
 * N = p3_bar u^2 + p4_bar u^3 + q2N v + q3 v^2 + q4_bar v^3 - kernel,
 * q2N = q21_bar T_var/T0, q3 = q31_bar (T_const + T_var)/T0 + q30_bar,
 * kernel = -(1 - exp(-T_var/T0)) P*psi; minus stabP u; psi_F = opL psi_F +
 * opN F[N]; psi = F^-1[psi_F].  Step s uses t = t0 + s dt_t. */
int orc_run_aluminum(const int n[3], const double dx[3], const double origin[3], const orc_aluminum_params *p,
                     double dt, double t0, double dt_t, double *psi, int nsteps, double *norms) {
  const size_t nr = (size_t)n[0] * n[1] * n[2];
  const size_t nc = (size_t)(n[0] / 2 + 1) * n[1] * n[2];
  double *fMF = malloc(sizeof(double) * nc), *oL = malloc(sizeof(double) * nc);
  double *oN = malloc(sizeof(double) * nc), *PF = malloc(sizeof(double) * nc);
  double *pF = malloc(sizeof(double) * 2 * nc), *wF = malloc(sizeof(double) * 2 * nc);
  double *pMF = malloc(sizeof(double) * nr), *Pp = malloc(sizeof(double) * nr), *Nr = malloc(sizeof(double) * nr);
  if (!fMF || !oL || !oN || !PF || !pF || !wF || !pMF || !Pp || !Nr) return -2;
  orc_ops_aluminum(n, dx, p, dt, fMF, oL, oN, PF);
  const double l = n[0] * dx[0];
  const double fullruns = floor(p->m_xpos / l) * l, steppoint = fmod(p->m_xpos, l);
  for (int s = 0; s < nsteps; ++s) {
    const double t = t0 + s * dt_t;
    orc_r2c(n[0], n[1], n[2], psi, pF);
    for (size_t i = 0; i < nc; ++i) {
      wF[2 * i] = fMF[i] * pF[2 * i];
      wF[2 * i + 1] = fMF[i] * pF[2 * i + 1];
    }
    orc_c2r(n[0], n[1], n[2], wF, pMF);
    for (size_t i = 0; i < nc; ++i) {
      wF[2 * i] = PF[i] * pF[2 * i];
      wF[2 * i + 1] = PF[i] * pF[2 * i + 1];
    }
    orc_c2r(n[0], n[1], n[2], wF, Pp);
    for (size_t idx = 0; idx < nr; ++idx) {
      const int i = (int)(idx % (size_t)n[0]);
      const double x = origin[0] + i * dx[0];
      const double dist = x + fullruns - (x > steppoint) * l;
      const double Tv = p->G_grid * (dist - p->x_initial - p->V_grid * t);
      const double q2N = p->q21_bar * Tv / p->T0;
      const double q3 = p->q31_bar * (p->T_const + Tv) / p->T0 + p->q30_bar;
      const double u = psi[idx], v = pMF[idx];
      const double kern = -(1.0 - exp(-Tv / p->T0)) * Pp[idx];
      Nr[idx] = p->p3_bar * u * u + p->p4_bar * u * u * u + q2N * v + q3 * v * v + p->q4_bar * v * v * v - kern;
    }
    if (p->stabP != 0.0)
      for (size_t i = 0; i < nr; ++i) Nr[i] = Nr[i] - p->stabP * psi[i];
    orc_r2c(n[0], n[1], n[2], Nr, wF);
    for (size_t i = 0; i < nc; ++i) {
      pF[2 * i] = oL[i] * pF[2 * i] + oN[i] * wF[2 * i];
      pF[2 * i + 1] = oL[i] * pF[2 * i + 1] + oN[i] * wF[2 * i + 1];
    }
    orc_c2r(n[0], n[1], n[2], pF, psi);
    if (norms) norms[s] = sumsq(psi, nr);
  }
  free(fMF); free(oL); free(oN); free(PF); free(pF); free(wF); free(pMF); free(Pp); free(Nr);
  return 0;
}

/* Mean-field-filtered PFC with a polynomial of the filtered density:
 * psi_MF = F^-1[chi F[psi]], chi = exp(-k^2/(2 alpha^2));
 * N = p2 psi_MF^2/2 + p3 psi_MF^3/3 + p4 psi_MF^4/4;
 * psi_F = opL psi_F + opN F[N] with the plain-PFC opL/opN at r. */
int orc_run_filtered(const int n[3], const double dx[3], double r, double alpha,
                     double p2, double p3, double p4, double dt, double *psi,
                     int nsteps, double *norms) {
  size_t nr = (size_t)n[0] * n[1] * n[2];
  size_t nc = (size_t)(n[0] / 2 + 1) * n[1] * n[2];
  double *opL = malloc(sizeof(double) * nc), *opN = malloc(sizeof(double) * nc);
  double *chi = malloc(sizeof(double) * nc);
  double *pF = malloc(sizeof(double) * 2 * nc), *mF = malloc(sizeof(double) * 2 * nc);
  double *NF = malloc(sizeof(double) * 2 * nc);
  double *pMF = malloc(sizeof(double) * nr), *Nr = malloc(sizeof(double) * nr);
  if (!opL || !opN || !chi || !pF || !mF || !NF || !pMF || !Nr) return -2;
  orc_ops_plain(n, dx, r, dt, opL, opN);
  orc_filter_gauss(n, dx, alpha, chi);
  for (int s = 0; s < nsteps; ++s) {
    orc_r2c(n[0], n[1], n[2], psi, pF);
    for (size_t i = 0; i < nc; ++i) {
      mF[2 * i] = chi[i] * pF[2 * i];
      mF[2 * i + 1] = chi[i] * pF[2 * i + 1];
    }
    orc_c2r(n[0], n[1], n[2], mF, pMF);
    for (size_t i = 0; i < nr; ++i) {
      double v = pMF[i], v2 = v * v;
      Nr[i] = p2 * v2 / 2.0 + p3 * v2 * v / 3.0 + p4 * v2 * v2 / 4.0;
    }
    orc_r2c(n[0], n[1], n[2], Nr, NF);
    for (size_t i = 0; i < nc; ++i) {
      pF[2 * i] = opL[i] * pF[2 * i] + opN[i] * NF[2 * i];
      pF[2 * i + 1] = opL[i] * pF[2 * i + 1] + opN[i] * NF[2 * i + 1];
    }
    orc_c2r(n[0], n[1], n[2], pF, psi);
    if (norms) norms[s] = sumsq(psi, nr);
  }
  free(opL); free(opN); free(chi); free(pF); free(mF); free(NF); free(pMF); free(Nr);
  return 0;
}

/* ------------------------------------------------------------------------- */
/* Diagnostics.                                                               */
/* ------------------------------------------------------------------------- */

/* Neumaier-compensated sum. */
double orc_sum(const double *a, size_t n) {
  double s = 0, c = 0;
  for (size_t i = 0; i < n; ++i) {
    double t = s + a[i];
    if (fabs(s) >= fabs(a[i]))
      c += (s - t) + a[i];
    else
      c += (a[i] - t) + s;
    s = t;
  }
  return s + c;
}

/* Free energy of the plain PFC (project-defined; the reference computes none):
 * F = sum_cells dV [ 1/2 psi F^-1{(r + (1-k^2)^2) psi_hat} + 1/4 psi^4 ]. */
double orc_free_energy_plain(const int n[3], const double dx[3], double r,
                             const double *psi) {
  size_t nr = (size_t)n[0] * n[1] * n[2];
  size_t nc = (size_t)(n[0] / 2 + 1) * n[1] * n[2];
  double *pF = malloc(sizeof(double) * 2 * nc);
  double *g = malloc(sizeof(double) * nr);
  double *terms = malloc(sizeof(double) * nr);
  orc_r2c(n[0], n[1], n[2], psi, pF);
  double fx = 2.0 * ORC_PI / (dx[0] * n[0]);
  double fy = 2.0 * ORC_PI / (dx[1] * n[1]);
  double fz = 2.0 * ORC_PI / (dx[2] * n[2]);
  int h = n[0] / 2 + 1;
  size_t idx = 0;
  for (int k = 0; k < n[2]; ++k)
    for (int j = 0; j < n[1]; ++j)
      for (int i = 0; i < h; ++i) {
        double kx = k_component(i, n[0], fx);
        double ky = k_component(j, n[1], fy);
        double kz = k_component(k, n[2], fz);
        double k2 = kx * kx + ky * ky + kz * kz;
        double G = r + (1.0 - k2) * (1.0 - k2);
        pF[2 * idx] *= G;
        pF[2 * idx + 1] *= G;
        ++idx;
      }
  orc_c2r(n[0], n[1], n[2], pF, g);
  double dV = dx[0] * dx[1] * dx[2];
  for (size_t i = 0; i < nr; ++i) {
    double p = psi[i];
    terms[i] = dV * (0.5 * p * g[i] + 0.25 * p * p * p * p);
  }
  double F = orc_sum(terms, nr);
  free(pF); free(g); free(terms);
  return F;
}

/* ------------------------------------------------------------------------- */
/* Initial conditions.                                                        */
/* ------------------------------------------------------------------------- */

/* MT19937-64 (Matsumoto & Nishimura 2000; the engine std::mt19937_64 names). */
typedef struct { uint64_t mt[312]; int mti; } orc_mt64;

void orc_mt64_seed(orc_mt64 *g, uint64_t seed) {
  g->mt[0] = seed;
  for (int i = 1; i < 312; ++i)
    g->mt[i] = 6364136223846793005ULL * (g->mt[i - 1] ^ (g->mt[i - 1] >> 62)) + (uint64_t)i;
  g->mti = 312;
}

uint64_t orc_mt64_next(orc_mt64 *g) {
  static const uint64_t UM = 0xFFFFFFFF80000000ULL, LM = 0x7FFFFFFFULL;
  static const uint64_t MAG[2] = {0ULL, 0xB5026F5AA96619E9ULL};
  if (g->mti >= 312) {
    int i;
    for (i = 0; i < 312 - 156; ++i) {
      uint64_t x = (g->mt[i] & UM) | (g->mt[i + 1] & LM);
      g->mt[i] = g->mt[i + 156] ^ (x >> 1) ^ MAG[(int)(x & 1ULL)];
    }
    for (; i < 311; ++i) {
      uint64_t x = (g->mt[i] & UM) | (g->mt[i + 1] & LM);
      g->mt[i] = g->mt[i + (156 - 312)] ^ (x >> 1) ^ MAG[(int)(x & 1ULL)];
    }
    uint64_t x = (g->mt[311] & UM) | (g->mt[0] & LM);
    g->mt[311] = g->mt[155] ^ (x >> 1) ^ MAG[(int)(x & 1ULL)];
    g->mti = 0;
  }
  uint64_t x = g->mt[g->mti++];
  x ^= (x >> 29) & 0x5555555555555555ULL;
  x ^= (x << 17) & 0x71D67FFFEDA60000ULL;
  x ^= (x << 37) & 0xFFF7EEE000000000ULL;
  x ^= (x >> 43);
  return x;
}

/* u in [0,1): top 53 bits of one 64-bit draw. */
static double mt_unit(orc_mt64 *g) {
  return (double)(orc_mt64_next(g) >> 11) * (1.0 / 9007199254740992.0);
}

/* psi = n0 + U(-amp, amp) per cell in x-fastest order, one draw per cell. */
void orc_ic_noise(size_t ncell, double n0, double amp, uint64_t seed, double *psi) {
  orc_mt64 g;
  orc_mt64_seed(&g, seed);
  for (size_t i = 0; i < ncell; ++i) psi[i] = n0 + (-amp + 2.0 * amp * mt_unit(&g));
}

/* Single seed exactly as the Tungsten regression test fills it
 * (apps/tungsten/tests/test_tungsten.cpp:231-280): cells with |x|^2 < R^2 get
 * rho + sum_q 2 amp cos(q.x); other cells keep their value. */
void orc_ic_seed_inside(const int n[3], const double dx[3], const double origin[3],
                        double radius, double rho, double amp, double *psi) {
  const double s = 1.0 / sqrt(2.0);
  const double q[6][3] = {{s, s, 0}, {s, 0, s}, {0, s, s},
                          {s, 0, -s}, {s, -s, 0}, {0, s, -s}};
  double r2 = pow(radius, 2);
  size_t idx = 0;
  for (int k = 0; k < n[2]; ++k)
    for (int j = 0; j < n[1]; ++j)
      for (int i = 0; i < n[0]; ++i) {
        double x = origin[0] + i * dx[0];
        double y = origin[1] + j * dx[1];
        double z = origin[2] + k * dx[2];
        if (x * x + y * y + z * z < r2) {
          double u = rho;
          for (int qi = 0; qi < 6; ++qi)
            u += 2.0 * amp * cos(q[qi][0] * x + q[qi][1] * y + q[qi][2] * z);
          psi[idx] = u;
        }
        ++idx;
      }
}

/* Seeded spheres on a noisy liquid: psi = n0 + U(-noise, noise) (one draw per
 * cell, x-fastest), then `nseeds` centres drawn from the same generator as
 * (u0*N0, u1*N1, u2*N2) in cell units; cells within `radius_cells` (periodic
 * minimum-image distance) of a centre get n0 + amp * sum_q cos(q.(x - c)) with
 * the six <110>/sqrt(2) vectors of single_seed.hpp and x in physical units. */
void orc_ic_seeds(const int n[3], const double dx[3], double n0, double noise,
                  int nseeds, double radius_cells, double amp, uint64_t seed,
                  double *psi) {
  size_t ncell = (size_t)n[0] * n[1] * n[2];
  orc_mt64 g;
  orc_mt64_seed(&g, seed);
  for (size_t i = 0; i < ncell; ++i) psi[i] = n0 + (-noise + 2.0 * noise * mt_unit(&g));
  const double s = 1.0 / sqrt(2.0);
  const double q[6][3] = {{s, s, 0}, {s, 0, s}, {0, s, s},
                          {s, 0, -s}, {s, -s, 0}, {0, s, -s}};
  for (int sd = 0; sd < nseeds; ++sd) {
    double c[3];
    for (int a = 0; a < 3; ++a) c[a] = mt_unit(&g) * n[a];
    double R2 = radius_cells * radius_cells;
    size_t idx = 0;
    for (int k = 0; k < n[2]; ++k)
      for (int j = 0; j < n[1]; ++j)
        for (int i = 0; i < n[0]; ++i, ++idx) {
          double d[3] = {i - c[0], j - c[1], k - c[2]};
          for (int a = 0; a < 3; ++a) {
            if (d[a] > 0.5 * n[a]) d[a] -= n[a];
            if (d[a] < -0.5 * n[a]) d[a] += n[a];
          }
          if (d[0] * d[0] + d[1] * d[1] + d[2] * d[2] >= R2) continue;
          double X = d[0] * dx[0], Y = d[1] * dx[1], Z = d[2] * dx[2];
          double u = n0;
          for (int qi = 0; qi < 6; ++qi) u += amp * cos(q[qi][0] * X + q[qi][1] * Y + q[qi][2] * Z);
          psi[idx] = u;
        }
  }
}
