/*
 * CPU restatement of the reference's covariance generator, used as the timed CPU
 * baseline (TEST INFRASTRUCTURE ONLY: never linked into the product).
 *
 * Follows UnivariateMaternStationary<T>::GenerateCovarianceMatrix
 * (src/kernels/concrete/UnivariateMaternStationary.cpp:39-67): for every lower
 * element, dist = sqrt(dx^2 + dy^2) / beta (DistanceCalculationHelpers.cpp:38-57),
 * C = sigma2 if dist == 0 else con * dist^nu * K_nu(dist) with
 * con = sigma2 / (2^(nu-1) Gamma(nu)).  The reference's K_nu is GSL 2.7.1's
 * gsl_sf_bessel_Knu (not in the reference tree); it is restated here from the
 * published method it uses: Temme's series for x <= 2 (N. M. Temme, J. Comput.
 * Phys. 19 (1975) 324-337) and Steed's CF2 for x > 2 (Thompson & Barnett,
 * J. Comput. Phys. 64 (1986) 490-509), with upward recurrence in nu.
 * The reference runs one StarPU task per tile on all CPU workers; here POSIX
 * threads take the columns cyclically over all online host cores.
 *
 * Build: make -C oracle   (-> oracle/_build/libegs_oracle.so)
 */
#include <math.h>
#include <stdint.h>
#include <pthread.h>
#include <unistd.h>

/* Taylor coefficients of 1/Gamma(1+z) at 0 (mathematical constants, 20 digits). */
static const double rg[24] = {
    1.0,
    5.77215664901532860607e-1,
    -6.55878071520253881077e-1,
    -4.2002635034095235529e-2,
    1.66538611382291489502e-1,
    -4.21977345555443367482e-2,
    -9.62197152787697356211e-3,
    7.2189432466630995424e-3,
    -1.16516759185906511211e-3,
    -2.15241674114950972816e-4,
    1.28050282388116186153e-4,
    -2.01348547807882386557e-5,
    -1.25049348214267065735e-6,
    1.13302723198169588237e-6,
    -2.05633841697760710345e-7,
    6.11609510448141581786e-9,
    5.00200764446922293006e-9,
    -1.18127457048702014459e-9,
    1.04342671169110051049e-10,
    7.78226343990507125405e-12,
    -3.69680561864220570819e-12,
    5.10037028745447597902e-13,
    -2.05832605356650678322e-14,
    -5.34812253942301798237e-15};

static void temme_gam(double mu, double* g1, double* g2) {
  double m2 = mu * mu, ev = 0.0, od = 0.0;
  for (int k = 22; k >= 0; k -= 2) {
    ev = ev * m2 + rg[k];
    od = od * m2 + rg[k + 1];
  }
  *g2 = ev;
  *g1 = -od;
}

static void k_series(double mu, double x, double* kmu, double* kmu1) {
  double hx = 0.5 * x, l2x = -log(hx), sg = mu * l2x, g1, g2;
  temme_gam(mu, &g1, &g2);
  double gp = g2 - mu * g1, gm = g2 + mu * g1;
  double fct = fabs(mu) < 1e-15 ? 1.0 : (mu * M_PI) / sin(mu * M_PI);
  double shs = fabs(sg) < 1e-4 ? 1.0 + sg * sg / 6.0 : sinh(sg) / sg;
  double es = exp(sg);
  double f = fct * (g1 * cosh(sg) + g2 * shs * l2x);
  double p = 0.5 * es / gp, q = 0.5 / (es * gm), c = 1.0, d = hx * hx;
  double s0 = f, s1 = p;
  for (int k = 1; k < 200; ++k) {
    f = (k * f + p + q) / ((double)k * k - mu * mu);
    c *= d / k;
    p /= (k - mu);
    q /= (k + mu);
    double t = c * f;
    s0 += t;
    s1 += c * (p - k * f);
    if (fabs(t) < 1e-17 * fabs(s0)) break;
  }
  *kmu = s0;
  *kmu1 = s1 * 2.0 / x;
}

/* e^x K_mu(x), e^x K_{mu+1}(x) for x > 2 */
static void k_cf2(double mu, double x, double* kmu, double* kmu1) {
  double a1 = 0.25 - mu * mu, b = 2.0 * (1.0 + x), dd = 1.0 / b, dh = dd, h = dd;
  double q0 = 0.0, q1 = 1.0, a = -a1, c = a1, qs = a1, s = 1.0 + qs * dh;
  for (int i = 2; i < 2000; ++i) {
    a -= 2.0 * (i - 1);
    c = -a * c / i;
    double qn = (q0 - b * q1) / a;
    q0 = q1;
    q1 = qn;
    qs += c * qn;
    b += 2.0;
    dd = 1.0 / (b + a * dd);
    dh = (b * dd - 1.0) * dh;
    h += dh;
    double ds = qs * dh;
    s += ds;
    if (fabs(ds) < 1e-17 * fabs(s)) break;
  }
  h *= a1;
  *kmu = sqrt(M_PI / (2.0 * x)) / s;
  *kmu1 = *kmu * (mu + x + 0.5 - h) / x;
}

static double matern(double x, double sigma2, double nu, double con) {
  if (x == 0.0) return sigma2;
  int n = (int)floor(nu + 0.5);
  double mu = nu - n, k0, k1, knu;
  int scaled = x > 2.0;
  if (scaled) k_cf2(mu, x, &k0, &k1); else k_series(mu, x, &k0, &k1);
  if (n == 0) {
    knu = k0;
  } else {
    double v = mu + 1.0;
    for (int j = 1; j < n; ++j) {
      double k2 = k0 + (2.0 * v / x) * k1;
      k0 = k1;
      k1 = k2;
      v += 1.0;
    }
    knu = k1;
  }
  return scaled ? con * exp(nu * log(x) - x) * knu : con * pow(x, nu) * knu;
}

int egs_oracle_max_threads(void);

struct job {
  double* a;
  long lda;
  int m, n, t, nthreads, lower;
  const double *x, *y, *x2, *y2;
  double sigma2, beta, nu, con;
};

/* Column j of the job: rows j..m-1 (lower triangle of a square matrix) or
 * rows 0..m-1 (a block between two location sets); entry (i, j) pairs row
 * location i of (x, y) with column location j of (x2, y2). */
static void* worker(void* arg) {
  struct job* jb = (struct job*)arg;
  for (int j = jb->t; j < jb->n; j += jb->nthreads) {
    for (int i = jb->lower ? j : 0; i < jb->m; ++i) {
      double dx = jb->x2[j] - jb->x[i], dy = jb->y2[j] - jb->y[i];
      double dist = sqrt(dx * dx + dy * dy) / jb->beta;
      jb->a[i + (long)j * jb->lda] = matern(dist, jb->sigma2, jb->nu, jb->con);
    }
  }
  return 0;
}

static void run_jobs(double* a, long lda, int m, int n, int lower, const double* x, const double* y,
                     const double* x2, const double* y2, const double* theta, int nthreads) {
  if (nthreads <= 0) nthreads = egs_oracle_max_threads();
  if (nthreads > 1024) nthreads = 1024;
  const double sigma2 = theta[0], beta = theta[1], nu = theta[2];
  const double con = sigma2 * (1.0 / (pow(2.0, nu - 1.0) * tgamma(nu)));
  pthread_t tid[1024];
  struct job jobs[1024];
  for (int t = 0; t < nthreads; ++t) {
    jobs[t] = (struct job){a, lda, m, n, t, nthreads, lower, x, y, x2, y2, sigma2, beta, nu, con};
    pthread_create(&tid[t], 0, worker, &jobs[t]);
  }
  for (int t = 0; t < nthreads; ++t) pthread_join(tid[t], 0);
}

int egs_oracle_max_threads(void) {
  long c = sysconf(_SC_NPROCESSORS_ONLN);
  return c > 0 ? (int)c : 1;
}

/* Lower triangle (i >= j) of the n x n Matern matrix, column-major with leading
 * dimension lda; the strictly upper part is left untouched.  nthreads <= 0 uses
 * every online core. */
void egs_oracle_matern_lower(double* a, long lda, int n, const double* x, const double* y, const double* theta,
                             int nthreads) {
  run_jobs(a, lda, n, n, 1, x, y, x, y, theta, nthreads);
}

/* The m x n Matern block between row locations (x1, y1) and column locations
 * (x2, y2), column-major with leading dimension lda (the C12 of the kriging,
 * LinearAlgebraMethods.cpp:535). */
void egs_oracle_matern_block(double* a, long lda, int m, int n, const double* x1, const double* y1,
                             const double* x2, const double* y2, const double* theta, int nthreads) {
  run_jobs(a, lda, m, n, 0, x1, y1, x2, y2, theta, nthreads);
}
