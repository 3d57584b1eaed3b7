// Bound-constrained derivative-free maximiser for the MLE driver.
//
// Replaces the NLopt 2.7.1 LN_BOBYQA optimiser that
// StarpuRuntimeSolver<T>::ModelingOperations (src/runtime-solver/concrete/
// StarpuRuntimeSolver.cpp:28-66) runs with box bounds, ftol_abs and maxeval,
// maximising the log-likelihood and returning the best value found
// (last_optimum_value, :64) with theta written back into the start vector (:48).
// NLopt is not part of the reference tree; this is written from M. J. D. Powell,
// "The BOBYQA algorithm for bound constrained optimization without derivatives",
// Report DAMTP 2009/NA06:
//
//  * initial points exactly as Powell's PRELIM: x0 (moved onto a bound when it is
//    within rhobeg of it), x0 + rhobeg e_i (-rhobeg at an upper bound), then the
//    second point per coordinate: -rhobeg, or min(2 rhobeg, u_i - x0_i) at a lower
//    bound, or max(-2 rhobeg, l_i - x0_i) at an upper bound -- so the first
//    evaluations are those of NLopt's BOBYQA;
//  * quadratic models by least-Frobenius-norm updating (Powell 2004): each new
//    model interpolates all 2n+1 points and changes the Hessian by the smallest
//    Frobenius norm; for n parameters the (2n+1)+n+1 KKT system is solved directly;
//  * trust-region steps by truncated conjugate gradients that fix variables as
//    they reach their bounds (the role of TRSBOX);
//  * Powell's rho / Delta management and geometry steps that move the farthest
//    interpolation point to where its Lagrange function is largest (ALTMOV's role).
//
// Stopping follows NLopt's semantics used by the reference: maxeval evaluations,
// or an improvement of the best value smaller than ftol_abs, or rho <= rhoend.
#include <algorithm>
#include <cmath>
#include <functional>
#include <limits>
#include <vector>
#include "exageostat_b200.h"

namespace {

using Vec = std::vector<double>;
using Mat = std::vector<Vec>;

// Solve A x = b by Gaussian elimination with partial pivoting; false if singular.
bool solve_dense(Mat a, Vec b, Vec& x) {
  const int m = (int)b.size();
  for (int c = 0; c < m; ++c) {
    int piv = c;
    for (int r = c + 1; r < m; ++r)
      if (std::fabs(a[r][c]) > std::fabs(a[piv][c])) piv = r;
    if (std::fabs(a[piv][c]) < 1e-300) return false;
    std::swap(a[piv], a[c]);
    std::swap(b[piv], b[c]);
    for (int r = c + 1; r < m; ++r) {
      const double f = a[r][c] / a[c][c];
      if (f == 0.0) continue;
      for (int k = c; k < m; ++k) a[r][k] -= f * a[c][k];
      b[r] -= f * b[c];
    }
  }
  x.assign(m, 0.0);
  for (int r = m - 1; r >= 0; --r) {
    double s = b[r];
    for (int k = r + 1; k < m; ++k) s -= a[r][k] * x[k];
    x[r] = s / a[r][r];
  }
  return true;
}

double norm(const Vec& v) {
  double s = 0;
  for (double e : v) s += e * e;
  return std::sqrt(s);
}

struct Optimizer {
  int n, npt;
  Vec lb, ub;
  double rhobeg, rhoend, ftol_abs;
  int maxeval;
  std::function<double(const Vec&)> fmin;  // function to minimise (negated objective)

  Vec x0;      // base point of the model
  Mat Y;       // interpolation points (absolute)
  Vec F;       // their values
  int kopt = 0;
  double c0 = 0;  // model: q(x) = c0 + g.(x-x0) + 1/2 (x-x0)^T H (x-x0)
  Vec g;
  Mat H;
  int nf = 0;
  bool stop = false;
  int status = EGS_OK;

  double eval(const Vec& x) {
    ++nf;
    const double v = fmin(x);
    if (!std::isfinite(v)) return std::numeric_limits<double>::max();
    return v;
  }

  double model(const Vec& x) const {
    double q = c0;
    Vec d(n);
    for (int i = 0; i < n; ++i) d[i] = x[i] - x0[i];
    for (int i = 0; i < n; ++i) {
      q += g[i] * d[i];
      double hd = 0;
      for (int j = 0; j < n; ++j) hd += H[i][j] * d[j];
      q += 0.5 * d[i] * hd;
    }
    return q;
  }

  // KKT matrix of least-Frobenius-norm interpolation for the current points.
  Mat kkt() const {
    const int m = npt + n + 1;
    Mat W(m, Vec(m, 0.0));
    for (int j = 0; j < npt; ++j) {
      for (int k = 0; k < npt; ++k) {
        double dp = 0;
        for (int i = 0; i < n; ++i) dp += (Y[j][i] - x0[i]) * (Y[k][i] - x0[i]);
        W[j][k] = 0.5 * dp * dp;
      }
      W[j][npt] = W[npt][j] = 1.0;
      for (int i = 0; i < n; ++i) W[j][npt + 1 + i] = W[npt + 1 + i][j] = Y[j][i] - x0[i];
    }
    return W;
  }

  // Update the model so that it interpolates every point, changing H least.
  bool update_model() {
    const int m = npt + n + 1;
    Vec rhs(m, 0.0);
    for (int j = 0; j < npt; ++j) rhs[j] = F[j] - model(Y[j]);
    Vec sol;
    if (!solve_dense(kkt(), rhs, sol)) return false;
    for (int j = 0; j < npt; ++j) {
      for (int a = 0; a < n; ++a)
        for (int b = 0; b < n; ++b) H[a][b] += sol[j] * (Y[j][a] - x0[a]) * (Y[j][b] - x0[b]);
    }
    c0 += sol[npt];
    for (int i = 0; i < n; ++i) g[i] += sol[npt + 1 + i];
    return true;
  }

  // Value at x of every Lagrange function of the current interpolation set.
  bool lagrange(const Vec& x, Vec& out) const {
    const int m = npt + n + 1;
    const Mat W = kkt();
    out.assign(npt, 0.0);
    for (int k = 0; k < npt; ++k) {
      Vec e(m, 0.0);
      e[k] = 1.0;
      Vec coef;
      if (!solve_dense(W, e, coef)) return false;
      double v = coef[npt];
      for (int i = 0; i < n; ++i) v += coef[npt + 1 + i] * (x[i] - x0[i]);
      for (int j = 0; j < npt; ++j) {
        double dp = 0;
        for (int i = 0; i < n; ++i) dp += (Y[j][i] - x0[i]) * (x[i] - x0[i]);
        v += coef[j] * 0.5 * dp * dp;
      }
      out[k] = v;
    }
    return true;
  }

  // Truncated conjugate gradients on the model around Y[kopt] within the box and
  // the trust region of radius delta.
  Vec trust_step(double delta) const {
    const Vec& xb = Y[kopt];
    Vec grad(n);
    for (int i = 0; i < n; ++i) {
      double s = g[i];
      for (int j = 0; j < n; ++j) s += H[i][j] * (xb[j] - x0[j]);
      grad[i] = s;
    }
    std::vector<bool> fixed(n, false);
    for (int i = 0; i < n; ++i) {
      if (xb[i] <= lb[i] && grad[i] > 0) fixed[i] = true;
      if (xb[i] >= ub[i] && grad[i] < 0) fixed[i] = true;
    }
    Vec d(n, 0.0);
    for (int restart = 0; restart <= n; ++restart) {
      Vec r(n, 0.0);
      for (int i = 0; i < n; ++i) {
        if (fixed[i]) continue;
        double hd = 0;
        for (int j = 0; j < n; ++j) hd += H[i][j] * d[j];
        r[i] = -(grad[i] + hd);
      }
      Vec s = r;
      double rr = 0;
      for (double v : r) rr += v * v;
      bool hit_bound = false;
      for (int it = 0; it < n && rr > 1e-30; ++it) {
        Vec hs(n, 0.0);
        for (int i = 0; i < n; ++i) {
          if (fixed[i]) continue;
          for (int j = 0; j < n; ++j) hs[i] += H[i][j] * s[j];
        }
        double shs = 0, ds = 0, ss = 0, dd = 0;
        for (int i = 0; i < n; ++i) {
          shs += s[i] * hs[i];
          ds += d[i] * s[i];
          ss += s[i] * s[i];
          dd += d[i] * d[i];
        }
        if (ss <= 0) break;
        const double disc = ds * ds + ss * (delta * delta - dd);
        const double a_tr = (disc > 0) ? (-ds + std::sqrt(disc)) / ss : 0.0;
        double a_bd = std::numeric_limits<double>::max();
        int ibd = -1;
        for (int i = 0; i < n; ++i) {
          if (fixed[i] || s[i] == 0.0) continue;
          const double lim = s[i] > 0 ? (ub[i] - xb[i] - d[i]) / s[i] : (lb[i] - xb[i] - d[i]) / s[i];
          if (lim < a_bd) {
            a_bd = std::max(lim, 0.0);
            ibd = i;
          }
        }
        const double a_cg = shs > 0 ? rr / shs : std::numeric_limits<double>::max();
        const double a = std::min(a_cg, std::min(a_tr, a_bd));
        for (int i = 0; i < n; ++i) d[i] += a * s[i];
        if (a == a_bd && ibd >= 0 && a_bd < std::min(a_cg, a_tr)) {
          fixed[ibd] = true;
          d[ibd] = (s[ibd] > 0 ? ub[ibd] : lb[ibd]) - xb[ibd];
          hit_bound = true;
          break;
        }
        if (a == a_tr && a_tr <= a_cg) return d;
        Vec rn(n);
        double rrn = 0;
        for (int i = 0; i < n; ++i) {
          rn[i] = fixed[i] ? 0.0 : r[i] - a * hs[i];
          rrn += rn[i] * rn[i];
        }
        const double beta = rrn / rr;
        for (int i = 0; i < n; ++i) s[i] = rn[i] + beta * s[i];
        r = rn;
        rr = rrn;
      }
      if (!hit_bound) break;
    }
    return d;
  }

  // Re-express the model around a new base point (Powell moves XBASE towards
  // XOPT so that the interpolation system stays well conditioned; the least
  // Frobenius norm interpolant does not depend on the origin).
  void shift_base(const Vec& xnew) {
    Vec v(n);
    for (int i = 0; i < n; ++i) v[i] = xnew[i] - x0[i];
    const double cnew = model(xnew);
    for (int i = 0; i < n; ++i) {
      double hv = 0;
      for (int j = 0; j < n; ++j) hv += H[i][j] * v[j];
      g[i] += hv;
    }
    c0 = cnew;
    x0 = xnew;
  }

  void clamp(Vec& x) const {
    for (int i = 0; i < n; ++i) x[i] = std::min(ub[i], std::max(lb[i], x[i]));
  }

  // Replace interpolation point k by x with value fx and refresh the model.
  void replace(int k, const Vec& x, double fx) {
    const double fbest = F[kopt];
    Y[k] = x;
    F[k] = fx;
    if (fx < fbest) {
      if (std::fabs(fbest - fx) < ftol_abs) stop = true;  // NLopt ftol_abs on an improvement
      kopt = k;
    }
    if (!update_model()) stop = true;
  }

  void run(Vec& x) {
    npt = 2 * n + 1;
    // x0 onto a bound when it lies within rhobeg of it (BOBYQA's start rule)
    x0 = x;
    clamp(x0);
    for (int i = 0; i < n; ++i) {
      if (x0[i] - lb[i] < rhobeg) x0[i] = (x0[i] <= lb[i]) ? lb[i] : lb[i] + rhobeg;
      else if (ub[i] - x0[i] < rhobeg) x0[i] = (x0[i] >= ub[i]) ? ub[i] : ub[i] - rhobeg;
    }
    g.assign(n, 0.0);
    H.assign(n, Vec(n, 0.0));
    Y.clear();
    F.clear();
    // PRELIM
    Y.push_back(x0);
    F.push_back(eval(x0));
    kopt = 0;
    Vec first_step(n, 0.0);
    for (int k = 1; k < npt && nf < maxeval; ++k) {
      Vec p = x0;
      if (k <= n) {
        const int i = k - 1;
        double st = rhobeg;
        if (x0[i] >= ub[i]) st = -rhobeg;
        first_step[i] = st;
        p[i] += st;
      } else {
        const int i = k - n - 1;
        double st = -rhobeg;
        if (x0[i] <= lb[i]) st = std::min(2.0 * rhobeg, ub[i] - x0[i]);
        if (x0[i] >= ub[i]) st = std::max(-2.0 * rhobeg, lb[i] - x0[i]);
        p[i] += st;
      }
      Y.push_back(p);
      F.push_back(eval(p));
      if (F.back() < F[kopt]) kopt = (int)F.size() - 1;
    }
    if ((int)Y.size() < npt) {  // stopped by maxeval during the initial points
      x = Y[kopt];
      return;
    }
    if (!update_model()) {
      x = Y[kopt];
      status = EGS_ERR_STATE;
      return;
    }
    double rho = rhobeg, delta = rhobeg;
    while (!stop && nf < maxeval) {
      shift_base(Y[kopt]);
      Vec d = trust_step(delta);
      const double dn = norm(d);
      const Vec& xb = Y[kopt];
      if (dn < 0.5 * rho) {
        // Short step: improve the geometry if a point is far away, else shrink rho.
        int far = -1;
        double fd = 0;
        for (int k = 0; k < npt; ++k) {
          Vec dv(n);
          for (int i = 0; i < n; ++i) dv[i] = Y[k][i] - xb[i];
          const double dist = norm(dv);
          if (dist > fd) {
            fd = dist;
            far = k;
          }
        }
        if (far >= 0 && fd > 2.0 * rho) {
          geometry_step(far, std::max(rho, std::min(0.5 * fd, delta)));
          continue;
        }
        if (rho <= rhoend) break;
        const double rnew = (rho > 250.0 * rhoend) ? 0.1 * rho : (rho > 16.0 * rhoend ? std::sqrt(rho * rhoend) : rhoend);
        delta = std::max(0.5 * rho, rnew);
        rho = rnew;
        continue;
      }
      Vec xn(n);
      for (int i = 0; i < n; ++i) xn[i] = xb[i] + d[i];
      clamp(xn);
      const double qold = model(xb), qnew = model(xn);
      const double fnew = eval(xn);
      const double pred = qold - qnew;
      const double ratio = pred > 0 ? (F[kopt] - fnew) / pred : -1.0;
      if (ratio <= 0.1) delta = std::min(0.5 * delta, dn);
      else if (ratio <= 0.7) delta = std::max(0.5 * delta, dn);
      else delta = std::max(0.5 * delta, 2.0 * dn);
      if (delta <= 1.5 * rho) delta = rho;
      // point to drop: largest |Lagrange value| weighted by distance from the best point
      Vec lag;
      int knew = -1;
      if (lagrange(xn, lag)) {
        const Vec& xbest = (fnew < F[kopt]) ? xn : Y[kopt];
        double best = -1;
        for (int k = 0; k < npt; ++k) {
          if (k == kopt && fnew >= F[kopt]) continue;
          Vec dv(n);
          for (int i = 0; i < n; ++i) dv[i] = Y[k][i] - xbest[i];
          const double dist = norm(dv);
          const double w = std::max(1.0, (dist / std::max(delta, 1e-300)) * (dist / std::max(delta, 1e-300)));
          const double sc = std::fabs(lag[k]) * w;
          if (sc > best) {
            best = sc;
            knew = k;
          }
        }
      }
      if (knew < 0) break;
      replace(knew, xn, fnew);
      if (ratio <= 0 && delta <= rho) {
        // no progress at the smallest radius: shrink rho
        if (rho <= rhoend) break;
        const double rnew = (rho > 250.0 * rhoend) ? 0.1 * rho : (rho > 16.0 * rhoend ? std::sqrt(rho * rhoend) : rhoend);
        delta = std::max(0.5 * rho, rnew);
        rho = rnew;
      }
    }
    x = Y[kopt];
  }

  void geometry_step(int k, double radius) {
    const Vec xb = Y[kopt];
    std::vector<Vec> cands;
    for (int i = 0; i < n; ++i) {
      for (int sgn = -1; sgn <= 1; sgn += 2) {
        Vec c = xb;
        c[i] += sgn * radius;
        clamp(c);
        cands.push_back(c);
      }
    }
    Vec dv(n);
    for (int i = 0; i < n; ++i) dv[i] = Y[k][i] - xb[i];
    const double dn = norm(dv);
    if (dn > 0) {
      for (int sgn = -1; sgn <= 1; sgn += 2) {
        Vec c = xb;
        for (int i = 0; i < n; ++i) c[i] += sgn * radius * dv[i] / dn;
        clamp(c);
        cands.push_back(c);
      }
    }
    double best = -1;
    int ibest = -1;
    for (int c = 0; c < (int)cands.size(); ++c) {
      Vec lag;
      if (!lagrange(cands[c], lag)) continue;
      if (std::fabs(lag[k]) > best) {
        best = std::fabs(lag[k]);
        ibest = c;
      }
    }
    if (ibest < 0 || nf >= maxeval) {
      stop = true;
      return;
    }
    const double fv = eval(cands[ibest]);
    replace(k, cands[ibest], fv);
  }
};

}  // namespace

extern "C" {

EGS_API int egs_bobyqa_maximize(int n, double* x, const double* lb, const double* ub, double rhobeg,
                                double ftol_abs, int maxeval, egs_objective_fn f, void* ctx, double* fbest,
                                int* nevals) {
  if (n <= 0 || !x || !lb || !ub || !f || maxeval <= 0) return EGS_ERR_INVALID;
  for (int i = 0; i < n; ++i)
    if (!(ub[i] > lb[i])) return EGS_ERR_INVALID;
  Optimizer opt;
  opt.n = n;
  opt.lb.assign(lb, lb + n);
  opt.ub.assign(ub, ub + n);
  double minwidth = std::numeric_limits<double>::max();
  for (int i = 0; i < n; ++i) minwidth = std::min(minwidth, ub[i] - lb[i]);
  opt.rhobeg = (rhobeg > 0) ? std::min(rhobeg, 0.5 * minwidth) : 0.25 * minwidth;
  opt.rhoend = 1e-8 * opt.rhobeg;
  opt.ftol_abs = ftol_abs;
  opt.maxeval = maxeval;
  opt.fmin = [&](const Vec& v) { return -f(n, v.data(), ctx); };
  Vec xv(x, x + n);
  opt.run(xv);
  for (int i = 0; i < n; ++i) x[i] = xv[i];
  if (fbest) *fbest = -opt.F[opt.kopt];
  if (nevals) *nevals = opt.nf;
  return opt.status;
}

}  // extern "C"
