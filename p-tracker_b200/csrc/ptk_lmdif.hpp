// Levenberg-Marquardt least squares with a forward-difference Jacobian, for
// the LEVMAR variant of the distortion-parameter fit
// (src/distortion_correction.cpp:400-479, which calls lmdif1 from the
// un-vendored toofus library with tol = DBL_EPSILON).
//
// Written from the published algorithm: J.J. More, "The Levenberg-Marquardt
// algorithm: implementation and theory", Lecture Notes in Mathematics 630
// (1978), and the MINPACK-1 user guide (More, Garbow, Hillstrom, Argonne
// ANL-80-74, 1980), whose lmdif1 driver sets ftol = xtol = tol, gtol = 0,
// maxfev = 200 (n + 1), a forward-difference step of sqrt(machine epsilon)
// relative to each parameter, scaling by the Jacobian's column norms, and an
// initial trust-region radius of 100 times the scaled parameter norm.  The
// steps: QR factorisation of the Jacobian with column pivoting (Householder),
// the Levenberg-Marquardt parameter for the trust region by the safeguarded
// Newton iteration on ||D p|| - delta, each trial step solved through Givens
// rotations of the triangular factor, the ratio of actual to predicted
// reduction deciding the radius, and the convergence tests on the relative
// reduction, the relative step and the number of evaluations.
//
// Host code; the residuals come from the caller's functor
//     bool f(const double* x, double* fvec)   (false: evaluation failed).
#pragma once

#include <cfloat>
#include <cmath>
#include <vector>

namespace ptk {
namespace lmdif {

// info codes (as lmdif): 0 bad input, 1 relative reduction <= ftol, 2
// relative step <= xtol, 3 both, 4 gradient orthogonal (gtol), 5 evaluation
// limit, 6 ftol too small, 7 xtol too small, 8 gtol too small; -1 the
// functor failed.
inline const char* info_text(int info) {
  switch (info) {
    case 0: return "improper input parameters";
    case 1: return "relative reduction in the sum of squares is at most tol";
    case 2: return "relative error between two consecutive iterates is at most tol";
    case 3: return "conditions for info = 1 and info = 2 both hold";
    case 4: return "fvec is orthogonal to the columns of the Jacobian to machine precision";
    case 5: return "number of calls to fcn has reached or exceeded 200*(n+1)";
    case 6: return "tol is too small: no further reduction in the sum of squares is possible";
    case 7: return "tol is too small: no further improvement in the approximate solution x is possible";
    case 8: return "the gradient is orthogonal to the Jacobian's columns to machine precision";
    default: return "the residual evaluation failed";
  }
}

// Euclidean norm with MINPACK's three accumulators (components below
// rdwarf, between, and above rgiant / n), so that no square under- or
// overflows; for ordinary magnitudes it is sqrt of the sum of squares taken in
// index order.
inline double enorm(int n, const double* x) {
  const double rdwarf = 3.834e-20, rgiant = 1.304e19;
  double s1 = 0.0, s2 = 0.0, s3 = 0.0, x1max = 0.0, x3max = 0.0;
  const double agiant = rgiant / (double)n;
  for (int i = 0; i < n; ++i) {
    const double xabs = std::fabs(x[i]);
    if (xabs > rdwarf && xabs < agiant) {
      s2 += xabs * xabs;
    } else if (xabs <= rdwarf) {
      if (xabs > x3max) {
        const double t = x3max / xabs;
        s3 = 1.0 + s3 * t * t;
        x3max = xabs;
      } else if (xabs != 0.0) {
        const double t = xabs / x3max;
        s3 += t * t;
      }
    } else {
      if (xabs > x1max) {
        const double t = x1max / xabs;
        s1 = 1.0 + s1 * t * t;
        x1max = xabs;
      } else {
        const double t = xabs / x1max;
        s1 += t * t;
      }
    }
  }
  if (s1 != 0.0) return x1max * std::sqrt(s1 + (s2 / x1max) / x1max);
  if (s2 != 0.0) {
    if (s2 >= x3max) return std::sqrt(s2 * (1.0 + (x3max / s2) * (x3max * s3)));
    return std::sqrt(x3max * ((s2 / x3max) + (x3max * s3)));
  }
  return x3max * std::sqrt(s3);
}

// Householder QR with column pivoting of the m x n matrix a (column-major,
// lda = m): on return the upper triangle holds R without its diagonal (rdiag),
// the lower part the Householder vectors, ipvt the permutation, acnorm the
// column norms of the input.
inline void qrfac(int m, int n, double* a, int* ipvt, double* rdiag, double* acnorm, double* wa) {
  const double epsmch = DBL_EPSILON;
  for (int j = 0; j < n; ++j) {
    acnorm[j] = enorm(m, a + (size_t)j * m);
    rdiag[j] = acnorm[j];
    wa[j] = rdiag[j];
    ipvt[j] = j;
  }
  const int minmn = m < n ? m : n;
  for (int j = 0; j < minmn; ++j) {
    int kmax = j;
    for (int k = j; k < n; ++k)
      if (rdiag[k] > rdiag[kmax]) kmax = k;
    if (kmax != j) {
      for (int i = 0; i < m; ++i) std::swap(a[i + (size_t)j * m], a[i + (size_t)kmax * m]);
      rdiag[kmax] = rdiag[j];
      wa[kmax] = wa[j];
      std::swap(ipvt[j], ipvt[kmax]);
    }
    double* aj = a + (size_t)j * m;
    double ajnorm = enorm(m - j, aj + j);
    if (ajnorm != 0.0) {
      if (aj[j] < 0.0) ajnorm = -ajnorm;
      for (int i = j; i < m; ++i) aj[i] /= ajnorm;
      aj[j] += 1.0;
      for (int k = j + 1; k < n; ++k) {
        double* ak = a + (size_t)k * m;
        double sum = 0.0;
        for (int i = j; i < m; ++i) sum += aj[i] * ak[i];
        const double temp = sum / aj[j];
        for (int i = j; i < m; ++i) ak[i] -= temp * aj[i];
        if (rdiag[k] != 0.0) {
          double t = ak[j] / rdiag[k];
          t = 1.0 - t * t;
          rdiag[k] *= std::sqrt(t > 0.0 ? t : 0.0);
          t = rdiag[k] / wa[k];
          if (0.05 * t * t <= epsmch) {
            rdiag[k] = enorm(m - j - 1, ak + j + 1);
            wa[k] = rdiag[k];
          }
        }
      }
    }
    rdiag[j] = -ajnorm;
  }
}

// Solves min || [A; D] x - [b; 0] || given the QR factors of A P (r: n x n,
// column-major, ldr = n, upper triangle R; on return its strict lower
// triangle holds the transpose of S with S^T S = P^T (A^T A + D D) P, sdiag
// the diagonal of S), qtb = first n entries of Q^T b.
inline void qrsolv(int n, double* r, int ldr, const int* ipvt, const double* diag, const double* qtb, double* x,
                   double* sdiag, double* wa) {
  for (int j = 0; j < n; ++j) {
    for (int i = j; i < n; ++i) r[i + (size_t)j * ldr] = r[j + (size_t)i * ldr];
    x[j] = r[j + (size_t)j * ldr];
    wa[j] = qtb[j];
  }
  for (int j = 0; j < n; ++j) {
    const int l = ipvt[j];
    if (diag[l] != 0.0) {
      for (int k = j; k < n; ++k) sdiag[k] = 0.0;
      sdiag[j] = diag[l];
      double qtbpj = 0.0;
      for (int k = j; k < n; ++k) {
        if (sdiag[k] == 0.0) continue;
        double cs, sn;
        const double rkk = r[k + (size_t)k * ldr];
        if (std::fabs(rkk) < std::fabs(sdiag[k])) {
          const double cot = rkk / sdiag[k];
          sn = 0.5 / std::sqrt(0.25 + 0.25 * cot * cot);
          cs = sn * cot;
        } else {
          const double tn = sdiag[k] / rkk;
          cs = 0.5 / std::sqrt(0.25 + 0.25 * tn * tn);
          sn = cs * tn;
        }
        r[k + (size_t)k * ldr] = cs * rkk + sn * sdiag[k];
        const double temp = cs * wa[k] + sn * qtbpj;
        qtbpj = -sn * wa[k] + cs * qtbpj;
        wa[k] = temp;
        for (int i = k + 1; i < n; ++i) {
          const double t2 = cs * r[i + (size_t)k * ldr] + sn * sdiag[i];
          sdiag[i] = -sn * r[i + (size_t)k * ldr] + cs * sdiag[i];
          r[i + (size_t)k * ldr] = t2;
        }
      }
    }
    sdiag[j] = r[j + (size_t)j * ldr];
    r[j + (size_t)j * ldr] = x[j];
  }
  int nsing = n;
  for (int j = 0; j < n; ++j) {
    if (sdiag[j] == 0.0 && nsing == n) nsing = j;
    if (nsing < n) wa[j] = 0.0;
  }
  for (int j = nsing - 1; j >= 0; --j) {
    double sum = 0.0;
    for (int i = j + 1; i < nsing; ++i) sum += r[i + (size_t)j * ldr] * wa[i];
    wa[j] = (wa[j] - sum) / sdiag[j];
  }
  for (int j = 0; j < n; ++j) x[ipvt[j]] = wa[j];
}

// Levenberg-Marquardt parameter for the trust region radius delta (More's
// safeguarded Newton iteration, at most 10 steps).
inline void lmpar(int n, double* r, int ldr, const int* ipvt, const double* diag, const double* qtb, double delta,
                  double* par, double* x, double* sdiag, double* wa1, double* wa2) {
  const double dwarf = DBL_MIN;
  const double p1 = 0.1, p001 = 0.001;
  int nsing = n;
  for (int j = 0; j < n; ++j) {
    wa1[j] = qtb[j];
    if (r[j + (size_t)j * ldr] == 0.0 && nsing == n) nsing = j;
    if (nsing < n) wa1[j] = 0.0;
  }
  for (int j = nsing - 1; j >= 0; --j) {
    wa1[j] /= r[j + (size_t)j * ldr];
    const double temp = wa1[j];
    for (int i = 0; i < j; ++i) wa1[i] -= r[i + (size_t)j * ldr] * temp;
  }
  for (int j = 0; j < n; ++j) x[ipvt[j]] = wa1[j];
  int iter = 0;
  for (int j = 0; j < n; ++j) wa2[j] = diag[j] * x[j];
  double dxnorm = enorm(n, wa2);
  double fp = dxnorm - delta;
  if (fp <= p1 * delta) {
    *par = 0.0;
    return;
  }
  double parl = 0.0;
  if (nsing >= n) {
    for (int j = 0; j < n; ++j) {
      const int l = ipvt[j];
      wa1[j] = diag[l] * (wa2[l] / dxnorm);
    }
    for (int j = 0; j < n; ++j) {
      double sum = 0.0;
      for (int i = 0; i < j; ++i) sum += r[i + (size_t)j * ldr] * wa1[i];
      wa1[j] = (wa1[j] - sum) / r[j + (size_t)j * ldr];
    }
    const double temp = enorm(n, wa1);
    parl = ((fp / delta) / temp) / temp;
  }
  for (int j = 0; j < n; ++j) {
    double sum = 0.0;
    for (int i = 0; i <= j; ++i) sum += r[i + (size_t)j * ldr] * qtb[i];
    wa1[j] = sum / diag[ipvt[j]];
  }
  const double gnorm = enorm(n, wa1);
  double paru = gnorm / delta;
  if (paru == 0.0) paru = dwarf / std::fmin(delta, p1);
  *par = std::fmax(*par, parl);
  *par = std::fmin(*par, paru);
  if (*par == 0.0) *par = gnorm / dxnorm;
  for (;;) {
    ++iter;
    if (*par == 0.0) *par = std::fmax(dwarf, p001 * paru);
    const double temp0 = std::sqrt(*par);
    for (int j = 0; j < n; ++j) wa1[j] = temp0 * diag[j];
    qrsolv(n, r, ldr, ipvt, wa1, qtb, x, sdiag, wa2);
    for (int j = 0; j < n; ++j) wa2[j] = diag[j] * x[j];
    dxnorm = enorm(n, wa2);
    const double temp = fp;
    fp = dxnorm - delta;
    if (std::fabs(fp) <= p1 * delta || (parl == 0.0 && fp <= temp && temp < 0.0) || iter == 10) return;
    for (int j = 0; j < n; ++j) {
      const int l = ipvt[j];
      wa1[j] = diag[l] * (wa2[l] / dxnorm);
    }
    for (int j = 0; j < n; ++j) {
      wa1[j] /= sdiag[j];
      const double t = wa1[j];
      for (int i = j + 1; i < n; ++i) wa1[i] -= r[i + (size_t)j * ldr] * t;
    }
    const double tn = enorm(n, wa1);
    const double parc = ((fp / delta) / tn) / tn;
    if (fp > 0.0) parl = std::fmax(parl, *par);
    if (fp < 0.0) paru = std::fmin(paru, *par);
    *par = std::fmax(parl, *par + parc);
  }
}

// lmdif1: minimises the sum of squares of m residuals of n parameters from x
// (updated in place); fvec holds the residuals at the returned x.  Returns the
// info code; *nfev counts the functor calls.
template <class F>
int lmdif1(F& fcn, int m, int n, double* x, double* fvec, double tol, int* nfev_out = nullptr) {
  if (n <= 0 || m < n || tol < 0.0) return 0;
  const double ftol = tol, xtol = tol, gtol = 0.0, factor = 100.0;
  const int maxfev = 200 * (n + 1);
  const double epsmch = DBL_EPSILON;
  const double eps = std::sqrt(epsmch);  // epsfcn = 0
  std::vector<double> fjac((size_t)m * n), diag(n), qtf(n), wa1(n), wa2(n), wa3(n), wa4(m);
  std::vector<int> ipvt(n);
  int nfev = 0, info = 0, iter = 1;
  auto eval = [&](const double* xx, double* fv) {
    ++nfev;
    return fcn(xx, fv);
  };
  if (!eval(x, fvec)) return -1;
  double fnorm = enorm(m, fvec);
  double par = 0.0, delta = 0.0, xnorm = 0.0;
  for (;;) {
    // forward-difference Jacobian
    for (int j = 0; j < n; ++j) {
      const double temp = x[j];
      double h = eps * std::fabs(temp);
      if (h == 0.0) h = eps;
      x[j] = temp + h;
      if (!eval(x, wa4.data())) {
        x[j] = temp;
        if (nfev_out) *nfev_out = nfev;
        return -1;
      }
      x[j] = temp;
      for (int i = 0; i < m; ++i) fjac[i + (size_t)j * m] = (wa4[i] - fvec[i]) / h;
    }
    qrfac(m, n, fjac.data(), ipvt.data(), wa1.data(), wa2.data(), wa3.data());
    if (iter == 1) {
      for (int j = 0; j < n; ++j) diag[j] = wa2[j] == 0.0 ? 1.0 : wa2[j];
      for (int j = 0; j < n; ++j) wa3[j] = diag[j] * x[j];
      xnorm = enorm(n, wa3.data());
      delta = factor * xnorm;
      if (delta == 0.0) delta = factor;
    }
    // Q^T fvec: the first n entries into qtf, the triangle R into fjac's upper part
    for (int i = 0; i < m; ++i) wa4[i] = fvec[i];
    for (int j = 0; j < n; ++j) {
      const double* aj = fjac.data() + (size_t)j * m;
      if (aj[j] != 0.0) {
        double sum = 0.0;
        for (int i = j; i < m; ++i) sum += aj[i] * wa4[i];
        const double temp = -sum / aj[j];
        for (int i = j; i < m; ++i) wa4[i] += aj[i] * temp;
      }
      fjac[j + (size_t)j * m] = wa1[j];
      qtf[j] = wa4[j];
    }
    // scaled gradient norm
    double gnorm = 0.0;
    if (fnorm != 0.0) {
      for (int j = 0; j < n; ++j) {
        const int l = ipvt[j];
        if (wa2[l] != 0.0) {
          double sum = 0.0;
          for (int i = 0; i <= j; ++i) sum += fjac[i + (size_t)j * m] * (qtf[i] / fnorm);
          gnorm = std::fmax(gnorm, std::fabs(sum / wa2[l]));
        }
      }
    }
    if (gnorm <= gtol) info = 4;
    if (info != 0) break;
    for (int j = 0; j < n; ++j) diag[j] = std::fmax(diag[j], wa2[j]);
    // the triangle as an n x n column-major matrix for lmpar / qrsolv
    std::vector<double> r((size_t)n * n);
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) r[i + (size_t)j * n] = fjac[i + (size_t)j * m];
    double ratio = 0.0;
    do {
      lmpar(n, r.data(), n, ipvt.data(), diag.data(), qtf.data(), delta, &par, wa1.data(), wa2.data(), wa3.data(),
            wa4.data());
      for (int j = 0; j < n; ++j) {
        wa1[j] = -wa1[j];
        wa2[j] = x[j] + wa1[j];
        wa3[j] = diag[j] * wa1[j];
      }
      const double pnorm = enorm(n, wa3.data());
      if (iter == 1) delta = std::fmin(delta, pnorm);
      std::vector<double> f1(m);
      if (!eval(wa2.data(), f1.data())) {
        if (nfev_out) *nfev_out = nfev;
        return -1;
      }
      const double fnorm1 = enorm(m, f1.data());
      double actred = -1.0;
      if (0.1 * fnorm1 < fnorm) {
        const double t = fnorm1 / fnorm;
        actred = 1.0 - t * t;
      }
      for (int j = 0; j < n; ++j) {
        wa3[j] = 0.0;
        const double temp = wa1[ipvt[j]];
        for (int i = 0; i <= j; ++i) wa3[i] += r[i + (size_t)j * n] * temp;
      }
      const double temp1 = enorm(n, wa3.data()) / fnorm;
      const double temp2 = (std::sqrt(par) * pnorm) / fnorm;
      const double prered = temp1 * temp1 + temp2 * temp2 / 0.5;
      const double dirder = -(temp1 * temp1 + temp2 * temp2);
      ratio = prered != 0.0 ? actred / prered : 0.0;
      if (ratio <= 0.25) {
        double temp = actred >= 0.0 ? 0.5 : 0.5 * dirder / (dirder + 0.5 * actred);
        if (0.1 * fnorm1 >= fnorm || temp < 0.1) temp = 0.1;
        delta = temp * std::fmin(delta, pnorm / 0.1);
        par /= temp;
      } else if (par == 0.0 || ratio >= 0.75) {
        delta = pnorm / 0.5;
        par = 0.5 * par;
      }
      if (ratio >= 1e-4) {  // successful step
        for (int j = 0; j < n; ++j) {
          x[j] = wa2[j];
          wa2[j] = diag[j] * x[j];
        }
        for (int i = 0; i < m; ++i) fvec[i] = f1[i];
        xnorm = enorm(n, wa2.data());
        fnorm = fnorm1;
        ++iter;
      }
      if (std::fabs(actred) <= ftol && prered <= ftol && 0.5 * ratio <= 1.0) info = 1;
      if (delta <= xtol * xnorm) info = 2;
      if (std::fabs(actred) <= ftol && prered <= ftol && 0.5 * ratio <= 1.0 && info == 2) info = 3;
      if (info != 0) break;
      if (nfev >= maxfev) info = 5;
      if (std::fabs(actred) <= epsmch && prered <= epsmch && 0.5 * ratio <= 1.0) info = 6;
      if (delta <= epsmch * xnorm) info = 7;
      if (gnorm <= epsmch) info = 8;
      if (info != 0) break;
    } while (ratio < 1e-4);
    if (info != 0) break;
  }
  if (nfev_out) *nfev_out = nfev;
  return info;
}

}  // namespace lmdif
}  // namespace ptk
