// ORACLE / TEST INFRASTRUCTURE ONLY -- never linked into the product library.
//
// Project-written Powell direction-set minimiser (M.J.D. Powell, "An efficient
// method for finding the minimum of a function of several variables without
// calculating derivatives", Comput. J. 7 (1964)) with Brent's parabolic /
// golden-section line minimiser (R.P. Brent, "Algorithms for Minimization
// without Derivatives", 1973, ch. 5).
//
// The reference includes `powell_nr3.hpp` from the un-vendored header library
// "toofus" (src/p-tracker.hpp:51, TOOFUSPATH in src/Makefile:1).  toofus is not
// present, has no pinned version, and the reference ships no tests, so the
// Powell boundary is PARITY UNPINNED: this file restates the published method
// with the interface the reference calls (src/p-tracker.cpp:1111-1116):
//     Powell<F> powell(func, ftol);  X = powell.minimize(X, DX);  powell.fret
// The CUDA path (p-tracker_b200/csrc/ptk_subpix.cu) implements the same
// algorithm step for step: same bracketing, same Brent constants, same
// termination tests, same direction-replacement test.
#pragma once

#include <cmath>
#include <vector>

namespace ptk_oracle {

// Constants shared with the device implementation.
constexpr double kGold = 1.6180339887498949;      // golden-ratio expansion factor
constexpr double kCGold = 0.3819660112501051;     // 2 - golden ratio
constexpr double kLineRelTol = 1.0e-4;            // Brent relative x tolerance
constexpr double kLineAbsTol = 1.0e-10;           // Brent absolute x tolerance
constexpr int kBracketMaxIter = 60;
constexpr int kBrentMaxIter = 100;
constexpr int kPowellMaxIter = 200;
constexpr double kTiny = 1.0e-25;

// One-dimensional minimisation of g(alpha) = f(p + alpha * d).
// Returns alpha at the minimum and writes g there to *gmin.
template <class G>
double line_minimize(G& g, double* gmin) {
  // --- bracket: golden expansion from {0, 1} (downhill direction first)
  double a = 0.0, b = 1.0;
  double ga = g(a), gb = g(b);
  if (gb > ga) {
    double t = a; a = b; b = t;
    t = ga; ga = gb; gb = t;
  }
  double c = b + kGold * (b - a);
  double gc = g(c);
  int it = 0;
  while (gc < gb && it < kBracketMaxIter) {
    a = b; ga = gb;
    b = c; gb = gc;
    c = b + kGold * (b - a);
    gc = g(c);
    ++it;
  }
  // interval [lo, hi] contains b with g(b) <= g(a), g(c)
  double lo = a < c ? a : c;
  double hi = a < c ? c : a;

  // --- Brent: parabolic interpolation safeguarded by golden sections
  double x = b, w = b, v = b;
  double fx = gb, fw = gb, fv = gb;
  double d = 0.0, e = 0.0;
  for (int iter = 0; iter < kBrentMaxIter; ++iter) {
    const double m = 0.5 * (lo + hi);
    const double tol1 = kLineRelTol * std::fabs(x) + kLineAbsTol;
    const double tol2 = 2.0 * tol1;
    if (std::fabs(x - m) <= tol2 - 0.5 * (hi - lo)) break;
    bool golden = true;
    if (std::fabs(e) > tol1) {
      double r = (x - w) * (fx - fv);
      double q = (x - v) * (fx - fw);
      double p = (x - v) * q - (x - w) * r;
      q = 2.0 * (q - r);
      if (q > 0.0) p = -p; else q = -q;
      const double eprev = e;
      e = d;
      if (std::fabs(p) < std::fabs(0.5 * q * eprev) && p > q * (lo - x) && p < q * (hi - x)) {
        d = p / q;
        const double u = x + d;
        if (u - lo < tol2 || hi - u < tol2) d = (m - x) >= 0.0 ? tol1 : -tol1;
        golden = false;
      }
    }
    if (golden) {
      e = (x >= m) ? lo - x : hi - x;
      d = kCGold * e;
    }
    const double u = (std::fabs(d) >= tol1) ? x + d : x + (d >= 0.0 ? tol1 : -tol1);
    const double fu = g(u);
    if (fu <= fx) {
      if (u >= x) lo = x; else hi = x;
      v = w; fv = fw;
      w = x; fw = fx;
      x = u; fx = fu;
    } else {
      if (u < x) lo = u; else hi = u;
      if (fu <= fw || w == x) {
        v = w; fv = fw;
        w = u; fw = fu;
      } else if (fu <= fv || v == x || v == w) {
        v = u; fv = fu;
      }
    }
  }
  *gmin = fx;
  return x;
}

template <class F>
class Powell {
 public:
  Powell(F& f, double ftol_ = 1.0e-8) : func(f), ftol(ftol_) {}

  // Initial directions are the coordinate axes scaled by `step`
  // (the reference passes DX = initial_direction_{dx,dy,dr}).
  std::vector<double> minimize(std::vector<double> p, std::vector<double> step) {
    const size_t n = p.size();
    std::vector<std::vector<double>> dirs(n, std::vector<double>(n, 0.0));
    for (size_t i = 0; i < n; ++i) dirs[i][i] = step[i];
    return minimize(p, dirs);
  }

  std::vector<double> minimize(std::vector<double> p, std::vector<std::vector<double>> dirs) {
    const size_t n = p.size();
    std::vector<double> pstart = p, ptt(n), xit(n), trial(n);
    fret = func(p);
    nfev = 1;
    if (!std::isfinite(fret)) return p;  // flat window: NCC undefined, nothing to minimise
    for (iter = 0; iter < kPowellMaxIter; ++iter) {
      const double fp = fret;
      size_t ibig = 0;
      double del = 0.0;
      for (size_t i = 0; i < n; ++i) {
        const double fptt = fret;
        line_search(p, dirs[i], trial);
        if (fptt - fret > del) {
          del = fptt - fret;
          ibig = i;
        }
      }
      if (2.0 * (fp - fret) <= ftol * (std::fabs(fp) + std::fabs(fret)) + kTiny) return p;
      for (size_t j = 0; j < n; ++j) {
        ptt[j] = 2.0 * p[j] - pstart[j];
        xit[j] = p[j] - pstart[j];
        pstart[j] = p[j];
      }
      const double fe = func(ptt);
      ++nfev;
      if (fe < fp) {
        const double t1 = fp - fret - del;
        const double t = 2.0 * (fp - 2.0 * fret + fe) * t1 * t1 - del * (fp - fe) * (fp - fe);
        if (t < 0.0) {
          line_search(p, xit, trial);
          dirs[ibig] = dirs[n - 1];
          dirs[n - 1] = xit;
        }
      }
    }
    return p;
  }

  double fret{0.0};
  int iter{0};
  int nfev{0};

 private:
  // Minimise along `dir` from p; moves p to the minimum, scales `dir` by the
  // step taken, and stores the minimum value in fret.
  void line_search(std::vector<double>& p, std::vector<double>& dir, std::vector<double>& trial) {
    const size_t n = p.size();
    auto g = [&](double alpha) {
      for (size_t j = 0; j < n; ++j) trial[j] = p[j] + alpha * dir[j];
      ++nfev;
      return func(trial);
    };
    double gmin;
    const double alpha = line_minimize(g, &gmin);
    for (size_t j = 0; j < n; ++j) {
      dir[j] *= alpha;
      p[j] += dir[j];
    }
    fret = gmin;
  }

  F& func;
  double ftol;
};

}  // namespace ptk_oracle
