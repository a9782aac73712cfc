// Test harness (not part of the library): runs the library's Levenberg-Marquardt
// restatement (p-tracker_b200/csrc/ptk_lmdif.hpp) on standard least-squares
// problems whose residuals tests/test_lmdif.py writes with the same operations,
// so that its results can be compared with MINPACK's lmdif run through scipy.
#include <cfloat>
#include <cmath>

#include "../p-tracker_b200/csrc/ptk_lmdif.hpp"

namespace {

// problem 0: Rosenbrock (m = n = 2); 1: Powell singular (m = n = 4);
// 2: exponential fit y = a exp(-b t) + c on 12 points (m = 12, n = 3);
// 3: linear least squares with a rank-deficient design (m = 6, n = 3).
struct Problem {
  int id;
  bool operator()(const double* x, double* f) const {
    switch (id) {
      case 0:
        f[0] = 10.0 * (x[1] - x[0] * x[0]);
        f[1] = 1.0 - x[0];
        return true;
      case 1:
        f[0] = x[0] + 10.0 * x[1];
        f[1] = std::sqrt(5.0) * (x[2] - x[3]);
        f[2] = (x[1] - 2.0 * x[2]) * (x[1] - 2.0 * x[2]);
        f[3] = std::sqrt(10.0) * (x[0] - x[3]) * (x[0] - x[3]);
        return true;
      case 2:
        for (int i = 0; i < 12; ++i) {
          const double t = 0.5 * (double)i;
          const double y = 2.5 * std::exp(-0.7 * t) + 0.3 + 0.01 * std::sin(3.0 * t);
          f[i] = x[0] * std::exp(-x[1] * t) + x[2] - y;
        }
        return true;
      default:
        for (int i = 0; i < 6; ++i) {
          const double t = (double)i;
          // columns 1 and 2 are identical: rank 2
          f[i] = x[0] + t * x[1] + t * x[2] - (1.0 + 2.0 * t + 0.1 * (double)((i * 7) % 3));
        }
        return true;
    }
  }
};

}  // namespace

extern "C" int lm_run(int problem, int m, int n, double* x, double* fvec, double tol, int* nfev) {
  Problem p{problem};
  return ptk::lmdif::lmdif1(p, m, n, x, fvec, tol, nfev);
}

// Residuals from the caller (a ctypes callback): returns 0 on success.
typedef int (*residual_fn)(const double* x, double* fvec);

extern "C" int lm_run_cb(int m, int n, double* x, double* fvec, double tol, int* nfev, residual_fn cb) {
  auto f = [cb](const double* xx, double* fv) { return cb(xx, fv) == 0; };
  return ptk::lmdif::lmdif1(f, m, n, x, fvec, tol, nfev);
}
