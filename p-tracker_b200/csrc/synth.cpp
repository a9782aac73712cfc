// Seeded synthetic frames for p-tracker workloads: non-overlapping disc grains
// textured with analytic Gaussian speckles on a dark background (the disc rim
// is anti-aliased with an erf profile of width 0.7 px), each grain
// rendered analytically (not resampled) at an arbitrary rigid pose, optionally
// seen through the Brown + parallax lens model of the reference's undistor
// (src/distortion_correction.cpp:20-61), plus additive Gaussian noise.
//
// Pose convention follows the tracker (src/p-tracker.cpp:615-621,1047-1053):
// the material point at offset p from a grain's centre in the reference frame
// appears at c + d + R(theta) p, with R(theta) p = (cos t px + sin t py,
// -sin t px + cos t py) (y axis pointing down).
//
// All randomness comes from counter-based SplitMix64 streams, so results are
// identical for any thread count.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

inline uint64_t splitmix(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

struct Rng {
  uint64_t s;
  explicit Rng(uint64_t seed) : s(splitmix(seed ^ 0x5DEECE66Dull)) {}
  uint64_t next() {
    s += 0x9E3779B97F4A7C15ull;
    uint64_t z = s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
  double uniform(double a, double b) { return a + (b - a) * uniform(); }
  double normal() {
    double u1 = uniform(), u2 = uniform();
    if (u1 < 1e-300) u1 = 1e-300;
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
  }
};

struct Speckle {
  double x, y, a;
};

// Speckles of one grain in its own (reference) frame: uniform in the disc of
// radius r + 2 sigma so the texture reaches the rim.
std::vector<Speckle> grain_speckles(uint64_t gseed, double r, double sigma, double density, double amp_lo,
                                    double amp_hi) {
  Rng rng(gseed);
  const double R = r + 2.0 * sigma;
  const int n = (int)std::lround(density * 3.141592653589793 * R * R);
  std::vector<Speckle> s;
  s.reserve(n);
  while ((int)s.size() < n) {
    double x = rng.uniform(-R, R), y = rng.uniform(-R, R);
    if (x * x + y * y > R * R) continue;
    s.push_back(Speckle{x, y, rng.uniform(amp_lo, amp_hi)});
  }
  return s;
}

void undistor(const double* X, const double* trig, double xd, double yd, double* xo, double* yo) {
  const double dx = xd - X[0], dy = yd - X[1];
  const double r2 = dx * dx + dy * dy, r4 = r2 * r2, r6 = r4 * r2;
  const double rad = X[2] * r2 + X[3] * r4 + X[4] * r6;
  double xu = xd + dx * rad + (X[5] * (r2 + 2.0 * dx * dx) + 2.0 * X[6] * dx * dy) * (1.0 + X[7] * r2);
  double yu = yd + dy * rad + (2.0 * X[5] * dx * dy + X[6] * (r2 + 2.0 * dy * dy)) * (1.0 + X[7] * r2);
  const double nx1 = trig[0], ny1 = trig[1], nx2 = trig[2], ny2 = trig[3];
  const double dX = xu - X[8], dY = yu - X[9];
  const double S1 = (1.0 + X[11]) * (dX * nx1 + dY * ny1);
  const double S2 = (1.0 + X[13]) * (dX * nx2 + dY * ny2);
  *xo = X[8] + S1 * nx1 + S2 * nx2;
  *yo = X[9] + S1 * ny1 + S2 * ny2;
}

}  // namespace

extern "C" {

// Places up to n non-overlapping discs.  Radii follow a mixture of uniform
// laws (weights w[k], range [rlo[k], rhi[k]]).  Disc centres keep `margin`
// pixels plus the radius away from the frame edge; edge-to-edge gaps are at
// least `gap`.  Per-grain speckle sigma is uniform in [sig_lo, sig_hi] and
// each grain receives its own texture seed.  Returns the number placed.
int ptk_synth_place(int dimx, int dimy, int n, int nmix, const double* w, const double* rlo, const double* rhi,
                    double sig_lo, double sig_hi, double margin, double gap, uint64_t seed, double* cx, double* cy,
                    double* r, double* sig, uint64_t* gseed) {
  Rng rng(seed);
  double rmax = 0.0, wsum = 0.0;
  for (int k = 0; k < nmix; ++k) {
    rmax = rhi[k] > rmax ? rhi[k] : rmax;
    wsum += w[k];
  }
  const double cell = 2.0 * rmax + gap + 1.0;
  const int gx = (int)(dimx / cell) + 1, gy = (int)(dimy / cell) + 1;
  std::vector<std::vector<int>> grid((size_t)gx * gy);
  int placed = 0;
  long attempts = 0;
  const long max_attempts = (long)n * 2000 + 100000;
  while (placed < n && attempts < max_attempts) {
    ++attempts;
    double pick = rng.uniform() * wsum;
    int k = 0;
    while (k < nmix - 1 && pick >= w[k]) pick -= w[k++];
    const double rr = rng.uniform(rlo[k], rhi[k]);
    const double lo = margin + rr;
    if (dimx - 1 - lo <= lo || dimy - 1 - lo <= lo) continue;
    const double x = rng.uniform(lo, dimx - 1 - lo);
    const double y = rng.uniform(lo, dimy - 1 - lo);
    const double ss = rng.uniform(sig_lo, sig_hi);
    const uint64_t gs = rng.next();
    const int ci = (int)(x / cell), cj = (int)(y / cell);
    bool ok = true;
    for (int j = cj - 1; j <= cj + 1 && ok; ++j)
      for (int i = ci - 1; i <= ci + 1 && ok; ++i) {
        if (i < 0 || j < 0 || i >= gx || j >= gy) continue;
        for (int o : grid[(size_t)j * gx + i]) {
          const double ddx = cx[o] - x, ddy = cy[o] - y, lim = r[o] + rr + gap;
          if (ddx * ddx + ddy * ddy < lim * lim) {
            ok = false;
            break;
          }
        }
      }
    if (!ok) continue;
    cx[placed] = x;
    cy[placed] = y;
    r[placed] = rr;
    sig[placed] = ss;
    gseed[placed] = gs;
    grid[(size_t)cj * gx + ci].push_back(placed);
    ++placed;
  }
  return placed;
}

// Renders one frame.  Grain g sits at (cx+dx, cy+dy) rotated by th.  If
// `disto` (14 parameters in undistor order) is non-null, pixel (X, Y) of the
// output shows the scene point undistor(X, Y), i.e. the frame is what a camera
// with that distortion records.  Values are background + speckles + noise,
// rounded and clamped to [0, maxval].
int ptk_synth_render(int dimx, int dimy, int maxval, double background, double noise_sigma, double density,
                     double amp_lo, double amp_hi, int n, const double* cx, const double* cy, const double* r,
                     const double* sig, const uint64_t* gseed, const double* dx, const double* dy, const double* th,
                     const double* disto, uint64_t noise_seed, int nthreads, uint16_t* out) {
  std::vector<float> img((size_t)dimx * dimy, (float)background);
  double trig[4] = {1, 0, 0, 1};
  double shift_max = 0.0;
  if (disto) {
    trig[0] = std::cos(disto[10]);
    trig[1] = -std::sin(disto[10]);
    trig[2] = -std::sin(disto[12]);
    trig[3] = std::cos(disto[12]);
    // largest displacement of the model over the frame corners and edges
    const double px[8] = {0, (double)dimx - 1, 0, (double)dimx - 1, 0.5 * dimx, 0.5 * dimx, 0, (double)dimx - 1};
    const double py[8] = {0, 0, (double)dimy - 1, (double)dimy - 1, 0, (double)dimy - 1, 0.5 * dimy, 0.5 * dimy};
    for (int k = 0; k < 8; ++k) {
      double xu, yu;
      undistor(disto, trig, px[k], py[k], &xu, &yu);
      double d = std::hypot(xu - px[k], yu - py[k]);
      shift_max = d > shift_max ? d : shift_max;
    }
  }
  if (nthreads < 1) nthreads = 1;
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads)
  for (int g = 0; g < n; ++g) {
    const double s = sig[g];
    std::vector<Speckle> sp = grain_speckles(gseed[g], r[g], s, density, amp_lo, amp_hi);
    // bucket speckles on a local grid with cells of 4 sigma
    const double R = r[g] + 2.0 * s;
    const double cs = 4.0 * s;
    const int nc = (int)std::ceil(2.0 * R / cs) + 1;
    std::vector<std::vector<int>> cells((size_t)nc * nc);
    for (int k = 0; k < (int)sp.size(); ++k) {
      int ci = (int)((sp[k].x + R) / cs), cj = (int)((sp[k].y + R) / cs);
      ci = ci < 0 ? 0 : (ci >= nc ? nc - 1 : ci);
      cj = cj < 0 ? 0 : (cj >= nc ? nc - 1 : cj);
      cells[(size_t)cj * nc + ci].push_back(k);
    }
    const double inv2s2 = 1.0 / (2.0 * s * s);
    const double ccx = cx[g] + dx[g], ccy = cy[g] + dy[g];
    const double c = std::cos(th[g]), sn = std::sin(th[g]);
    double ext = r[g] + 4.0 + (disto ? shift_max + 2.0 : 0.0);
    int x0 = (int)std::floor(ccx - ext), x1 = (int)std::ceil(ccx + ext);
    int y0 = (int)std::floor(ccy - ext), y1 = (int)std::ceil(ccy + ext);
    x0 = x0 < 0 ? 0 : x0;
    y0 = y0 < 0 ? 0 : y0;
    x1 = x1 > dimx - 1 ? dimx - 1 : x1;
    y1 = y1 > dimy - 1 ? dimy - 1 : y1;
    const double rsoft2 = (r[g] + 2.5) * (r[g] + 2.5);
    for (int Y = y0; Y <= y1; ++Y) {
      for (int X = x0; X <= x1; ++X) {
        double sx = X, sy = Y;
        if (disto) undistor(disto, trig, (double)X, (double)Y, &sx, &sy);
        const double qx = sx - ccx, qy = sy - ccy;
        const double rho2 = qx * qx + qy * qy;
        if (rho2 > rsoft2) continue;
        // anti-aliased rim: texture weight 0.5 (1 + erf((r - rho) / 0.7))
        const double alpha = 0.5 * (1.0 + std::erf((r[g] - std::sqrt(rho2)) * (1.0 / 0.7)));
        // material point in the grain's reference frame: p = R(-theta) q
        const double pxl = c * qx - sn * qy;
        const double pyl = sn * qx + c * qy;
        int ci = (int)((pxl + R) / cs), cj = (int)((pyl + R) / cs);
        double val = 0.0;
        for (int jj = cj - 1; jj <= cj + 1; ++jj)
          for (int ii = ci - 1; ii <= ci + 1; ++ii) {
            if (ii < 0 || jj < 0 || ii >= nc || jj >= nc) continue;
            for (int k : cells[(size_t)jj * nc + ii]) {
              const double ex = pxl - sp[k].x, ey = pyl - sp[k].y;
              val += sp[k].a * std::exp(-(ex * ex + ey * ey) * inv2s2);
            }
          }
        img[(size_t)Y * dimx + X] = (float)(background + alpha * val);
      }
    }
  }
#pragma omp parallel for schedule(static) num_threads(nthreads)
  for (int Y = 0; Y < dimy; ++Y) {
    for (int X = 0; X < dimx; ++X) {
      const size_t idx = (size_t)Y * dimx + X;
      double v = img[idx];
      if (noise_sigma > 0.0) {
        Rng rng(noise_seed * 0x100000001B3ull + idx);
        v += noise_sigma * rng.normal();
      }
      double q = std::floor(v + 0.5);
      q = q < 0.0 ? 0.0 : (q > (double)maxval ? (double)maxval : q);
      out[idx] = (uint16_t)q;
    }
  }
  return 0;
}

}  // extern "C"
