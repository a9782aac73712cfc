// ORACLE / TEST INFRASTRUCTURE ONLY -- never linked into the product library.
//
// CPU restatement of p-tracker's per-grain tracking path, used by the tests and
// by bench.py's CPU-baseline leg as the checker.  Every function follows the
// reference operation for operation (same FP64 operations in the same order,
// no FMA contraction), so on the same inputs it reproduces the compiled
// reference bit for bit; tests/golden pins that.  Images are row-major
// uint16 (index y*dimx + x) instead of the reference's x-major
// vector<vector<uint16_t>> (src/p-tracker.hpp:80); values are identical.
//
// Extra pieces that have no reference counterpart are marked as such:
// the inverse-distortion remap (Newton inversion of undistor + the reference's
// bicubic), the analytic gradient of the subpixel objective, and the top-two
// NCC diagnostic used to exclude near-ties from argmax parity.
#include <omp.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <sstream>
#include <string>
#include <vector>

#include "../powell.hpp"

namespace {

struct Coord {
  int dx{0}, dy{0};
};

// grain_type_2D, src/grain_type_2D.hpp:23-71
struct Grain {
  int refx{0}, refy{0};
  double refrot{0}, radius{0};
  double dx{0}, dy{0}, drot{0};
  double dx_prev{0}, dy_prev{0}, drot_prev{0};
  double upix{0}, vpix{0}, rot_inc{0};
  double NCC{0}, NCC_rescue{0}, NCC_subpix{0};
  double mean0{0}, C0C0{0};
  bool masked{false};
  std::vector<Coord> pattern, pattern0;
  double top1{0}, top2{0};  // diagnostic: two best NCC of the last search
};

// search_zone_type, src/search_zone_type.hpp:20-27
struct Zone {
  int left{0}, right{0}, up{0}, down{0}, num_rot{0};
  double inc_rot{1.0};
};

struct Tracker {
  int dimx{0}, dimy{0};
  std::vector<uint16_t> image[2];
  int iref_idx{0}, icur_idx{1};
  int iref{0}, iraz{0};
  int nthreads{1};
  std::vector<Grain> grain;
  Zone zone[3];
  int rescue_level{2};
  double NCC_min{0.7}, NCC_min_super{0.5};
  int subpixel{1};
  double subpix_tol{1e-8};
  double init_dir[3]{0.01, 0.01, 0.01};
  double subpix_displacement_max{3.0}, overflow_stiffness{0.0};
  int interpolator{1};  // 0 linear, 1 cubic, 2 quintic
  bool require_precomputations{true};
  std::vector<int> rescued, super_rescued;

  inline double pix(int slot, int x, int y) const { return (double)image[slot][(size_t)y * dimx + x]; }
};

// src/p-tracker.cpp:615-621 (round half away from zero, y pointing down)
inline void rotate_pixel(const Coord& p, double c, double s, int* xo, int* yo) {
  double xpix = c * p.dx + s * p.dy;
  double ypix = -s * p.dx + c * p.dy;
  *xo = (int)std::round(xpix);
  *yo = (int)std::round(ypix);
}

// src/p-tracker.cpp:624-656
void precompute(Tracker& t) {
  for (Grain& g : t.grain) {
    const double c0 = std::cos(g.refrot), s0 = std::sin(g.refrot);
    const size_t P = g.pattern.size();
    g.pattern0.resize(P);
    g.mean0 = 0.0;
    g.C0C0 = 0.0;
    for (size_t i = 0; i < P; ++i) {
      int x, y;
      rotate_pixel(g.pattern[i], c0, s0, &x, &y);
      g.pattern0[i].dx = x;
      g.pattern0[i].dy = y;
      g.mean0 += t.pix(t.iref_idx, x + g.refx, y + g.refy);
    }
    g.mean0 /= (double)P;
    for (size_t i = 0; i < P; ++i) {
      double d = t.pix(t.iref_idx, g.pattern0[i].dx + g.refx, g.pattern0[i].dy + g.refy) - g.mean0;
      g.C0C0 += d * d;
    }
  }
  t.require_precomputations = false;
}

// The rotation-step list exactly as the reference's loops produce it
// (src/p-tracker.cpp:684-686, :822-824, :959-961): a double accumulated from
// -rotmax in steps of inc_rot while <= rotmax.
std::vector<double> rotation_steps(const Zone& z) {
  std::vector<double> out;
  double rotmax = std::fabs(z.inc_rot * z.num_rot);
  for (double drot = -rotmax; drot <= rotmax; drot += z.inc_rot) out.push_back(drot);
  return out;
}

// Exhaustive NCC search over the zone (the loop bodies of
// follow_pattern_pixel src/p-tracker.cpp:684-730, follow_pattern_rescue_pixel
// :822-862 and follow_pattern_super_rescue_pixel :959-998).  The neighbour
// exclusion of the rescue variants never removes a candidate in the reference
// (num_neighbour is never incremented, src/p-tracker.cpp:1136-1146), so the
// allowed list is the full zone in x-major order.
struct SearchResult {
  double best{0.0}, best_drot{0.0};
  int best_u{0}, best_v{0};
  double top1{0.0}, top2{0.0};
};

SearchResult search(const Tracker& t, const Grain& g, const Zone& z) {
  SearchResult r;
  const int gdx = (int)std::round(g.dx);
  const int gdy = (int)std::round(g.dy);
  const size_t P = g.pattern.size();
  std::vector<Coord> p1(P);
  const std::vector<double> steps = rotation_steps(z);
  for (double drot : steps) {
    const double total_rot = g.refrot + g.drot + drot;
    const double c1 = std::cos(total_rot), s1 = std::sin(total_rot);
    for (size_t i = 0; i < P; ++i) rotate_pixel(g.pattern[i], c1, s1, &p1[i].dx, &p1[i].dy);
    for (int u = -z.left; u <= z.right; ++u) {
      for (int v = -z.up; v <= z.down; ++v) {
        double mean1 = 0.0, C0C1 = 0.0, C1C1 = 0.0;
        for (size_t i = 0; i < P; ++i)
          mean1 += t.pix(t.icur_idx, p1[i].dx + g.refx + u + gdx, p1[i].dy + g.refy + v + gdy);
        mean1 /= (double)P;
        for (size_t i = 0; i < P; ++i) {
          const double d1 = t.pix(t.icur_idx, p1[i].dx + g.refx + u + gdx, p1[i].dy + g.refy + v + gdy) - mean1;
          C0C1 += (t.pix(t.iref_idx, g.pattern0[i].dx + g.refx, g.pattern0[i].dy + g.refy) - g.mean0) * d1;
          C1C1 += d1 * d1;
        }
        const double ncc = C0C1 / std::sqrt(g.C0C0 * C1C1);
        if (r.best < ncc) {
          r.best = ncc;
          r.best_u = u;
          r.best_v = v;
          r.best_drot = drot;
        }
        // diagnostic (not part of the reference): the best NCC and the best
        // value distinct from it.  Bit-identical values (identical rotated
        // patterns at neighbouring rotation steps) are resolved by iteration
        // order in every implementation and are not near-ties.
        if (ncc > r.top1) {
          r.top2 = r.top1;
          r.top1 = ncc;
        } else if (ncc < r.top1 && ncc > r.top2) {
          r.top2 = ncc;
        }
      }
    }
  }
  return r;
}

void apply_accept(Grain& g, const SearchResult& r) {
  // src/p-tracker.cpp:735-742 (identical in the rescue variants)
  const int gdx = (int)std::round(g.dx);
  const int gdy = (int)std::round(g.dy);
  const double rest_dx = g.dx - gdx;
  const double rest_dy = g.dy - gdy;
  g.upix = (double)r.best_u - rest_dx;
  g.vpix = (double)r.best_v - rest_dy;
  g.rot_inc = r.best_drot;
  g.dx = gdx + (double)r.best_u;
  g.dy = gdy + (double)r.best_v;
  g.drot += r.best_drot;
}

// follow_pattern_pixel, src/p-tracker.cpp:659-743
bool pixel_one(Tracker& t, Grain& g) {
  g.upix = g.vpix = g.rot_inc = 0.0;
  SearchResult r = search(t, g, t.zone[0]);
  g.top1 = r.top1;
  g.top2 = r.top2;
  g.NCC = r.best;
  g.NCC_rescue = r.best;
  if (r.best < t.NCC_min) return true;  // queued for rescue
  apply_accept(g, r);
  return false;
}

// follow_pattern_rescue_pixel, src/p-tracker.cpp:745-881
bool rescue_one(Tracker& t, Grain& g) {
  SearchResult r = search(t, g, t.zone[1]);
  g.top1 = r.top1;
  g.top2 = r.top2;
  g.NCC_rescue = r.best;
  if (r.best < t.NCC_min_super) return true;  // queued for super-rescue
  apply_accept(g, r);
  return false;
}

// follow_pattern_super_rescue_pixel, src/p-tracker.cpp:883-1016
void super_rescue_one(Tracker& t, Grain& g) {
  SearchResult r = search(t, g, t.zone[2]);
  g.top1 = r.top1;
  g.top2 = r.top2;
  g.NCC_rescue = r.best;
  if (r.best > t.NCC_min_super) apply_accept(g, r);
}

// --- interpolators, src/interpol.cpp:19-144 (rows of the 4x4 block are x)
inline double lin1(const double p[2], double x) { return (p[1] - p[0]) * x + p[0]; }

inline double cubic1(const double p[4], double x) {
  double f0 = p[1];
  double f1 = p[2];
  double fp0 = 0.5 * (p[2] - p[0]);
  double fp1 = 0.5 * (p[3] - p[1]);
  double d = f0;
  double c = fp0;
  double b = -3.0 * f0 + 3.0 * f1 - 2.0 * fp0 - fp1;
  double a = 2.0 * f0 - 2.0 * f1 + fp0 + fp1;
  double x2 = x * x;
  return (a * x2 * x + b * x2 + c * x + d);
}

inline double quintic1(const double p[4], double x) {
  double f0 = p[1];
  double f1 = p[2];
  double fp0 = 0.5 * (p[2] - p[0]);
  double fp1 = 0.5 * (p[3] - p[1]);
  double fs0 = p[0] - 2.0 * p[1] + p[2];
  double fs1 = p[1] - 2.0 * p[2] + p[3];
  double f = f0;
  double e = fp0;
  double d = 0.5 * fs0;
  double c = 0.5 * (fs1 - 8.0 * fp1 + 20.0 * f1 - 3.0 * fs0 - 12.0 * fp0 - 20.0 * f0);
  double b = 15.0 * f0 + 8.0 * fp0 + 1.5 * fs0 - 15.0 * f1 + 7.0 * fp1 - fs1;
  double a = f1 - b - c - 0.5 * fs0 - fp0 - f0;
  double x2 = x * x;
  double x4 = x2 * x2;
  return (a * x4 * x + b * x4 + c * x2 * x + d * x2 + e * x + f);
}

double interp(const Tracker& t, int kind, int slot, double x, double y) {
  const int ix = (int)std::floor(x);
  const int iy = (int)std::floor(y);
  const double x01 = x - (double)ix;
  const double y01 = y - (double)iy;
  if (kind == 0) {
    double p0[2] = {t.pix(slot, ix, iy), t.pix(slot, ix, iy + 1)};
    double p1[2] = {t.pix(slot, ix + 1, iy), t.pix(slot, ix + 1, iy + 1)};
    double arr[2] = {lin1(p0, y01), lin1(p1, y01)};
    return lin1(arr, x01);
  }
  double p[4][4];
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) p[i][j] = t.pix(slot, ix - 1 + i, iy - 1 + j);
  double arr[4];
  if (kind == 2) {
    for (int i = 0; i < 4; ++i) arr[i] = quintic1(p[i], y01);
    return quintic1(arr, x01);
  }
  for (int i = 0; i < 4; ++i) arr[i] = cubic1(p[i], y01);
  return cubic1(arr, x01);
}

// NCC_to_minimize_xyR, src/p-tracker.cpp:1018-1088
double objective(const Tracker& t, const Grain& g, const double* X) {
  const size_t P = g.pattern0.size();
  const double inv_num_pix = 1.0 / (double)P;
  const double xpix1 = (double)g.refx + (double)g.dx + X[0];
  const double ypix1 = (double)g.refy + (double)g.dy + X[1];
  const double rot = g.drot + X[2];
  const double c1 = std::cos(rot), s1 = std::sin(rot);
  std::vector<double> vals(P);
  double mean1 = 0.0;
  for (size_t i = 0; i < P; ++i) {
    const double x = g.pattern0[i].dx, y = g.pattern0[i].dy;
    const double xs = xpix1 + c1 * x + s1 * y;
    const double ys = ypix1 - s1 * x + c1 * y;
    vals[i] = interp(t, t.interpolator, t.icur_idx, xs, ys);
    mean1 += vals[i];
  }
  mean1 *= inv_num_pix;
  double C0C1 = 0.0, C1C1 = 0.0;
  for (size_t i = 0; i < P; ++i) {
    const double d1 = vals[i] - mean1;
    const double d0 = t.pix(t.iref_idx, g.refx + g.pattern0[i].dx, g.refy + g.pattern0[i].dy) - g.mean0;
    C0C1 += d0 * d1;
    C1C1 += d1 * d1;
  }
  const double NCC = C0C1 / std::sqrt(g.C0C0 * C1C1);
  double W = 1.0;
  const double disp = std::sqrt(X[0] * X[0] + X[1] * X[1]);
  if (disp > t.subpix_displacement_max) W = t.overflow_stiffness * (disp - t.subpix_displacement_max) + 1.0;
  return (1.0 - NCC) * W;
}

// Analytic gradient of the objective (no reference counterpart): chain rule
// through the cubic interpolant and the rotation, FP64 throughout.  Used as the
// FP64 CPU reference gradient for the adjoint kernel.  Cubic interpolator only.
double objective_grad(const Tracker& t, const Grain& g, const double* X, double* grad) {
  const size_t P = g.pattern0.size();
  const double xpix1 = (double)g.refx + (double)g.dx + X[0];
  const double ypix1 = (double)g.refy + (double)g.dy + X[1];
  const double rot = g.drot + X[2];
  const double c1 = std::cos(rot), s1 = std::sin(rot);
  std::vector<double> v(P), gx(P), gy(P), gr(P), a(P);
  double mean1 = 0.0;
  for (size_t i = 0; i < P; ++i) {
    const double x = g.pattern0[i].dx, y = g.pattern0[i].dy;
    const double xs = xpix1 + c1 * x + s1 * y;
    const double ys = ypix1 - s1 * x + c1 * y;
    const int ix = (int)std::floor(xs), iy = (int)std::floor(ys);
    const double tx = xs - ix, ty = ys - iy;
    // Catmull-Rom weights and their derivatives
    double wx[4], wy[4], dwx[4], dwy[4];
    auto wts = [](double s, double* w, double* dw) {
      const double s2 = s * s, s3 = s2 * s;
      w[0] = -0.5 * s3 + s2 - 0.5 * s;
      w[1] = 1.5 * s3 - 2.5 * s2 + 1.0;
      w[2] = -1.5 * s3 + 2.0 * s2 + 0.5 * s;
      w[3] = 0.5 * s3 - 0.5 * s2;
      dw[0] = -1.5 * s2 + 2.0 * s - 0.5;
      dw[1] = 4.5 * s2 - 5.0 * s;
      dw[2] = -4.5 * s2 + 4.0 * s + 0.5;
      dw[3] = 1.5 * s2 - s;
    };
    wts(tx, wx, dwx);
    wts(ty, wy, dwy);
    double val = 0, dvx = 0, dvy = 0;
    for (int ii = 0; ii < 4; ++ii)
      for (int jj = 0; jj < 4; ++jj) {
        const double pv = t.pix(t.icur_idx, ix - 1 + ii, iy - 1 + jj);
        val += wx[ii] * wy[jj] * pv;
        dvx += dwx[ii] * wy[jj] * pv;
        dvy += wx[ii] * dwy[jj] * pv;
      }
    v[i] = val;
    gx[i] = dvx;
    gy[i] = dvy;
    // d(xs)/d(rot) = -s1 x + c1 y ; d(ys)/d(rot) = -c1 x - s1 y
    gr[i] = dvx * (-s1 * x + c1 * y) + dvy * (-c1 * x - s1 * y);
    mean1 += val;
    a[i] = t.pix(t.iref_idx, g.refx + g.pattern0[i].dx, g.refy + g.pattern0[i].dy) - g.mean0;
  }
  mean1 /= (double)P;
  double C01 = 0, C11 = 0;
  for (size_t i = 0; i < P; ++i) {
    const double b = v[i] - mean1;
    C01 += a[i] * b;
    C11 += b * b;
  }
  const double den = std::sqrt(g.C0C0 * C11);
  const double ncc = C01 / den;
  // dNCC/dv_i = (a_i - (C01/C11) b_i) / den   (the mean term cancels: sum a = sum b = 0)
  double G[3] = {0, 0, 0};
  for (size_t i = 0; i < P; ++i) {
    const double b = v[i] - mean1;
    const double dn = (a[i] - (C01 / C11) * b) / den;
    G[0] += dn * gx[i];
    G[1] += dn * gy[i];
    G[2] += dn * gr[i];
  }
  grad[0] = -G[0];
  grad[1] = -G[1];
  grad[2] = -G[2];
  return 1.0 - ncc;
}

// follow_pattern_subpixel_xyR, src/p-tracker.cpp:1090-1128
void subpixel_one(Tracker& t, Grain& g) {
  struct Func {
    const Tracker* t;
    const Grain* g;
    double operator()(std::vector<double>& X) const { return objective(*t, *g, X.data()); }
  } f{&t, &g};
  std::vector<double> X(3, 0.0), DX(t.init_dir, t.init_dir + 3);
  ptk_oracle::Powell<Func> powell(f, t.subpix_tol);
  X = powell.minimize(X, DX);
  g.NCC_subpix = 1.0 - powell.fret;
  g.upix += X[0];
  g.vpix += X[1];
  g.rot_inc += X[2];
  g.dx += X[0];
  g.dy += X[1];
  g.drot += X[2];
}

// undistor, src/distortion_correction.cpp:20-61 (Brown K1-K3, P1-P3 + parallax)
void undistor(const double* X, double xd, double yd, double* xu_out, double* yu_out) {
  double Xc = X[0], Yc = X[1], K1 = X[2], K2 = X[3], K3 = X[4], P1 = X[5], P2 = X[6], P3 = X[7];
  double dx = xd - Xc;
  double dy = yd - Yc;
  double r2 = dx * dx + dy * dy;
  double r4 = r2 * r2;
  double r6 = r4 * r2;
  double xu = xd + dx * (K1 * r2 + K2 * r4 + K3 * r6) + (P1 * (r2 + 2.0 * dx * dx) + 2.0 * P2 * dx * dy) * (1.0 + P3 * r2);
  double yu = yd + dy * (K1 * r2 + K2 * r4 + K3 * r6) + (2.0 * P1 * dx * dy + P2 * (r2 + 2.0 * dy * dy)) * (1.0 + P3 * r2);
  double Xcp = X[8], Ycp = X[9], theta1 = X[10], parallax1 = X[11], theta2 = X[12], parallax2 = X[13];
  double nx1 = std::cos(theta1);
  double ny1 = -std::sin(theta1);
  double nx2 = -std::sin(theta2);
  double ny2 = std::cos(theta2);
  double dX = xu - Xcp;
  double dY = yu - Ycp;
  double S1 = (1.0 + parallax1) * (dX * nx1 + dY * ny1);
  double S2 = (1.0 + parallax2) * (dX * nx2 + dY * ny2);
  *xu_out = Xcp + S1 * nx1 + S2 * nx2;
  *yu_out = Ycp + S1 * ny1 + S2 * ny2;
}

}  // namespace

// ---------------------------------------------------------------------------
extern "C" {

void* orc_create(int dimx, int dimy) {
  Tracker* t = new Tracker();
  t->dimx = dimx;
  t->dimy = dimy;
  t->image[0].assign((size_t)dimx * dimy, 0);
  t->image[1].assign((size_t)dimx * dimy, 0);
  return t;
}

void orc_destroy(void* p) { delete static_cast<Tracker*>(p); }

void orc_set_threads(void* p, int n) { static_cast<Tracker*>(p)->nthreads = n < 1 ? 1 : n; }

void orc_load_first(void* p, const uint16_t* img) {
  Tracker* t = static_cast<Tracker*>(p);
  std::memcpy(t->image[t->iref_idx].data(), img, sizeof(uint16_t) * t->image[0].size());
  std::memcpy(t->image[t->icur_idx].data(), img, sizeof(uint16_t) * t->image[0].size());
}

void orc_load_reference(void* p, const uint16_t* img) {
  Tracker* t = static_cast<Tracker*>(p);
  std::memcpy(t->image[t->iref_idx].data(), img, sizeof(uint16_t) * t->image[0].size());
}

void orc_load_current(void* p, const uint16_t* img) {
  Tracker* t = static_cast<Tracker*>(p);
  std::memcpy(t->image[t->icur_idx].data(), img, sizeof(uint16_t) * t->image[0].size());
}

void orc_get_indices(void* p, int* iref_idx, int* icur_idx, int* iref) {
  Tracker* t = static_cast<Tracker*>(p);
  *iref_idx = t->iref_idx;
  *icur_idx = t->icur_idx;
  *iref = t->iref;
}

void orc_set_grains(void* p, int n, const double* rec13, const uint8_t* masked) {
  Tracker* t = static_cast<Tracker*>(p);
  std::vector<Grain> old;
  old.swap(t->grain);
  t->grain.resize(n);
  for (int i = 0; i < n; ++i) {
    const double* r = rec13 + 13 * (size_t)i;
    Grain& g = t->grain[i];
    if (i < (int)old.size()) g.pattern = old[i].pattern;  // keep patterns set earlier
    g.refx = (int)r[0];
    g.refy = (int)r[1];
    g.refrot = r[2];
    g.radius = r[3];
    g.dx = r[4];
    g.dy = r[5];
    g.drot = r[6];
    g.upix = r[7];
    g.vpix = r[8];
    g.rot_inc = r[9];
    g.NCC = r[10];
    g.NCC_rescue = r[11];
    g.NCC_subpix = r[12];
    g.masked = masked ? masked[i] != 0 : false;
  }
  t->require_precomputations = true;
}

void orc_get_grains(void* p, double* rec13) {
  Tracker* t = static_cast<Tracker*>(p);
  for (size_t i = 0; i < t->grain.size(); ++i) {
    double* r = rec13 + 13 * i;
    const Grain& g = t->grain[i];
    r[0] = g.refx;
    r[1] = g.refy;
    r[2] = g.refrot;
    r[3] = g.radius;
    r[4] = g.dx;
    r[5] = g.dy;
    r[6] = g.drot;
    r[7] = g.upix;
    r[8] = g.vpix;
    r[9] = g.rot_inc;
    r[10] = g.NCC;
    r[11] = g.NCC_rescue;
    r[12] = g.NCC_subpix;
  }
}

void orc_get_precomp(void* p, double* mean0, double* C0C0) {
  Tracker* t = static_cast<Tracker*>(p);
  for (size_t i = 0; i < t->grain.size(); ++i) {
    mean0[i] = t->grain[i].mean0;
    C0C0[i] = t->grain[i].C0C0;
  }
}

void orc_get_top2(void* p, double* top12) {
  Tracker* t = static_cast<Tracker*>(p);
  for (size_t i = 0; i < t->grain.size(); ++i) {
    top12[2 * i] = t->grain[i].top1;
    top12[2 * i + 1] = t->grain[i].top2;
  }
}

void orc_set_pattern(void* p, int ig, int npts, const int32_t* xy) {
  Tracker* t = static_cast<Tracker*>(p);
  Grain& g = t->grain[ig];
  g.pattern.resize(npts);
  for (int i = 0; i < npts; ++i) {
    g.pattern[i].dx = xy[2 * i];
    g.pattern[i].dy = xy[2 * i + 1];
  }
  t->require_precomputations = true;
}

// make_circ_pattern / make_ring_pattern / make_rect_pattern,
// src/p-tracker.cpp:1369-1442.  kind: 0 circ(a), 1 ring(a, b), 2 rect(a, b).
void orc_make_pattern(void* p, int ig, int kind, int a, int b) {
  Tracker* t = static_cast<Tracker*>(p);
  std::vector<Coord>& pat = t->grain[ig].pattern;
  pat.clear();
  if (kind == 2) {
    for (int dy = -b; dy <= b; ++dy)
      for (int dx = -a; dx <= a; ++dx) pat.push_back(Coord{dx, dy});
  } else {
    const int rout = kind == 0 ? a : b;
    for (int dy = -rout; dy <= rout; ++dy)
      for (int dx = -rout; dx <= rout; ++dx) {
        double dst = std::sqrt((double)dx * (double)dx + (double)dy * (double)dy);
        bool in = kind == 0 ? dst <= (double)a : (dst <= (double)b && dst >= (double)a);
        if (in) pat.push_back(Coord{dx, dy});
      }
  }
  t->require_precomputations = true;
}

int orc_pattern_size(void* p, int ig) { return (int)static_cast<Tracker*>(p)->grain[ig].pattern.size(); }

void orc_get_pattern(void* p, int ig, int which, int32_t* xy) {
  const Grain& g = static_cast<Tracker*>(p)->grain[ig];
  const std::vector<Coord>& v = which == 0 ? g.pattern : g.pattern0;
  for (size_t i = 0; i < v.size(); ++i) {
    xy[2 * i] = v[i].dx;
    xy[2 * i + 1] = v[i].dy;
  }
}

void orc_set_zone(void* p, int level, int left, int right, int up, int down, int num_rot, double inc_rot) {
  Tracker* t = static_cast<Tracker*>(p);
  t->zone[level] = Zone{left, right, up, down, num_rot, inc_rot};
}

int orc_set_param(void* p, const char* key, double v) {
  Tracker* t = static_cast<Tracker*>(p);
  std::string k(key);
  if (k == "NCC_min") t->NCC_min = v;
  else if (k == "NCC_min_super") t->NCC_min_super = v;
  else if (k == "rescue_level") t->rescue_level = (int)v;
  else if (k == "subpixel") t->subpixel = (int)v;
  else if (k == "subpix_tol") t->subpix_tol = v;
  else if (k == "initial_direction_dx") t->init_dir[0] = v;
  else if (k == "initial_direction_dy") t->init_dir[1] = v;
  else if (k == "initial_direction_dr") t->init_dir[2] = v;
  else if (k == "overflow_stiffness") t->overflow_stiffness = v;
  else if (k == "subpix_displacement_max") t->subpix_displacement_max = v;
  else if (k == "image_interpolator") t->interpolator = (int)v;
  else if (k == "iref") t->iref = (int)v;
  else if (k == "iraz") t->iraz = (int)v;
  else if (k == "use_neighbour_list" || k == "neighbour_dist_pix" || k == "period_rebuild_neighbour_list") {
    // accepted, no effect: the neighbour exclusion is inert in the reference
  } else return -1;
  return 0;
}

int orc_rotation_steps(double inc_rot, int num_rot, double* out, int cap) {
  Zone z;
  z.inc_rot = inc_rot;
  z.num_rot = num_rot;
  std::vector<double> s = rotation_steps(z);
  for (size_t i = 0; i < s.size() && (int)i < cap; ++i) out[i] = s[i];
  return (int)s.size();
}

void orc_precompute(void* p) { precompute(*static_cast<Tracker*>(p)); }

// Pixel stage, src/p-tracker.cpp:471-484.  Returns the rescue count.
int orc_pixel_all(void* p) {
  Tracker* t = static_cast<Tracker*>(p);
  const int n = (int)t->grain.size();
  std::vector<uint8_t> flag(n, 0);
#pragma omp parallel for schedule(dynamic) num_threads(t->nthreads)
  for (int i = 0; i < n; ++i) {
    Grain& g = t->grain[i];
    g.NCC = g.NCC_rescue = g.NCC_subpix = 0.0;  // grain_type_2D::reset
    g.dx_prev = g.dx;                            // grain_type_2D::backup
    g.dy_prev = g.dy;
    g.drot_prev = g.drot;
    if (g.masked) continue;
    flag[i] = pixel_one(*t, g) ? 1 : 0;
  }
  // The reference appends under omp critical (arrival order); the order of
  // the list does not affect results, so it is kept ascending here.
  t->rescued.clear();
  t->super_rescued.clear();
  for (int i = 0; i < n; ++i)
    if (flag[i]) t->rescued.push_back(i);
  return (int)t->rescued.size();
}

int orc_rescue_all(void* p) {
  Tracker* t = static_cast<Tracker*>(p);
  const int n = (int)t->rescued.size();
  std::vector<uint8_t> flag(n, 0);
#pragma omp parallel for schedule(dynamic) num_threads(t->nthreads)
  for (int k = 0; k < n; ++k) flag[k] = rescue_one(*t, t->grain[t->rescued[k]]) ? 1 : 0;
  t->super_rescued.clear();
  for (int k = 0; k < n; ++k)
    if (flag[k]) t->super_rescued.push_back(t->rescued[k]);
  return (int)t->super_rescued.size();
}

void orc_super_rescue_all(void* p) {
  Tracker* t = static_cast<Tracker*>(p);
  const int n = (int)t->super_rescued.size();
#pragma omp parallel for schedule(dynamic) num_threads(t->nthreads)
  for (int k = 0; k < n; ++k) super_rescue_one(*t, t->grain[t->super_rescued[k]]);
}

int orc_get_lists(void* p, int* rescued, int* super_rescued, int* n_super) {
  Tracker* t = static_cast<Tracker*>(p);
  for (size_t i = 0; i < t->rescued.size(); ++i) rescued[i] = t->rescued[i];
  for (size_t i = 0; i < t->super_rescued.size(); ++i) super_rescued[i] = t->super_rescued[i];
  *n_super = (int)t->super_rescued.size();
  return (int)t->rescued.size();
}

void orc_subpixel_all(void* p) {
  Tracker* t = static_cast<Tracker*>(p);
  const int n = (int)t->grain.size();
#pragma omp parallel for schedule(dynamic) num_threads(t->nthreads)
  for (int i = 0; i < n; ++i)
    if (!t->grain[i].masked) subpixel_one(*t, t->grain[i]);
}

// src/p-tracker.cpp:577-611
void orc_end_frame(void* p, int num_image) {
  Tracker* t = static_cast<Tracker*>(p);
  for (Grain& g : t->grain) {
    g.upix = g.dx - g.dx_prev;
    g.vpix = g.dy - g.dy_prev;
    g.rot_inc = g.drot - g.drot_prev;
  }
  if (num_image - t->iref >= t->iraz) {
    std::swap(t->iref_idx, t->icur_idx);
    for (Grain& g : t->grain) {
      double actual = (double)g.refx + g.dx;
      g.refx = (int)std::round(actual);
      g.dx = actual - g.refx;
      actual = (double)g.refy + g.dy;
      g.refy = (int)std::round(actual);
      g.dy = actual - g.refy;
      g.refrot += g.drot;
      g.drot = 0.0;
    }
    t->iref = num_image;
    t->require_precomputations = true;
  }
}

void orc_track_frame(void* p, int num_image) {
  Tracker* t = static_cast<Tracker*>(p);
  if (t->require_precomputations) precompute(*t);
  t->rescued.clear();
  t->super_rescued.clear();
  if (t->rescue_level >= 0) orc_pixel_all(p);
  if (t->rescue_level >= 1) orc_rescue_all(p);
  if (t->rescue_level >= 2) orc_super_rescue_all(p);
  if (t->subpixel) orc_subpixel_all(p);
  orc_end_frame(p, num_image);
}

double orc_objective(void* p, int ig, const double* X3) {
  Tracker* t = static_cast<Tracker*>(p);
  return objective(*t, t->grain[ig], X3);
}

double orc_gradient(void* p, int ig, const double* X3, double* g3) {
  Tracker* t = static_cast<Tracker*>(p);
  return objective_grad(*t, t->grain[ig], X3, g3);
}

double orc_interp(void* p, int kind, int slot, double x, double y) {
  return interp(*static_cast<Tracker*>(p), kind, slot, x, y);
}

void orc_undistor(const double* params14, double xd, double yd, double* xu, double* yu) {
  undistor(params14, xd, yd, xu, yu);
}

// precompute_paires, src/distortion_correction.cpp:63-81: the pairs (i < j) of
// grains whose reference positions lie dmin .. dmax apart, i-major.  Writes at
// most cap pairs (i, j) and returns the count.
int64_t orc_disto_pairs(const int32_t* refx, const int32_t* refy, int n, double dmin, double dmax, int32_t* out,
                        int64_t cap) {
  int64_t np = 0;
  for (int i = 0; i < n; ++i) {
    const double xi = (double)refx[i], yi = (double)refy[i];
    for (int j = i + 1; j < n; ++j) {
      const double xij = (double)refx[j] - xi, yij = (double)refy[j] - yi;
      const double dij = std::sqrt(xij * xij + yij * yij);
      if (dij >= dmin && dij <= dmax) {
        if (np < cap) {
          out[2 * np] = i;
          out[2 * np + 1] = j;
        }
        ++np;
      }
    }
  }
  return np;
}

// The equiprojectivity criterion of correction_distortion
// (src/distortion_correction.cpp:249-290 for POWELL, with A1 and B1 the
// undistorted reference positions; :318-351 for POWELL_ITER, with A1 and B1
// taken from orig): sum over images 1.. and pairs of err^2, where
// err = AB_unit . ((B2 - B1) - (A2 - A1)); pairs with a subpixel NCC below
// NCC_min on either grain are skipped (their fvec entry is 0).
// dx, dy, ncc: [image - 1][grain].
double orc_disto_objective(const double* X, const int32_t* refx, const int32_t* refy, const double* origx,
                           const double* origy, int n, int nimg1, const double* dx, const double* dy,
                           const double* ncc, double NCC_min, const int32_t* pairs, int64_t npairs, int use_orig,
                           double* fvec) {
  double val = 0.0;
  for (int im = 0; im < nimg1; ++im) {
    for (int64_t il = 0; il < npairs; ++il) {
      const int i = pairs[2 * il], j = pairs[2 * il + 1];
      if (fvec) fvec[(size_t)im * npairs + il] = 0.0;
      if (ncc[(size_t)im * n + i] < NCC_min || ncc[(size_t)im * n + j] < NCC_min) continue;
      double A1x, A1y, A2x, A2y, B1x, B1y, B2x, B2y;
      if (use_orig) {
        A1x = origx[i];
        A1y = origy[i];
        B1x = origx[j];
        B1y = origy[j];
      } else {
        undistor(X, (double)refx[i], (double)refy[i], &A1x, &A1y);
        undistor(X, (double)refx[j], (double)refy[j], &B1x, &B1y);
      }
      undistor(X, (double)refx[i] + dx[(size_t)im * n + i], (double)refy[i] + dy[(size_t)im * n + i], &A2x, &A2y);
      undistor(X, (double)refx[j] + dx[(size_t)im * n + j], (double)refy[j] + dy[(size_t)im * n + j], &B2x, &B2y);
      double ABx = B1x - A1x, ABy = B1y - A1y;
      const double AB = std::sqrt(ABx * ABx + ABy * ABy);
      ABx /= AB;
      ABy /= AB;
      const double BBx = B2x - B1x, BBy = B2y - B1y;
      const double AAx = A2x - A1x, AAy = A2y - A1y;
      const double err = (ABx * (BBx - AAx)) + (ABy * (BBy - AAy));
      if (fvec) fvec[(size_t)im * npairs + il] = err;
      val += err * err;
    }
  }
  return val;
}

// The minimisation of correction_distortion (src/distortion_correction.cpp:
// 222-386): default centres (negative entries -> frame centre, :222-226), then
// algo 0 (POWELL): one Powell minimisation (ftol 1e-12, initial directions the
// perturbations); algo 1 (POWELL_ITER): num_iter minimisations, each followed
// by re-anchoring A1/B1 and the displacements on the undistorted reference
// positions.  history (optional, num_iter x 15): index and parameters after
// each iteration.  dx, dy are updated in place by POWELL_ITER.
void orc_disto_fit(double* X14, const double* perturb14, int algo, int num_iter, int dimx, int dimy,
                   const int32_t* refx, const int32_t* refy, int n, int nimg1, double* dx, double* dy,
                   const double* ncc, double NCC_min, const int32_t* pairs, int64_t npairs, double* index_ini,
                   double* index_end, double* history) {
  std::vector<double> X(X14, X14 + 14), DX(perturb14, perturb14 + 14);
  if (X[0] < 0.0) X[0] = 0.5 * (double)dimx;
  if (X[1] < 0.0) X[1] = 0.5 * (double)dimy;
  if (X[8] < 0.0) X[8] = 0.5 * (double)dimx;
  if (X[9] < 0.0) X[9] = 0.5 * (double)dimy;
  std::vector<double> ox(n), oy(n);
  for (int g = 0; g < n; ++g) {
    ox[g] = (double)refx[g];
    oy[g] = (double)refy[g];
  }
  const int use_orig = algo == 1 ? 1 : 0;
  struct F {
    const int32_t *rx, *ry;
    std::vector<double>*ox, *oy;
    int n, nimg1;
    double *dx, *dy;
    const double* ncc;
    double NCC_min;
    const int32_t* pairs;
    int64_t npairs;
    int use_orig;
    double operator()(std::vector<double>& X) {
      return orc_disto_objective(X.data(), rx, ry, ox->data(), oy->data(), n, nimg1, dx, dy, ncc, NCC_min, pairs,
                                 npairs, use_orig, nullptr);
    }
  } func{refx, refy, &ox, &oy, n, nimg1, dx, dy, ncc, NCC_min, pairs, npairs, use_orig};
  const double nb = (double)nimg1;
  ptk_oracle::Powell<F> powell(func, 1e-12);
  *index_ini = func(X) / nb;
  if (algo == 1) {
    std::vector<double> dx0(dx, dx + (size_t)nimg1 * n), dy0(dy, dy + (size_t)nimg1 * n);
    for (int it = 1; it <= num_iter; ++it) {
      X = powell.minimize(X, DX);
      const double idx = func(X) / nb;
      if (history) {
        history[(size_t)(it - 1) * 15] = idx;
        for (int k = 0; k < 14; ++k) history[(size_t)(it - 1) * 15 + 1 + k] = X[k];
      }
      for (int g = 0; g < n; ++g) {
        double xu, yu;
        undistor(X.data(), (double)refx[g], (double)refy[g], &xu, &yu);
        const double dxc = xu - (double)refx[g], dyc = yu - (double)refy[g];
        for (int im = 0; im < nimg1; ++im) {
          dx[(size_t)im * n + g] = dx0[(size_t)im * n + g] + dxc;
          dy[(size_t)im * n + g] = dy0[(size_t)im * n + g] + dyc;
        }
        ox[g] = xu;
        oy[g] = yu;
      }
    }
  } else {
    X = powell.minimize(X, DX);
  }
  *index_end = func(X) / nb;
  for (int k = 0; k < 14; ++k) X14[k] = X[k];
}

// Inverse of undistor (no reference counterpart: the reference applies
// undistor to points only, src/distortion_correction.cpp:20-61).  Newton
// iteration on F(xd) = undistor(xd) - xu with a forward-difference Jacobian
// (step 1e-3 px), a fixed count of 8 iterations from xd = xu, so the device
// remap can follow the same sequence of FP64 operations.
void orc_distort_point(const double* X, double xu, double yu, double* xd_out, double* yd_out) {
  double xd = xu, yd = yu;
  const double h = 1e-3;
  for (int it = 0; it < 8; ++it) {
    double fx, fy, fx1, fy1, fx2, fy2;
    undistor(X, xd, yd, &fx, &fy);
    undistor(X, xd + h, yd, &fx1, &fy1);
    undistor(X, xd, yd + h, &fx2, &fy2);
    const double j11 = (fx1 - fx) / h, j21 = (fy1 - fy) / h;
    const double j12 = (fx2 - fx) / h, j22 = (fy2 - fy) / h;
    const double rx = fx - xu, ry = fy - yu;
    const double det = j11 * j22 - j12 * j21;
    xd = xd - (j22 * rx - j12 * ry) / det;
    yd = yd - (j11 * ry - j21 * rx) / det;
  }
  *xd_out = xd;
  *yd_out = yd;
}

// Undistortion remap of a whole frame: out(x, y) = cubic(src, distort(x, y)),
// rounded half up and clamped to [0, 65535]; pixels whose 4x4 cubic support
// leaves the frame are 0.
void orc_remap(const double* X, const uint16_t* src, int dimx, int dimy, uint16_t* out, int nthreads) {
  Tracker t;
  t.dimx = dimx;
  t.dimy = dimy;
  t.image[0].assign(src, src + (size_t)dimx * dimy);
#pragma omp parallel for schedule(static) num_threads(nthreads < 1 ? 1 : nthreads)
  for (int y = 0; y < dimy; ++y) {
    for (int x = 0; x < dimx; ++x) {
      double xd, yd;
      orc_distort_point(X, (double)x, (double)y, &xd, &yd);
      const int ix = (int)std::floor(xd), iy = (int)std::floor(yd);
      uint16_t v = 0;
      if (ix >= 1 && iy >= 1 && ix + 2 < dimx && iy + 2 < dimy) {
        double val = interp(t, 1, 0, xd, yd);
        double r = std::floor(val + 0.5);
        if (r < 0.0) r = 0.0;
        if (r > 65535.0) r = 65535.0;
        v = (uint16_t)r;
      }
      out[(size_t)y * dimx + x] = v;
    }
  }
}

int orc_save_grains(void* p, const char* path, const char* from_name, const char* to_name) {
  // save_grains, src/p-tracker.cpp:1313-1360 (13-column form)
  Tracker* t = static_cast<Tracker*>(p);
  std::ofstream f(path);
  if (!f) return -1;
  f << t->grain.size() << std::endl;
  for (const Grain& g : t->grain) {
    f << std::scientific << std::setprecision(15) << std::setw(6) << std::left << g.refx << ' ' << std::setw(6)
      << std::left << g.refy << ' ' << std::setw(23) << std::right << g.refrot << ' ' << std::setw(23) << std::right
      << g.radius << ' ' << std::setw(23) << std::right << g.dx << ' ' << std::setw(23) << std::right << g.dy << ' '
      << std::setw(23) << std::right << g.drot << ' ' << std::setw(23) << std::right << g.upix << ' ' << std::setw(23)
      << std::right << g.vpix << ' ' << std::setw(23) << std::right << g.rot_inc << ' ' << std::setw(23) << std::right
      << g.NCC << ' ' << std::setw(23) << std::right << g.NCC_rescue << ' ' << std::setw(23) << std::right
      << g.NCC_subpix << '\n';
  }
  f << std::endl;
  f << "#_FROM_image: " << from_name << '\n';
  f << "#___dateTime: " << "dateTime unknown" << '\n';
  f << "#___TO_image: " << to_name << '\n';
  f << "#___dateTime: " << "dateTime unknown" << '\n';
  f << std::flush;
  return 0;
}

// Grey frame from an unpacked RAW sensor mosaic (read_raw_image,
// src/p-tracker.cpp:288-372): -1 the floor of the 2x2 mean of the pixel and
// its right/lower neighbours, -2 the floor of the 1-2-1 x 1-2-1 / 16 weighted
// mean of the 3x3 block around it, -20 the raw value; neighbours are found
// in the flat raw array (index (left + x + i) + raw_width (top + y + j)).
// Then (:374-383) with rescale: floor((v - min) * (65535 / (max - min))).
// Returns 0, or -1 when a stencil index leaves the array or the mode is
// not one of the three; min_max receives the frame's MinGray/MaxGray.
int orc_raw_demosaic(const uint16_t* raw, int raw_width, int raw_height, int width, int height, int left, int top,
                     int mode, int rescale, uint16_t* out, uint16_t* min_max) {
  int lo = 0, hi = 0;
  static const double w2[2][2] = {{0.25, 0.25}, {0.25, 0.25}};
  static const double w3[3][3] = {{0.0625, 0.125, 0.0625}, {0.125, 0.25, 0.125}, {0.0625, 0.125, 0.0625}};
  if (mode == -1) {
    lo = 0;
    hi = 1;
  } else if (mode == -2) {
    lo = -1;
    hi = 1;
  } else if (mode != -20) {
    return -1;
  }
  const long long n = (long long)raw_width * raw_height;
  const long long first = (long long)(left + lo) + (long long)raw_width * (top + lo);
  const long long last = (long long)(left + width - 1 + hi) + (long long)raw_width * (top + height - 1 + hi);
  if (first < 0 || last >= n) return -1;
  unsigned mn = 65535, mx = 0;
  for (int y = 0; y < height; ++y) {
    for (int x = 0; x < width; ++x) {
      double v = 0.0;
      for (int j = lo; j <= hi; ++j)
        for (int i = lo; i <= hi; ++i) {
          const double w = mode == -1 ? w2[j][i] : mode == -2 ? w3[j + 1][i + 1] : 1.0;
          v += w * (double)raw[(long long)(left + x + i) + (long long)raw_width * (top + y + j)];
        }
      const uint16_t g = (uint16_t)(unsigned)std::floor(v);
      out[(size_t)y * width + x] = g;
      if (g < mn) mn = g;
      if (g > mx) mx = g;
    }
  }
  if (rescale && mx > mn) {
    const double fact = 65535.0 / (double)(int)(mx - mn);
    for (size_t k = 0; k < (size_t)width * height; ++k)
      out[k] = (uint16_t)std::floor((double)((int)out[k] - (int)mn) * fact);
  }
  if (min_max) {
    min_max[0] = (uint16_t)mn;
    min_max[1] = (uint16_t)mx;
  }
  return 0;
}

}  // extern "C"
