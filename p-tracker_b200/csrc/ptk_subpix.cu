// Subpixel refinement on sm_100a: the NCC objective through image
// interpolation, its adjoint gradient, and a per-grain Powell minimiser.
//
// The objective (objective_exact) follows the reference's FP64 operations
// (src/p-tracker.cpp:1018-1088, src/interpol.cpp:19-144) in their order and
// without FMA contraction (this file is compiled with -fmad=false): the
// interpolated values are computed in parallel, and its sums run over the
// pattern points in point order, rounded after every point, as the
// reference's loops round them; cos / sin come from ptk_crtrig.cuh.  Inside
// Powell the frame region under the grain is staged in shared memory.
//
// One CTA of kSubpixThreads refines one grain.  The Powell driver
// (follow_pattern_subpixel_xyR, src/p-tracker.cpp:1090-1128; the minimiser
// comes from the un-vendored toofus powell_nr3.hpp, src/p-tracker.hpp:51) runs
// redundantly on every thread with block-uniform control flow: each objective
// value is produced by a block reduction and broadcast, so every thread takes
// the same branches.  The algorithm is Powell's direction-set method with
// golden-ratio bracketing and Brent's parabolic line minimiser; its constants
// and tests match the CPU oracle's restatement exactly.
#include <climits>

#include "ptk_crtrig.cuh"
#include "ptk_internal.cuh"

namespace ptk {

namespace {

constexpr double kGold = 1.6180339887498949;
constexpr double kCGold = 0.3819660112501051;
constexpr double kLineRelTol = 1.0e-4;
constexpr double kLineAbsTol = 1.0e-10;
constexpr int kBracketMaxIter = 60;
constexpr int kBrentMaxIter = 100;
constexpr int kPowellMaxIter = 200;
constexpr double kTiny = 1.0e-25;

__device__ __forceinline__ double pixd(const FrameDev& f, int x, int y) {
  return (double)__ldg(&f.pix[(size_t)y * f.pitch + x]);
}

// CubicInterpolate, src/interpol.cpp:42-53
__device__ __forceinline__ double cubic1(double p0, double p1, double p2, double p3, double x) {
  const double f0 = p1, f1 = p2;
  const double fp0 = 0.5 * (p2 - p0);
  const double fp1 = 0.5 * (p3 - p1);
  const double d = f0, c = fp0;
  const double b = -3.0 * f0 + 3.0 * f1 - 2.0 * fp0 - fp1;
  const double a = 2.0 * f0 - 2.0 * f1 + fp0 + fp1;
  const double x2 = x * x;
  return (a * x2 * x + b * x2 + c * x + d);
}

// derivative of cubic1 with respect to x
__device__ __forceinline__ double cubic1_dx(double p0, double p1, double p2, double p3, double x) {
  const double f0 = p1, f1 = p2;
  const double fp0 = 0.5 * (p2 - p0);
  const double fp1 = 0.5 * (p3 - p1);
  const double c = fp0;
  const double b = -3.0 * f0 + 3.0 * f1 - 2.0 * fp0 - fp1;
  const double a = 2.0 * f0 - 2.0 * f1 + fp0 + fp1;
  return (3.0 * a * x * x + 2.0 * b * x + c);
}

// Catmull-Rom weight of control point k at x (cubic1 is linear in p)
__device__ __forceinline__ void cubic_weights(double x, double w[4]) {
  const double x2 = x * x, x3 = x2 * x;
  w[0] = -0.5 * x3 + x2 - 0.5 * x;
  w[1] = 1.5 * x3 - 2.5 * x2 + 1.0;
  w[2] = -1.5 * x3 + 2.0 * x2 + 0.5 * x;
  w[3] = 0.5 * x3 - 0.5 * x2;
}

// QuinticInterpolate, src/interpol.cpp:89-111
__device__ __forceinline__ double quintic1(double p0, double p1, double p2, double p3, double x) {
  const double f0 = p1, f1 = p2;
  const double fp0 = 0.5 * (p2 - p0);
  const double fp1 = 0.5 * (p3 - p1);
  const double fs0 = p0 - 2.0 * p1 + p2;
  const double fs1 = p1 - 2.0 * p2 + p3;
  const double f = f0, e = fp0, d = 0.5 * fs0;
  const double c = 0.5 * (fs1 - 8.0 * fp1 + 20.0 * f1 - 3.0 * fs0 - 12.0 * fp0 - 20.0 * f0);
  const double b = 15.0 * f0 + 8.0 * fp0 + 1.5 * fs0 - 15.0 * f1 + 7.0 * fp1 - fs1;
  const double a = f1 - b - c - 0.5 * fs0 - fp0 - f0;
  const double x2 = x * x, x4 = x2 * x2;
  return (a * x4 * x + b * x4 + c * x2 * x + d * x2 + e * x + f);
}

// image_interp*::getValue (src/interpol.cpp:21-39, 55-86, 113-144).  The
// reference reads out of bounds when the support leaves the frame; here the
// support is clamped into the frame and *clamped is set.
__device__ double interp(const FrameDev& f, int kind, double x, double y, bool* clamped) {
  int ix = (int)floor(x);
  int iy = (int)floor(y);
  const double x01 = x - (double)ix;
  const double y01 = y - (double)iy;
  const int lo = kind == PTK_INTERP_LINEAR ? 0 : 1;
  const int hi = kind == PTK_INTERP_LINEAR ? 1 : 2;
  if (ix - lo < 0 || iy - lo < 0 || ix + hi >= f.dimx || iy + hi >= f.dimy || !(x == x) || !(y == y)) {
    *clamped = true;
    ix = min(max(ix, lo), f.dimx - 1 - hi);
    iy = min(max(iy, lo), f.dimy - 1 - hi);
  }
  if (kind == PTK_INTERP_LINEAR) {
    const double a0 = pixd(f, ix, iy), a1 = pixd(f, ix, iy + 1);
    const double b0 = pixd(f, ix + 1, iy), b1 = pixd(f, ix + 1, iy + 1);
    const double r0 = (a1 - a0) * y01 + a0;
    const double r1 = (b1 - b0) * y01 + b0;
    return (r1 - r0) * x01 + r0;
  }
  double arr[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int xx = ix - 1 + i;
    const double q0 = pixd(f, xx, iy - 1), q1 = pixd(f, xx, iy), q2 = pixd(f, xx, iy + 1), q3 = pixd(f, xx, iy + 2);
    arr[i] = kind == PTK_INTERP_QUINTIC ? quintic1(q0, q1, q2, q3, y01) : cubic1(q0, q1, q2, q3, y01);
  }
  return kind == PTK_INTERP_QUINTIC ? quintic1(arr[0], arr[1], arr[2], arr[3], x01)
                                    : cubic1(arr[0], arr[1], arr[2], arr[3], x01);
}

// Cubic value and its partial derivatives at (x, y).
__device__ double interp_cubic_grad(const FrameDev& f, double x, double y, double* gx, double* gy, bool* clamped) {
  int ix = (int)floor(x);
  int iy = (int)floor(y);
  const double x01 = x - (double)ix;
  const double y01 = y - (double)iy;
  if (ix - 1 < 0 || iy - 1 < 0 || ix + 2 >= f.dimx || iy + 2 >= f.dimy || !(x == x) || !(y == y)) {
    *clamped = true;
    ix = min(max(ix, 1), f.dimx - 3);
    iy = min(max(iy, 1), f.dimy - 3);
  }
  double arr[4], darr[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int xx = ix - 1 + i;
    const double q0 = pixd(f, xx, iy - 1), q1 = pixd(f, xx, iy), q2 = pixd(f, xx, iy + 1), q3 = pixd(f, xx, iy + 2);
    arr[i] = cubic1(q0, q1, q2, q3, y01);
    darr[i] = cubic1_dx(q0, q1, q2, q3, y01);
  }
  double w[4];
  cubic_weights(x01, w);
  *gx = cubic1_dx(arr[0], arr[1], arr[2], arr[3], x01);
  *gy = w[0] * darr[0] + w[1] * darr[1] + w[2] * darr[2] + w[3] * darr[3];
  return cubic1(arr[0], arr[1], arr[2], arr[3], x01);
}

template <int NT>
__device__ __forceinline__ double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5;
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[w] = v;
  __syncthreads();
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < NT / 32; ++k) s += red[k];
  return s;
}

// Per-grain constants of the objective.
struct ObjGrain {
  int b, P;
  double xref, yref;  // (double)refcoord + d, in the reference's order
  double drot;
  double mean0, c0c0;
  int refx, refy;
};

// Current-frame region around a grain, staged once in shared memory for the
// objective evaluations of its Powell run (uint16, row-major).  w == 0: none.
struct Patch {
  const uint16_t* pix;
  int x0, y0, w, h;
};

__device__ __forceinline__ double patch_px(const Patch& pt, int x, int y) {
  return (double)pt.pix[(y - pt.y0) * pt.w + (x - pt.x0)];
}

// Per-grain state of the exact objective, in shared memory: the samples of
// the last evaluation, the reference values under pattern0_rotated, and the
// cosine and sine of the last rotation angle.
struct ExactObj {
  const uint16_t* w0;    // P reference values (staged)
  double* v;             // P interpolated values of the current evaluation (shared memory)
  double* bcast;         // 8 doubles: [0] the evaluation's NCC, [3] cos, [4] sin, [5] C0C0
  double inv_num_pix;    // 1 / P
  double last_rot, c1, s1;
};

// Sum of d0_i^2 over the grain's points in point order, each step rounded:
// C0C0 of do_precomputations (src/p-tracker.cpp:646-651).  One thread.
__device__ double c0c0_in_order(const uint16_t* w0, int P, double mean0) {
  double c = 0.0;
  for (int i = 0; i < P; ++i) {
    const double d0 = (double)w0[i] - mean0;
    c += d0 * d0;
  }
  return c;
}

// NCC_to_minimize_xyR (src/p-tracker.cpp:1018-1088): the sample positions
// xpix1 + c1 x + s1 y and ypix1 - s1 x + c1 y and the interpolators in the
// reference's operations and order, every product and sum rounded separately
// (this file is compiled without FMA contraction), cos / sin correctly
// rounded (ptk_crtrig.cuh) where the host C library is within an ulp.  The
// block's threads interpolate the points in parallel into shared memory; one
// thread then runs the reference's two loops over them in point order,
//     mean1 = (sum v) * (1 / P),  C0C1 = sum d0 (v - mean1),  C1C1 = sum (v - mean1)^2
// (d0 = I0 - mean0), each sum rounded after every point as the reference's
// loops round it, so that the value is the reference's bit for bit and Powell
// takes the reference's path even where the objective is flat.  Called by
// every thread of the block with the same X; returns the same value on every
// thread.
template <int NT>
__device__ double objective_exact(const GrainsDev& g, const FrameDev& cur, const SubpixParams& sp,
                                  const ObjGrain& o, const Patch& pt, ExactObj& ex, const double X[3],
                                  bool* clamped) {
  const int tid = threadIdx.x;
  const double xpix1 = o.xref + X[0];
  const double ypix1 = o.yref + X[1];
  const double rot = o.drot + X[2];
  if (!(rot == ex.last_rot)) {  // block-uniform: the line searches along x and y keep the angle
    if (tid == 0) ex.bcast[3] = crtrig::cr_cos(rot);
    if (tid == 32) ex.bcast[4] = crtrig::cr_sin(rot);
    __syncthreads();
    ex.c1 = ex.bcast[3];
    ex.s1 = ex.bcast[4];
    ex.last_rot = rot;
  }
  const double c1 = ex.c1, s1 = ex.s1;
  for (int i = tid; i < o.P; i += NT) {
    const short2 q = g.pat0[o.b + i];
    const double x = (double)q.x, y = (double)q.y;
    const double xs = xpix1 + c1 * x + s1 * y;
    const double ys = ypix1 - s1 * x + c1 * y;
    double v;
    const int ix = (int)floor(xs), iy = (int)floor(ys);
    if (sp.interp == PTK_INTERP_CUBIC && pt.w > 0 && ix - 1 >= pt.x0 && iy - 1 >= pt.y0 && ix + 2 < pt.x0 + pt.w &&
        iy + 2 < pt.y0 + pt.h) {
      const double x01 = xs - (double)ix, y01 = ys - (double)iy;
      double arr[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int xx = ix - 1 + k;
        arr[k] = cubic1(patch_px(pt, xx, iy - 1), patch_px(pt, xx, iy), patch_px(pt, xx, iy + 1),
                        patch_px(pt, xx, iy + 2), y01);
      }
      v = cubic1(arr[0], arr[1], arr[2], arr[3], x01);
    } else {
      v = interp(cur, sp.interp, xs, ys, clamped);
    }
    ex.v[i] = v;
  }
  __syncthreads();
  if (tid == 0) {
    const double* v = ex.v;
    double mean1 = 0.0;
#pragma unroll 8
    for (int i = 0; i < o.P; ++i) mean1 += v[i];
    mean1 *= ex.inv_num_pix;
    double c01 = 0.0, c11 = 0.0;
#pragma unroll 8
    for (int i = 0; i < o.P; ++i) {
      const double d1 = v[i] - mean1;
      const double d0 = (double)ex.w0[i] - o.mean0;
      c01 += d0 * d1;
      c11 += d1 * d1;
    }
    ex.bcast[0] = c01 / sqrt(o.c0c0 * c11);
  }
  __syncthreads();
  const double ncc = ex.bcast[0];
  double W = 1.0;
  const double disp = sqrt(X[0] * X[0] + X[1] * X[1]);
  if (disp > sp.disp_max) W = sp.stiffness * (disp - sp.disp_max) + 1.0;
  return (1.0 - ncc) * W;
}

// Once per grain: C0C0 as do_precomputations sums it (point order, each step
// rounded; src/p-tracker.cpp:646-651) in bcast[5].  Every thread must call it.
__device__ void grain_sums(const uint16_t* w0, int P, double mean0, double* bcast) {
  if (threadIdx.x == 0) bcast[5] = c0c0_in_order(w0, P, mean0);
  __syncthreads();
}

// Objective and its gradient (adjoint through the cubic interpolant and the
// rotation; no reference counterpart).  dNCC/dv_i = (a_i - (C01/C11) b_i) / den
// with a, b the centred reference and current values; the mean terms cancel.
template <int NT>
__device__ double objective_grad(const GrainsDev& g, const FrameDev& cur, const SubpixParams& sp,
                                 const ObjGrain& o, const double X[3], double* vals, double* red, double grad[3],
                                 bool* clamped) {
  const double xpix1 = o.xref + X[0];
  const double ypix1 = o.yref + X[1];
  const double rot = o.drot + X[2];
  double s1, c1;
  sincos(rot, &s1, &c1);
  double* gxs = vals + o.P;
  double* gys = vals + 2 * o.P;
  double sum = 0.0;
  for (int i = threadIdx.x; i < o.P; i += NT) {
    const short2 q = g.pat0[o.b + i];
    const double x = (double)q.x, y = (double)q.y;
    const double xs = xpix1 + c1 * x + s1 * y;
    const double ys = ypix1 - s1 * x + c1 * y;
    double gx, gy;
    const double v = interp_cubic_grad(cur, xs, ys, &gx, &gy, clamped);
    vals[i] = v;
    gxs[i] = gx;
    gys[i] = gy;
    sum += v;
  }
  const double mean1 = block_sum<NT>(sum, red) * (1.0 / (double)o.P);
  double c01 = 0.0, c11 = 0.0;
  for (int i = threadIdx.x; i < o.P; i += NT) {
    const double d1 = vals[i] - mean1;
    const double d0 = (double)g.w0[o.b + i] - o.mean0;
    c01 += d0 * d1;
    c11 += d1 * d1;
  }
  c01 = block_sum<NT>(c01, red);
  c11 = block_sum<NT>(c11, red);
  const double den = sqrt(o.c0c0 * c11);
  const double ncc = c01 / den;
  const double ratio = c01 / c11;
  double G0 = 0.0, G1 = 0.0, G2 = 0.0;
  for (int i = threadIdx.x; i < o.P; i += NT) {
    const short2 q = g.pat0[o.b + i];
    const double x = (double)q.x, y = (double)q.y;
    const double d1 = vals[i] - mean1;
    const double d0 = (double)g.w0[o.b + i] - o.mean0;
    const double dn = (d0 - ratio * d1) / den;
    G0 += dn * gxs[i];
    G1 += dn * gys[i];
    G2 += dn * (gxs[i] * (-s1 * x + c1 * y) + gys[i] * (-c1 * x - s1 * y));
  }
  G0 = block_sum<NT>(G0, red);
  G1 = block_sum<NT>(G1, red);
  G2 = block_sum<NT>(G2, red);
  double W = 1.0, dW0 = 0.0, dW1 = 0.0;
  const double disp = sqrt(X[0] * X[0] + X[1] * X[1]);
  if (disp > sp.disp_max) {
    W = sp.stiffness * (disp - sp.disp_max) + 1.0;
    dW0 = sp.stiffness * X[0] / disp;
    dW1 = sp.stiffness * X[1] / disp;
  }
  const double f0 = 1.0 - ncc;
  grad[0] = -G0 * W + f0 * dW0;
  grad[1] = -G1 * W + f0 * dW1;
  grad[2] = -G2 * W;
  return f0 * W;
}

__device__ ObjGrain load_grain(const GrainsDev& g, int gi) {
  ObjGrain o;
  o.b = g.pstart[gi];
  o.P = g.pstart[gi + 1] - o.b;
  o.refx = g.refx[gi];
  o.refy = g.refy[gi];
  o.xref = (double)o.refx + g.dx[gi];
  o.yref = (double)o.refy + g.dy[gi];
  o.drot = g.drot[gi];
  o.mean0 = g.mean0[gi];
  o.c0c0 = g.c0c0[gi];
  return o;
}

// --- Powell on the device, block-uniform ----------------------------------
template <int NT>
struct PowellEval {
  const GrainsDev* g;
  const FrameDev* cur;
  const SubpixParams* sp;
  const ObjGrain* o;
  const Patch* pt;
  ExactObj* ex;
  bool* clamped;
  int nfev;
  __device__ double operator()(const double X[3]) {
    ++nfev;
    return objective_exact<NT>(*g, *cur, *sp, *o, *pt, *ex, X, clamped);
  }
};

template <class F>
__device__ double line_minimize(F& f, const double p[3], const double dir[3], double* gmin) {
  auto g = [&](double alpha) {
    double t[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) t[j] = p[j] + alpha * dir[j];
    return f(t);
  };
  double a = 0.0, b = 1.0;
  double ga = g(a), gb = g(b);
  if (gb > ga) {
    double t = a;
    a = b;
    b = t;
    t = ga;
    ga = gb;
    gb = t;
  }
  double c = b + kGold * (b - a);
  double gc = g(c);
  int it = 0;
  while (gc < gb && it < kBracketMaxIter) {
    a = b;
    ga = gb;
    b = c;
    gb = gc;
    c = b + kGold * (b - a);
    gc = g(c);
    ++it;
  }
  double lo = a < c ? a : c;
  double hi = a < c ? c : a;
  double x = b, w = b, v = b;
  double fx = gb, fw = gb, fv = gb;
  double d = 0.0, e = 0.0;
  for (int iter = 0; iter < kBrentMaxIter; ++iter) {
    const double m = 0.5 * (lo + hi);
    const double tol1 = kLineRelTol * fabs(x) + kLineAbsTol;
    const double tol2 = 2.0 * tol1;
    if (fabs(x - m) <= tol2 - 0.5 * (hi - lo)) break;
    bool golden = true;
    if (fabs(e) > tol1) {
      double r = (x - w) * (fx - fv);
      double q = (x - v) * (fx - fw);
      double pp = (x - v) * q - (x - w) * r;
      q = 2.0 * (q - r);
      if (q > 0.0) pp = -pp;
      else q = -q;
      const double eprev = e;
      e = d;
      if (fabs(pp) < fabs(0.5 * q * eprev) && pp > q * (lo - x) && pp < q * (hi - x)) {
        d = pp / q;
        const double u = x + d;
        if (u - lo < tol2 || hi - u < tol2) d = (m - x) >= 0.0 ? tol1 : -tol1;
        golden = false;
      }
    }
    if (golden) {
      e = (x >= m) ? lo - x : hi - x;
      d = kCGold * e;
    }
    const double u = (fabs(d) >= tol1) ? x + d : x + (d >= 0.0 ? tol1 : -tol1);
    const double fu = g(u);
    if (fu <= fx) {
      if (u >= x) lo = x;
      else hi = x;
      v = w;
      fv = fw;
      w = x;
      fw = fx;
      x = u;
      fx = fu;
    } else {
      if (u < x) lo = u;
      else hi = u;
      if (fu <= fw || w == x) {
        v = w;
        fv = fw;
        w = u;
        fw = fu;
      } else if (fu <= fv || v == x || v == w) {
        v = u;
        fv = fu;
      }
    }
  }
  *gmin = fx;
  return x;
}

template <class F>
__device__ void powell_minimize(F& f, double p[3], const double step[3], double ftol, double* fret_out) {
  double dirs[3][3] = {{step[0], 0.0, 0.0}, {0.0, step[1], 0.0}, {0.0, 0.0, step[2]}};
  double pstart[3] = {p[0], p[1], p[2]};
  double fret = f(p);
  if (!isfinite(fret)) {  // flat window: NCC undefined, nothing to minimise
    *fret_out = fret;
    return;
  }
  for (int iter = 0; iter < kPowellMaxIter; ++iter) {
    const double fp = fret;
    int ibig = 0;
    double del = 0.0;
    for (int i = 0; i < 3; ++i) {
      const double fptt = fret;
      double gmin;
      const double alpha = line_minimize(f, p, dirs[i], &gmin);
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        dirs[i][j] *= alpha;
        p[j] += dirs[i][j];
      }
      fret = gmin;
      if (fptt - fret > del) {
        del = fptt - fret;
        ibig = i;
      }
    }
    if (2.0 * (fp - fret) <= ftol * (fabs(fp) + fabs(fret)) + kTiny) break;
    double ptt[3], xit[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      ptt[j] = 2.0 * p[j] - pstart[j];
      xit[j] = p[j] - pstart[j];
      pstart[j] = p[j];
    }
    const double fe = f(ptt);
    if (fe < fp) {
      const double t1 = fp - fret - del;
      const double t = 2.0 * (fp - 2.0 * fret + fe) * t1 * t1 - del * (fp - fe) * (fp - fe);
      if (t < 0.0) {
        double gmin;
        const double alpha = line_minimize(f, p, xit, &gmin);
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          xit[j] *= alpha;
          p[j] += xit[j];
        }
        fret = gmin;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          dirs[ibig][j] = dirs[2][j];
          dirs[2][j] = xit[j];
        }
      }
    }
  }
  *fret_out = fret;
}

}  // namespace

// Dynamic shared memory of the Powell kernel: the staged frame region (its
// cap in uint16 elements first), then per pattern point its uint16 reference
// value, then per pattern point the interpolated value of the current
// evaluation (double).
struct PowellSmem {
  int patch_cap;   // elements of the staged frame region
  int max_points;  // largest pattern of the grains
  size_t bytes;
};

__host__ __device__ inline size_t powell_vals_offset(int patch_cap) {
  return ((size_t)patch_cap * sizeof(uint16_t) + 15) & ~(size_t)15;
}

// bytes of the staged reference values, padded so that the interpolated
// values (doubles) after them stay 16-byte aligned
__host__ __device__ inline size_t powell_w0_bytes(int max_points) {
  return ((size_t)max_points * sizeof(uint16_t) + 15) & ~(size_t)15;
}

// follow_pattern_subpixel_xyR (src/p-tracker.cpp:1090-1128) for every grain,
// one block per grain, grains taken in `order` (decreasing pattern size) when
// given.
__global__ void __launch_bounds__(kSubpixThreads, 3) k_subpix_powell(GrainsDev g, FrameDev cur, SubpixParams sp,
                                                                       int patch_cap, int max_points,
                                                                       const int* order, const int* list_count) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ double bcast[8];
  __shared__ int s_clamped, s_bb[4];
  if (list_count && (int)blockIdx.x >= *list_count) return;
  const int gi = order ? order[blockIdx.x] : (int)blockIdx.x;
  if (g.masked[gi] || (g.flags[gi] & 3)) return;
  ObjGrain o = load_grain(g, gi);
  if (o.P <= 0 || o.P > max_points) return;
  // stage the frame region under the pattern, with a margin for the Powell steps
  if (threadIdx.x == 0) {
    s_clamped = 0;
    s_bb[0] = s_bb[2] = 1 << 30;
    s_bb[1] = s_bb[3] = -(1 << 30);
  }
  __syncthreads();
  uint16_t* s_patch = reinterpret_cast<uint16_t*>(smem);
  uint16_t* s_w0 = reinterpret_cast<uint16_t*>(smem + powell_vals_offset(patch_cap));
  double* s_v = reinterpret_cast<double*>(smem + powell_vals_offset(patch_cap) + powell_w0_bytes(max_points));
  int xmn = 1 << 30, xmx = -(1 << 30), ymn = 1 << 30, ymx = -(1 << 30);
  for (int i = threadIdx.x; i < o.P; i += kSubpixThreads) {
    const short2 q = g.pat0[o.b + i];
    xmn = min(xmn, (int)q.x);
    xmx = max(xmx, (int)q.x);
    ymn = min(ymn, (int)q.y);
    ymx = max(ymx, (int)q.y);
    s_w0[i] = g.w0[o.b + i];
  }
  atomicMin(&s_bb[0], xmn);
  atomicMax(&s_bb[1], xmx);
  atomicMin(&s_bb[2], ymn);
  atomicMax(&s_bb[3], ymx);
  __syncthreads();
  constexpr int kMargin = 6;
  const int cx = (int)floor(o.xref), cy = (int)floor(o.yref);
  int px0 = max(cx + s_bb[0] - kMargin, 0), py0 = max(cy + s_bb[2] - kMargin, 0);
  int px1 = min(cx + s_bb[1] + kMargin + 2, cur.dimx), py1 = min(cy + s_bb[3] + kMargin + 2, cur.dimy);
  int pw = max(px1 - px0, 0), ph = max(py1 - py0, 0);
  if (pw * ph > patch_cap) ph = pw > 0 ? min(ph, patch_cap / pw) : 0;  // samples outside read the frame
  for (int e = threadIdx.x; e < pw * ph; e += kSubpixThreads) {
    const int yy = e / pw, xx = e - yy * pw;
    s_patch[e] = cur.pix[(size_t)(py0 + yy) * cur.pitch + (px0 + xx)];
  }
  __syncthreads();
  grain_sums(s_w0, o.P, o.mean0, bcast);
  o.c0c0 = bcast[5];
  const Patch pt{s_patch, px0, py0, pw, ph};
  ExactObj ex{s_w0, s_v, bcast, 1.0 / (double)o.P, __longlong_as_double(0x7ff8000000000000ll), 0.0, 0.0};
  bool clamped = false;
  PowellEval<kSubpixThreads> f{&g, &cur, &sp, &o, &pt, &ex, &clamped, 0};
  double X[3] = {0.0, 0.0, 0.0};
  double fret;
  powell_minimize(f, X, sp.init_dir, sp.tol, &fret);
  if (clamped) atomicOr(&s_clamped, 1);
  __syncthreads();
  if (threadIdx.x == 0) {
    g.ncc_subpix[gi] = 1.0 - fret;
    g.upix[gi] += X[0];
    g.vpix[gi] += X[1];
    g.rot_inc[gi] += X[2];
    g.dx[gi] += X[0];
    g.dy[gi] += X[1];
    g.drot[gi] += X[2];
    if (s_clamped) g.status[gi] |= PTK_ST_SUBPIX_CLAMPED;
  }
}

// Objective (the exact one, as Powell evaluates it) or its FP64 gradient at
// caller-given X for every grain.
__global__ void __launch_bounds__(kSubpixThreads) k_objective(GrainsDev g, FrameDev cur, SubpixParams sp,
                                                                const double* Xall, double* f, double* grad,
                                                                int max_points) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ double red[kSubpixThreads / 32];
  __shared__ double bcast[8];
  const int gi = blockIdx.x;
  ObjGrain o = load_grain(g, gi);
  if (o.P <= 0 || o.P > max_points) {
    if (threadIdx.x == 0) {
      f[gi] = __longlong_as_double(0x7ff8000000000000ll);
      if (grad) grad[3 * gi] = grad[3 * gi + 1] = grad[3 * gi + 2] = f[gi];
    }
    return;
  }
  double* vals = reinterpret_cast<double*>(smem);
  const double X[3] = {Xall[3 * gi], Xall[3 * gi + 1], Xall[3 * gi + 2]};
  bool clamped = false;
  double val;
  if (grad) {
    double G[3];
    val = objective_grad<kSubpixThreads>(g, cur, sp, o, X, vals, red, G, &clamped);
    if (threadIdx.x == 0) {
      grad[3 * gi] = G[0];
      grad[3 * gi + 1] = G[1];
      grad[3 * gi + 2] = G[2];
    }
  } else {
    uint16_t* s_w0 = reinterpret_cast<uint16_t*>(smem);
    double* s_v = reinterpret_cast<double*>(smem + powell_w0_bytes(max_points));
    for (int i = threadIdx.x; i < o.P; i += kSubpixThreads) s_w0[i] = g.w0[o.b + i];
    __syncthreads();
    grain_sums(s_w0, o.P, o.mean0, bcast);
    o.c0c0 = bcast[5];
    const Patch none{nullptr, 0, 0, 0, 0};
    ExactObj ex{s_w0, s_v, bcast, 1.0 / (double)o.P, __longlong_as_double(0x7ff8000000000000ll), 0.0, 0.0};
    val = objective_exact<kSubpixThreads>(g, cur, sp, o, none, ex, X, &clamped);
  }
  if (threadIdx.x == 0) f[gi] = val;
}

static PowellSmem powell_smem(int max_points, int max_r) {
  PowellSmem m;
  const size_t side = (size_t)(2 * max_r + 1 + 2 * 6 + 2);
  size_t patch = side * side;
  const size_t rest = powell_w0_bytes(max_points) + (size_t)max_points * sizeof(double);
  constexpr size_t kCap = 227 * 1024 - 1024;  // the kernel's static shared memory included
  if (powell_vals_offset((int)patch) + rest > kCap)
    patch = rest < kCap ? (kCap - rest) / sizeof(uint16_t) - 8 : 0;  // samples outside the region read the frame
  m.patch_cap = (int)patch;
  m.max_points = max_points;
  m.bytes = powell_vals_offset(m.patch_cap) + rest;
  return m;
}

void prepare_subpix(int max_points, int max_r) {
  const PowellSmem m = powell_smem(max_points, max_r);
  ensure_smem((const void*)k_subpix_powell, m.bytes);
  // the objective alone: reference and interpolated values; with the gradient: three doubles per point
  const size_t bf = powell_w0_bytes(max_points) + (size_t)max_points * sizeof(double);
  const size_t bg = (size_t)max_points * sizeof(double) * 3;
  ensure_smem((const void*)k_objective, bg <= 227 * 1024 && bg > bf ? bg : bf);
}

void launch_subpix_powell(const GrainsDev& g, const FrameDev& cur, const FrameDev& /*ref*/, const SubpixParams& sp,
                          int max_points, int max_r, const int* order, cudaStream_t s, const int* list_count) {
  if (g.n <= 0) return;
  prepare_subpix(max_points, max_r);
  const PowellSmem m = powell_smem(max_points, max_r);
  k_subpix_powell<<<g.n, kSubpixThreads, m.bytes, s>>>(g, cur, sp, m.patch_cap, max_points, order, list_count);
}

void launch_objective(const GrainsDev& g, const FrameDev& cur, const SubpixParams& sp, const double* X, double* f,
                      double* grad, int max_points, cudaStream_t s) {
  if (g.n <= 0) return;
  prepare_subpix(max_points, 0);
  const size_t smem = grad ? (size_t)max_points * sizeof(double) * 3
                           : powell_w0_bytes(max_points) + (size_t)max_points * sizeof(double);
  k_objective<<<g.n, kSubpixThreads, smem, s>>>(g, cur, sp, X, f, grad, max_points);
}

}  // namespace ptk
