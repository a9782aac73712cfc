// Subpixel refinement by adjoint Levenberg-Marquardt (the differentiation
// form), replacing Powell in follow_pattern_subpixel_xyR
// (src/p-tracker.cpp:1090-1128).  No reference counterpart.
//
// Objective: the reference's 1 - NCC(X) (src/p-tracker.cpp:1018-1088, W = 1,
// i.e. overflow_stiffness 0) written as a least-squares problem,
//     F(X) = sum_i r_i^2 = 2 (1 - NCC),   r_i = a_i/|a| - b_i(X)/|b(X)|,
// with a the centred reference values and b the centred cubic samples of the
// current frame at the pattern points moved by X = (dx, dy, drot).  With
// g_i = dv_i/dX (cubic derivatives chained through the rotation),
// gbar = mean g, n = |b|, c = sum b_i g_i / n:
//     J^T J = (sum g g^T - P gbar gbar^T - c c^T) / n^2
//     J^T r = -(sum a_i g_i / |a| - c NCC) / n
// so one pass over the points accumulates 18 sums.  Samples and derivatives
// are FP32 (values centred on mean0 to avoid cancellation), the sums of the
// objective FP64 and the derivative sums FP32; the 3x3
// damped normal equations are solved in FP64 and X and the cumulative grain
// state accumulate in FP64.
//
// One 128-thread block per grain, grains in decreasing pattern size (the
// level-0 order) so that the large ones start first; the iteration stops when
// the step is below the tolerance, or after two rejected steps in a row once
// a step was accepted (the FP32 sums' noise floor: further steps only
// re-sample it).  A grain whose refinement ends outside the cell of its
// integer optimum (more than half a pixel, or half a rotation step, away) is
// left untouched and listed for the Powell kernel, which then refines it as
// the reference does: there the objective has several maxima within reach and
// the result depends on the minimiser's path.
#include "ptk_internal.cuh"

namespace ptk {

namespace {

constexpr int kLmThreads = 128;
constexpr int kNSums = 18;

// exact uint16 -> float: bits of 2^23 + v, minus 2^23
__device__ __forceinline__ float u16f(unsigned v) { return __int_as_float(0x4B000000 | v) - 8388608.0f; }

// Catmull-Rom weights of the reference's CubicInterpolate (src/interpol.cpp:42-53)
// and their derivatives.
__device__ __forceinline__ void cr_weights(float t, float w[4], float dw[4]) {
  const float t2 = t * t, t3 = t2 * t;
  w[0] = -0.5f * t3 + t2 - 0.5f * t;
  w[1] = 1.5f * t3 - 2.5f * t2 + 1.0f;
  w[2] = -1.5f * t3 + 2.0f * t2 + 0.5f * t;
  w[3] = 0.5f * t3 - 0.5f * t2;
  dw[0] = -1.5f * t2 + 2.0f * t - 0.5f;
  dw[1] = 4.5f * t2 - 5.0f * t;
  dw[2] = -4.5f * t2 + 4.0f * t + 0.5f;
  dw[3] = 1.5f * t2 - t;
}

struct LmGrain {
  int b, P;
  int ix0, iy0;       // integer part of refcoord + d
  float fx, fy;       // fractional part
  double drot;
  float mean0;
  double norm_a;      // |a| = sqrt(C0C0)
};

// Current-frame region around a grain, staged once in shared memory as FP32
// (exact for 16-bit pixels) for the evaluations of its LM run.  w == 0: none.
struct LmPatch {
  const float* pix;
  int x0, y0, w, h;
};

// Margin of the staged region around the pattern's bounding box: the LM's
// moves (pixels) plus the cubic support.
constexpr int kLmMargin = 4;

struct LmEval {
  double F, ncc;
  double H[6];  // xx, xy, xr, yy, yr, rr
  double gv[3];
  bool clamped;
};

// Sums over the grain's points at X, reduced over the block in a fixed order
// (every thread returns the same values).
template <int NT>
__device__ LmEval lm_eval(const GrainsDev& g, const FrameDev& cur, const LmPatch& pt, const LmGrain& o,
                          const double X[3], double (*part)[kNSums]) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  double sr, cr;
  sincos(o.drot + X[2], &sr, &cr);
  const float c = (float)cr, s = (float)sr;
  const float bx = o.fx + (float)X[0], by = o.fy + (float)X[1];
  // the objective's three sums accumulate in FP64 (they set the noise floor of
  // the acceptance test), the derivative sums in FP32
  double S0 = 0.0, S1 = 0.0, S2 = 0.0;
  float S[kNSums];
#pragma unroll
  for (int k = 3; k < kNSums; ++k) S[k] = 0.0f;
  bool clamped = false;
  for (int i = tid; i < o.P; i += NT) {
    const short2 q = g.pat0[o.b + i];
    const float x = (float)q.x, y = (float)q.y;
    const float px = bx + c * x + s * y;
    const float py = by - s * x + c * y;
    const float fpx = floorf(px), fpy = floorf(py);
    const float tx = px - fpx, ty = py - fpy;
    int ix = o.ix0 + (int)fpx, iy = o.iy0 + (int)fpy;
    float wx[4], dwx[4], wy[4], dwy[4];
    cr_weights(tx, wx, dwx);
    cr_weights(ty, wy, dwy);
    float v = 0.f, gx = 0.f, gy = 0.f;
    if (ix - 1 >= pt.x0 && iy - 1 >= pt.y0 && ix + 2 < pt.x0 + pt.w && iy + 2 < pt.y0 + pt.h) {
      // the 4x4 support lies in the staged region (which lies in the frame)
      const float* row = pt.pix + (iy - 1 - pt.y0) * pt.w + (ix - 1 - pt.x0);
#pragma unroll
      for (int jj = 0; jj < 4; ++jj) {
        const float* rp = row + jj * pt.w;
        const float p0 = rp[0], p1 = rp[1], p2 = rp[2], p3 = rp[3];
        const float hx = wx[0] * p0 + wx[1] * p1 + wx[2] * p2 + wx[3] * p3;
        const float dhx = dwx[0] * p0 + dwx[1] * p1 + dwx[2] * p2 + dwx[3] * p3;
        v += wy[jj] * hx;
        gx += wy[jj] * dhx;
        gy += dwy[jj] * hx;
      }
    } else {
      if (ix < 1 || iy < 1 || ix + 2 >= cur.dimx || iy + 2 >= cur.dimy) {
        clamped = true;
        ix = min(max(ix, 1), cur.dimx - 3);
        iy = min(max(iy, 1), cur.dimy - 3);
      }
      const uint16_t* row = cur.pix + (size_t)(iy - 1) * cur.pitch + (ix - 1);
#pragma unroll
      for (int jj = 0; jj < 4; ++jj) {
        const uint16_t* rp = row + (size_t)jj * cur.pitch;
        const float p0 = u16f(__ldg(rp)), p1 = u16f(__ldg(rp + 1)), p2 = u16f(__ldg(rp + 2)),
                    p3 = u16f(__ldg(rp + 3));
        const float hx = wx[0] * p0 + wx[1] * p1 + wx[2] * p2 + wx[3] * p3;
        const float dhx = dwx[0] * p0 + dwx[1] * p1 + dwx[2] * p2 + dwx[3] * p3;
        v += wy[jj] * hx;
        gx += wy[jj] * dhx;
        gy += dwy[jj] * hx;
      }
    }
    const float gr = gx * (-s * x + c * y) + gy * (-c * x - s * y);
    const float vc = v - o.mean0;
    const float a = u16f(g.w0[o.b + i]) - o.mean0;
    S0 += (double)vc;
    S1 = fma((double)vc, (double)vc, S1);
    S2 = fma((double)a, (double)vc, S2);
    S[3] += gx;
    S[4] += gy;
    S[5] += gr;
    S[6] += gx * gx;
    S[7] += gx * gy;
    S[8] += gx * gr;
    S[9] += gy * gy;
    S[10] += gy * gr;
    S[11] += gr * gr;
    S[12] += vc * gx;
    S[13] += vc * gy;
    S[14] += vc * gr;
    S[15] += a * gx;
    S[16] += a * gy;
    S[17] += a * gr;
  }
  // warp sums in FP64, then the warps' partial sums in index order
#pragma unroll
  for (int k = 0; k < kNSums; ++k) {
    double t = k == 0 ? S0 : (k == 1 ? S1 : (k == 2 ? S2 : (double)S[k]));
    for (int off = 16; off > 0; off >>= 1) t += __shfl_xor_sync(0xffffffffu, t, off);
    if (lane == 0) part[warp][k] = t;
  }
  const int any_clamped = __syncthreads_or(clamped ? 1 : 0);
  double T[kNSums];
#pragma unroll
  for (int k = 0; k < kNSums; ++k) {
    double t = part[0][k];
    for (int w = 1; w < NT / 32; ++w) t += part[w][k];
    T[k] = t;
  }
  __syncthreads();  // part[] is rewritten by the next evaluation
  LmEval e;
  e.clamped = any_clamped != 0;
  const double P = (double)o.P;
  const double mv = T[0] / P;
  const double n2 = T[1] - P * mv * mv;  // sum b^2
  const double n = sqrt(n2);
  // sum a = 0 up to rounding, so sum a b = sum a vc
  e.ncc = T[2] / (o.norm_a * n);
  e.F = 2.0 * (1.0 - e.ncc);
  const double gb[3] = {T[3] / P, T[4] / P, T[5] / P};
  const double cc[3] = {(T[12] - mv * T[3]) / n, (T[13] - mv * T[4]) / n, (T[14] - mv * T[5]) / n};
  const double gg[6] = {T[6], T[7], T[8], T[9], T[10], T[11]};
  const int ia[6] = {0, 0, 0, 1, 1, 2}, ib[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
  for (int k = 0; k < 6; ++k) e.H[k] = (gg[k] - P * gb[ia[k]] * gb[ib[k]] - cc[ia[k]] * cc[ib[k]]) / n2;
  const double ga[3] = {T[15] / o.norm_a, T[16] / o.norm_a, T[17] / o.norm_a};
#pragma unroll
  for (int k = 0; k < 3; ++k) e.gv[k] = -(ga[k] - cc[k] * e.ncc) / n;
  return e;
}

// (H + lambda diag H) d = -gv, symmetric 3x3 by Cramer's rule in FP64.
__device__ bool lm_solve(const double H[6], const double gv[3], double lambda, double d[3]) {
  const double a = H[0] * (1.0 + lambda), b = H[1], c = H[2];
  const double e = H[3] * (1.0 + lambda), f = H[4];
  const double i = H[5] * (1.0 + lambda);
  const double A = e * i - f * f, B = c * f - b * i, Cc = b * f - c * e;
  const double det = a * A + b * B + c * Cc;
  if (!(fabs(det) > 0.0) || !isfinite(det)) return false;
  const double D = a * i - c * c, E = b * c - a * f, I = a * e - b * b;
  const double r0 = -gv[0], r1 = -gv[1], r2 = -gv[2];
  d[0] = (A * r0 + B * r1 + Cc * r2) / det;
  d[1] = (B * r0 + D * r1 + E * r2) / det;
  d[2] = (Cc * r0 + E * r1 + I * r2) / det;
  return isfinite(d[0]) && isfinite(d[1]) && isfinite(d[2]);
}

}  // namespace

// Stages the frame region under the grain's pattern0_rotated points (their
// bounding box at the start position, widened by kLmMargin plus the cubic
// support, clipped to the frame) as FP32 in shared memory of `cap` floats.
__device__ LmPatch lm_stage(const GrainsDev& g, const FrameDev& cur, const LmGrain& o, float* s_patch, int cap,
                            int* s_bb) {
  if (threadIdx.x == 0) {
    s_bb[0] = s_bb[2] = 1 << 30;
    s_bb[1] = s_bb[3] = -(1 << 30);
  }
  __syncthreads();
  int xmn = 1 << 30, xmx = -(1 << 30), ymn = 1 << 30, ymx = -(1 << 30);
  for (int i = threadIdx.x; i < o.P; i += kLmThreads) {
    const short2 q = g.pat0[o.b + i];
    xmn = min(xmn, (int)q.x);
    xmx = max(xmx, (int)q.x);
    ymn = min(ymn, (int)q.y);
    ymx = max(ymx, (int)q.y);
  }
  atomicMin(&s_bb[0], xmn);
  atomicMax(&s_bb[1], xmx);
  atomicMin(&s_bb[2], ymn);
  atomicMax(&s_bb[3], ymx);
  __syncthreads();
  const int x0 = max(o.ix0 + s_bb[0] - kLmMargin - 1, 0), y0 = max(o.iy0 + s_bb[2] - kLmMargin - 1, 0);
  const int x1 = min(o.ix0 + s_bb[1] + kLmMargin + 3, cur.dimx), y1 = min(o.iy0 + s_bb[3] + kLmMargin + 3, cur.dimy);
  int w = max(x1 - x0, 0), h = max(y1 - y0, 0);
  if (w * h > cap) h = w > 0 ? min(h, cap / w) : 0;  // never expected: the host sizes the cap
  for (int e = threadIdx.x; e < w * h; e += kLmThreads) {
    const int yy = e / w, xx = e - yy * w;
    s_patch[e] = u16f(__ldg(cur.pix + (size_t)(y0 + yy) * cur.pitch + (x0 + xx)));
  }
  __syncthreads();
  return LmPatch{s_patch, x0, y0, w, h};
}

__global__ void __launch_bounds__(kLmThreads) k_subpix_lm(GrainsDev g, FrameDev cur, LmParams lp, int patch_cap) {
  extern __shared__ __align__(16) float s_lm_patch[];
  __shared__ double part[kLmThreads / 32][kNSums];
  __shared__ int s_bb[4];
  const int gi = lp.order ? lp.order[blockIdx.x] : (int)blockIdx.x;
  if (g.masked[gi] || (g.flags[gi] & 3)) return;
  LmGrain o;
  o.b = g.pstart[gi];
  o.P = g.pstart[gi + 1] - o.b;
  if (o.P <= 0) return;
  const double xr = (double)g.refx[gi] + g.dx[gi];
  const double yr = (double)g.refy[gi] + g.dy[gi];
  const double fxr = floor(xr), fyr = floor(yr);
  o.ix0 = (int)fxr;
  o.iy0 = (int)fyr;
  o.fx = (float)(xr - fxr);
  o.fy = (float)(yr - fyr);
  o.drot = g.drot[gi];
  o.mean0 = (float)g.mean0[gi];
  o.norm_a = sqrt(g.c0c0[gi]);
  const double rscale = g.radius[gi] > 1.0 ? g.radius[gi] : 1.0;  // rotation step in pixels at the rim
  const LmPatch pt = lm_stage(g, cur, o, s_lm_patch, patch_cap, s_bb);

  double X[3] = {0.0, 0.0, 0.0};
  LmEval cur_e = lm_eval<kLmThreads>(g, cur, pt, o, X, part);
  bool clamped = cur_e.clamped;
  double lambda = 1e-3;
  int it = 0, accepted = 0, rejected_run = 0;
  if (isfinite(cur_e.F)) {
    for (it = 0; it < lp.max_iter; ++it) {
      double d[3];
      if (!lm_solve(cur_e.H, cur_e.gv, lambda, d)) {
        lambda *= 10.0;
        if (lambda > 1e8) break;
        continue;
      }
      const double step = fmax(fmax(fabs(d[0]), fabs(d[1])), fabs(d[2]) * rscale);
      if (step < lp.tol) break;
      const double Xn[3] = {X[0] + d[0], X[1] + d[1], X[2] + d[2]};
      const LmEval ne = lm_eval<kLmThreads>(g, cur, pt, o, Xn, part);
      if (isfinite(ne.F) && ne.F < cur_e.F) {
        X[0] = Xn[0];
        X[1] = Xn[1];
        X[2] = Xn[2];
        cur_e = ne;
        clamped = clamped || ne.clamped;
        lambda = fmax(lambda * 0.1, 1e-12);
        ++accepted;
        rejected_run = 0;
      } else {
        lambda *= 10.0;
        if (lambda > 1e8) break;
        if (++rejected_run >= 2 && accepted > 0) break;
      }
    }
  }
  // Outside the cell of the integer optimum (the local quadratic model of the
  // objective did not hold: another maximum attracted the steps), the grain
  // keeps its pixel-stage state and goes to the reference's Powell.
  if (lp.redo_list && (fabs(X[0]) > lp.cell_px || fabs(X[1]) > lp.cell_px || fabs(X[2]) > lp.cell_rot)) {
    if (threadIdx.x == 0) lp.redo_list[atomicAdd(lp.redo_count, 1)] = gi;
    return;
  }
  if (threadIdx.x == 0) {
    g.ncc_subpix[gi] = 1.0 - 0.5 * cur_e.F;
    g.upix[gi] += X[0];
    g.vpix[gi] += X[1];
    g.rot_inc[gi] += X[2];
    g.dx[gi] += X[0];
    g.dy[gi] += X[1];
    g.drot[gi] += X[2];
    if (clamped) g.status[gi] |= PTK_ST_SUBPIX_CLAMPED;
    if (lp.iters) lp.iters[gi] = it;
  }
}

// F = 1 - NCC and its gradient from the FP32 adjoint sums (for checks).
__global__ void __launch_bounds__(kLmThreads) k_grad_f32(GrainsDev g, FrameDev cur, const double* Xall, double* f,
                                                        double* grad) {
  __shared__ double part[kLmThreads / 32][kNSums];
  const int gi = blockIdx.x;
  LmGrain o;
  o.b = g.pstart[gi];
  o.P = g.pstart[gi + 1] - o.b;
  if (o.P <= 0) return;
  const double xr = (double)g.refx[gi] + g.dx[gi];
  const double yr = (double)g.refy[gi] + g.dy[gi];
  const double fxr = floor(xr), fyr = floor(yr);
  o.ix0 = (int)fxr;
  o.iy0 = (int)fyr;
  o.fx = (float)(xr - fxr);
  o.fy = (float)(yr - fyr);
  o.drot = g.drot[gi];
  o.mean0 = (float)g.mean0[gi];
  o.norm_a = sqrt(g.c0c0[gi]);
  const double X[3] = {Xall[3 * gi], Xall[3 * gi + 1], Xall[3 * gi + 2]};
  const LmPatch none{nullptr, 0, 0, 0, 0};
  const LmEval e = lm_eval<kLmThreads>(g, cur, none, o, X, part);
  if (threadIdx.x == 0) {
    f[gi] = 1.0 - e.ncc;
    // d(1 - NCC)/dX = (1/2) dF/dX = J^T r
    grad[3 * gi] = e.gv[0];
    grad[3 * gi + 1] = e.gv[1];
    grad[3 * gi + 2] = e.gv[2];
  }
}

void launch_subpix_lm(const GrainsDev& g, const FrameDev& cur, const LmParams& lp, cudaStream_t s) {
  if (g.n <= 0) return;
  // staged region: pattern0_rotated extent (|q| <= max_r + 1) plus the margins
  const int side = 2 * (lp.max_r + 1) + 1 + 2 * (kLmMargin + 2);
  int cap = side * side;
  if ((size_t)cap * sizeof(float) > 200 * 1024) cap = 200 * 1024 / (int)sizeof(float);  // larger regions read the frame
  ensure_smem((const void*)k_subpix_lm, (size_t)cap * sizeof(float));
  k_subpix_lm<<<g.n, kLmThreads, (size_t)cap * sizeof(float), s>>>(g, cur, lp, cap);
}

void launch_grad_f32(const GrainsDev& g, const FrameDev& cur, const double* X, double* f, double* grad,
                     cudaStream_t s) {
  if (g.n <= 0) return;
  k_grad_f32<<<g.n, kLmThreads, 0, s>>>(g, cur, X, f, grad);
}

}  // namespace ptk
