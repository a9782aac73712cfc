// Distortion-parameter fit (the correction_distortion procedure,
// src/distortion_correction.cpp:135-479) with its objective on sm_100a.
//
// The procedure tracks a set of images against a reference image (pixel
// search without rescue, then subpixel), then fits the 14 undistor parameters
// by minimising the equiprojectivity criterion
//     sum over images and grain pairs (i, j) of err^2,
//     err = AB_unit . ((B2 - B1) - (A2 - A1)),
// with A1/B1 the undistorted reference positions of i and j, A2/B2 their
// undistorted tracked positions, over the pairs whose reference positions lie
// equiProj_dist_min .. equiProj_dist_max apart (precompute_paires, :63-81) and
// skipping pairs with a subpixel NCC below NCC_min.  One evaluation is
// (images - 1) x pairs residuals.  The reference undistorts four points per
// residual; here every (image, grain) point is undistorted once (a per-point
// kernel, images x grains undistor calls instead of 4 x images x pairs) and
// the residual kernel gathers the four positions of each pair, which stay in
// L2, and adds the squares up (its last block to finish sums the blocks'
// partial sums).  Both run in FP64 (this file is compiled with -fmad=false, so
// each residual is the CPU's value bit for bit) and the sum is reduced in a
// fixed order over a fixed grid, so it is reproducible.  The minimiser runs on the host and calls the
// kernel for every objective value: POWELL (one minimisation, ftol 1e-12,
// initial directions the perturbations) and POWELL_ITER (num_iter
// minimisations, each followed by re-anchoring A1/B1 and the displacements on
// the undistorted reference positions, :300-386), and LEVMAR (:400-479):
// Levenberg-Marquardt over the residual vector of the GPU kernel, restated in
// ptk_lmdif.hpp from the published MINPACK algorithm (the reference calls
// lmdif1 from the absent toofus library with tol = DBL_EPSILON; pairs it
// skips keep a zero residual there as here).
#include <cfloat>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "ptk.h"
#include "ptk_internal.cuh"
#include "ptk_lmdif.hpp"
#include "ptk_undistor.cuh"

struct ptk_disto {
  int n{0}, nimg1{0}, dimx{0}, dimy{0};
  long long npairs{0};
  double NCC_min{0.0};
  std::vector<int32_t> refx, refy;
  int32_t *d_refx{nullptr}, *d_refy{nullptr};
  int2* d_pairs{nullptr};
  double *d_dx{nullptr}, *d_dy{nullptr}, *d_dx0{nullptr}, *d_dy0{nullptr}, *d_ncc{nullptr};
  double *d_origx{nullptr}, *d_origy{nullptr};
  double *d_partial{nullptr}, *d_sum{nullptr}, *d_fvec{nullptr};
  unsigned* d_done{nullptr};  // blocks of the residual kernel finished (the last one sums and resets it)
  double2* d_pos{nullptr};  // undistorted points: slot 0 A1 (reference), slot 1 + im the tracked ones
  cudaStream_t stream{nullptr};
  std::string err;
  int lm_info{-2}, lm_nfev{0};  // exit state and residual evaluations of the last LEVMAR fit
};

namespace ptk {

namespace {

constexpr int kDThreads = 256;
constexpr int kDBlocks = 592;  // fixed grid: the reduction order does not depend on the device

struct DistoData {
  int n, nimg1;
  long long npairs;
  const int32_t *refx, *refy;
  const double *origx, *origy;
  const double *dx, *dy, *ncc;
  double NCC_min;
  const int2* pairs;
  int use_orig;
};

// The undistorted points of one evaluation: pos[g] = A1 of grain g (undistor
// of its reference position, or the re-anchored position of POWELL_ITER) and
// pos[(1 + im) * n + g] = undistor of its tracked position in image im.
__global__ void __launch_bounds__(kDThreads) k_disto_points(DistoData d, Disto X, double2* pos) {
  const long long k = (long long)blockIdx.x * kDThreads + threadIdx.x;
  if (k >= (long long)(d.nimg1 + 1) * d.n) return;
  const int s = (int)(k / d.n), g = (int)(k - (long long)s * d.n);
  double x, y;
  if (s == 0) {
    if (d.use_orig) {
      x = d.origx[g];
      y = d.origy[g];
    } else {
      undistor_d(X, (double)d.refx[g], (double)d.refy[g], &x, &y);
    }
  } else {
    const size_t o = (size_t)(s - 1) * d.n + g;
    undistor_d(X, (double)d.refx[g] + d.dx[o], (double)d.refy[g] + d.dy[o], &x, &y);
  }
  pos[k] = make_double2(x, y);
}

// One residual per (image, pair) from the undistorted points, images
// outermost (no 64-bit division per residual); partial[block] = the block's
// sum of err^2, and the block that finishes last adds the partial sums in
// block order into *out (the same order whichever block is last).
__global__ void __launch_bounds__(kDThreads) k_disto_residuals(DistoData d, const double2* __restrict__ pos,
                                                               double* fvec, double* partial, unsigned* done,
                                                               double* out) {
  __shared__ double red[kDThreads / 32];
  __shared__ bool s_last;
  double acc = 0.0;
  const long long stride = (long long)gridDim.x * kDThreads;
  for (int im = 0; im < d.nimg1; ++im) {
    const size_t io = (size_t)im * d.n;
    const double2* pimg = pos + (size_t)d.n + io;
    for (long long il = (long long)blockIdx.x * kDThreads + threadIdx.x; il < d.npairs; il += stride) {
      const int2 pr = d.pairs[il];
      const int i = pr.x, j = pr.y;
      double e = 0.0;
      if (!(d.ncc[io + i] < d.NCC_min || d.ncc[io + j] < d.NCC_min)) {
        const double2 A1 = pos[i], B1 = pos[j];
        const double2 A2 = pimg[i], B2 = pimg[j];
        double ABx = B1.x - A1.x, ABy = B1.y - A1.y;
        const double AB = sqrt(ABx * ABx + ABy * ABy);
        ABx /= AB;
        ABy /= AB;
        const double BBx = B2.x - B1.x, BBy = B2.y - B1.y;
        const double AAx = A2.x - A1.x, AAy = A2.y - A1.y;
        e = (ABx * (BBx - AAx)) + (ABy * (BBy - AAy));
        acc += e * e;
      }
      if (fvec) fvec[(size_t)im * d.npairs + il] = e;
    }
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < kDThreads / 32; ++w) s += red[w];
    partial[blockIdx.x] = s;
    __threadfence();
    s_last = atomicAdd(done, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  double a2 = 0.0;
  for (int k = threadIdx.x; k < (int)gridDim.x; k += kDThreads) a2 += __ldcg(partial + k);
  for (int o = 16; o > 0; o >>= 1) a2 += __shfl_xor_sync(0xffffffffu, a2, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = a2;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < kDThreads / 32; ++w) t += red[w];
    *out = t;
    *done = 0u;  // ready for the next evaluation
  }
}

// POWELL_ITER re-anchoring (src/distortion_correction.cpp:367-380): A1/B1 and
// the displacements move to the undistorted reference positions.
__global__ void k_disto_reanchor(DistoData d, Disto X, double* origx, double* origy, double* dx, double* dy,
                                 const double* dx0, const double* dy0) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= d.n) return;
  double xu, yu;
  undistor_d(X, (double)d.refx[g], (double)d.refy[g], &xu, &yu);
  const double dxc = xu - (double)d.refx[g], dyc = yu - (double)d.refy[g];
  for (int im = 0; im < d.nimg1; ++im) {
    const size_t o = (size_t)im * d.n + g;
    dx[o] = dx0[o] + dxc;
    dy[o] = dy0[o] + dyc;
  }
  origx[g] = xu;
  origy[g] = yu;
}

// ---- Powell's direction-set method (Powell 1964) with Brent's line
// minimiser (Brent 1973, ch. 5): golden expansion from {0, 1} to a bracket,
// then parabolic steps safeguarded by golden sections; the same constants as
// the subpixel minimiser.
constexpr double kGold = 1.6180339887498949;
constexpr double kCGold = 0.3819660112501051;
constexpr double kLineRelTol = 1.0e-4;
constexpr double kLineAbsTol = 1.0e-10;
constexpr int kBracketMaxIter = 60;
constexpr int kBrentMaxIter = 100;
constexpr int kPowellMaxIter = 200;
constexpr double kTiny = 1.0e-25;

template <class G>
double brent_line(G& g, double* gmin, bool* ok) {
  double a = 0.0, b = 1.0;
  double ga = g(a), gb = g(b);
  if (gb > ga) {
    std::swap(a, b);
    std::swap(ga, gb);
  }
  double c = b + kGold * (b - a);
  double gc = g(c);
  for (int it = 0; it < kBracketMaxIter && gc < gb; ++it) {
    a = b;
    ga = gb;
    b = c;
    gb = gc;
    c = b + kGold * (b - a);
    gc = g(c);
  }
  double lo = a < c ? a : c, hi = a < c ? c : a;
  double x = b, w = b, v = b, fx = gb, fw = gb, fv = gb, d = 0.0, e = 0.0;
  for (int it = 0; it < kBrentMaxIter; ++it) {
    const double m = 0.5 * (lo + hi);
    const double tol1 = kLineRelTol * std::fabs(x) + kLineAbsTol, tol2 = 2.0 * tol1;
    if (std::fabs(x - m) <= tol2 - 0.5 * (hi - lo)) break;
    bool golden = true;
    if (std::fabs(e) > tol1) {
      double r = (x - w) * (fx - fv);
      double q = (x - v) * (fx - fw);
      double p = (x - v) * q - (x - w) * r;
      q = 2.0 * (q - r);
      if (q > 0.0) p = -p;
      else q = -q;
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
  *ok = true;
  return x;
}

// Minimises f from p with the scaled coordinate directions; f returns false
// when an evaluation failed (the minimisation then stops with that status).
template <class F>
bool powell_minimize(F& f, std::vector<double>& p, const std::vector<double>& step, double ftol) {
  const size_t n = p.size();
  std::vector<std::vector<double>> dirs(n, std::vector<double>(n, 0.0));
  for (size_t i = 0; i < n; ++i) dirs[i][i] = step[i];
  std::vector<double> pstart = p, ptt(n), xit(n), trial(n);
  bool good = true;
  auto eval = [&](const std::vector<double>& x) {
    double v = 0.0;
    if (!f(x, &v)) good = false;
    return v;
  };
  double fret = eval(p);
  if (!good || !std::isfinite(fret)) return good;
  auto line_search = [&](std::vector<double>& dir) {
    auto g = [&](double alpha) {
      for (size_t j = 0; j < n; ++j) trial[j] = p[j] + alpha * dir[j];
      return eval(trial);
    };
    double gmin;
    bool ok;
    const double alpha = brent_line(g, &gmin, &ok);
    for (size_t j = 0; j < n; ++j) {
      dir[j] *= alpha;
      p[j] += dir[j];
    }
    fret = gmin;
  };
  for (int iter = 0; iter < kPowellMaxIter && good; ++iter) {
    const double fp = fret;
    size_t ibig = 0;
    double del = 0.0;
    for (size_t i = 0; i < n; ++i) {
      const double fptt = fret;
      line_search(dirs[i]);
      if (fptt - fret > del) {
        del = fptt - fret;
        ibig = i;
      }
    }
    if (2.0 * (fp - fret) <= ftol * (std::fabs(fp) + std::fabs(fret)) + kTiny) break;
    for (size_t j = 0; j < n; ++j) {
      ptt[j] = 2.0 * p[j] - pstart[j];
      xit[j] = p[j] - pstart[j];
      pstart[j] = p[j];
    }
    const double fe = eval(ptt);
    if (fe < fp) {
      const double t1 = fp - fret - del;
      const double t = 2.0 * (fp - 2.0 * fret + fe) * t1 * t1 - del * (fp - fe) * (fp - fe);
      if (t < 0.0) {
        line_search(xit);
        dirs[ibig] = dirs[n - 1];
        dirs[n - 1] = xit;
      }
    }
  }
  return good;
}

int dfail(ptk_disto* d, int code, const std::string& msg) {
  if (d) d->err = msg;
  return code;
}

DistoData data_of(const ptk_disto* d, int use_orig) {
  DistoData x;
  x.n = d->n;
  x.nimg1 = d->nimg1;
  x.npairs = d->npairs;
  x.refx = d->d_refx;
  x.refy = d->d_refy;
  x.origx = d->d_origx;
  x.origy = d->d_origy;
  x.dx = d->d_dx;
  x.dy = d->d_dy;
  x.ncc = d->d_ncc;
  x.NCC_min = d->NCC_min;
  x.pairs = d->d_pairs;
  x.use_orig = use_orig;
  return x;
}

// One objective value (and, with fvec, the residual vector copied to the host).
int disto_eval(ptk_disto* d, const double* X14, int use_orig, double* value, double* fvec_host) {
  const Disto X = make_disto(X14);
  const long long m = (long long)d->nimg1 * d->npairs;
  double* fv = nullptr;
  if (fvec_host && m > 0) {
    if (!d->d_fvec && cudaMalloc(&d->d_fvec, sizeof(double) * m) != cudaSuccess)
      return dfail(d, PTK_ERR_CUDA, "cudaMalloc(residuals)");
    fv = d->d_fvec;
  }
  const DistoData dd = data_of(d, use_orig);
  const long long npts = (long long)(d->nimg1 + 1) * d->n;
  if (npts > 0) k_disto_points<<<(unsigned)((npts + kDThreads - 1) / kDThreads), kDThreads, 0, d->stream>>>(dd, X, d->d_pos);
  k_disto_residuals<<<kDBlocks, kDThreads, 0, d->stream>>>(dd, d->d_pos, fv, d->d_partial, d->d_done, d->d_sum);
  cudaError_t e = cudaMemcpyAsync(value, d->d_sum, sizeof(double), cudaMemcpyDeviceToHost, d->stream);
  if (e == cudaSuccess && fv) e = cudaMemcpyAsync(fvec_host, fv, sizeof(double) * m, cudaMemcpyDeviceToHost, d->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(d->stream);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return dfail(d, PTK_ERR_CUDA, std::string("distortion objective: ") + cudaGetErrorString(e));
  return PTK_OK;
}

}  // namespace
}  // namespace ptk

using namespace ptk;

extern "C" {

int ptk_disto_pairs(const int32_t* refx, const int32_t* refy, int n, double dmin, double dmax, int32_t* pairs_ij,
                    int64_t capacity, int64_t* npairs) {
  if (!refx || !refy || n < 0 || !npairs || (capacity > 0 && !pairs_ij)) return PTK_ERR_ARG;
  int64_t np = 0;
  for (int i = 0; i < n; ++i) {
    const double xi = (double)refx[i], yi = (double)refy[i];
    for (int j = i + 1; j < n; ++j) {
      const double xij = (double)refx[j] - xi, yij = (double)refy[j] - yi;
      const double dij = std::sqrt(xij * xij + yij * yij);
      if (dij >= dmin && dij <= dmax) {
        if (np < capacity) {
          pairs_ij[2 * np] = i;
          pairs_ij[2 * np + 1] = j;
        }
        ++np;
      }
    }
  }
  *npairs = np;
  return np <= capacity ? PTK_OK : PTK_ERR_LIMIT;
}

int ptk_disto_create(ptk_disto** out, int dimx, int dimy, const int32_t* refx, const int32_t* refy, int n,
                     int n_tracked, const double* dx, const double* dy, const double* ncc_subpix, double NCC_min,
                     const int32_t* pairs_ij, int64_t npairs) {
  if (!out || n < 1 || n_tracked < 1 || npairs < 0 || !refx || !refy || !dx || !dy || !ncc_subpix ||
      (npairs > 0 && !pairs_ij))
    return PTK_ERR_ARG;
  *out = nullptr;
  for (int64_t k = 0; k < 2 * npairs; ++k)
    if (pairs_ij[k] < 0 || pairs_ij[k] >= n) return PTK_ERR_ARG;
  ptk_disto* d = new ptk_disto();
  d->n = n;
  d->nimg1 = n_tracked;
  d->dimx = dimx;
  d->dimy = dimy;
  d->npairs = npairs;
  d->NCC_min = NCC_min;
  d->refx.assign(refx, refx + n);
  d->refy.assign(refy, refy + n);
  const size_t ng = (size_t)n_tracked * n;
  bool ok = cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking) == cudaSuccess;
  auto alloc = [&](void** p, size_t bytes) { ok = ok && cudaMalloc(p, bytes > 0 ? bytes : 16) == cudaSuccess; };
  alloc((void**)&d->d_refx, sizeof(int32_t) * n);
  alloc((void**)&d->d_refy, sizeof(int32_t) * n);
  alloc((void**)&d->d_pairs, sizeof(int2) * npairs);
  alloc((void**)&d->d_dx, sizeof(double) * ng);
  alloc((void**)&d->d_dy, sizeof(double) * ng);
  alloc((void**)&d->d_dx0, sizeof(double) * ng);
  alloc((void**)&d->d_dy0, sizeof(double) * ng);
  alloc((void**)&d->d_ncc, sizeof(double) * ng);
  alloc((void**)&d->d_origx, sizeof(double) * n);
  alloc((void**)&d->d_origy, sizeof(double) * n);
  alloc((void**)&d->d_partial, sizeof(double) * kDBlocks);
  alloc((void**)&d->d_sum, sizeof(double));
  alloc((void**)&d->d_done, sizeof(unsigned));
  alloc((void**)&d->d_pos, sizeof(double2) * (size_t)(n_tracked + 1) * n);
  if (ok) {
    std::vector<double> ox(n), oy(n);
    for (int g = 0; g < n; ++g) {
      ox[g] = (double)refx[g];
      oy[g] = (double)refy[g];
    }
    ok = cudaMemcpyAsync(d->d_refx, refx, sizeof(int32_t) * n, cudaMemcpyHostToDevice, d->stream) == cudaSuccess &&
         cudaMemcpyAsync(d->d_refy, refy, sizeof(int32_t) * n, cudaMemcpyHostToDevice, d->stream) == cudaSuccess &&
         (npairs == 0 ||
          cudaMemcpyAsync(d->d_pairs, pairs_ij, sizeof(int2) * npairs, cudaMemcpyHostToDevice, d->stream) == cudaSuccess) &&
         cudaMemcpyAsync(d->d_dx, dx, sizeof(double) * ng, cudaMemcpyHostToDevice, d->stream) == cudaSuccess &&
         cudaMemcpyAsync(d->d_dy, dy, sizeof(double) * ng, cudaMemcpyHostToDevice, d->stream) == cudaSuccess &&
         cudaMemcpyAsync(d->d_dx0, dx, sizeof(double) * ng, cudaMemcpyHostToDevice, d->stream) == cudaSuccess &&
         cudaMemcpyAsync(d->d_dy0, dy, sizeof(double) * ng, cudaMemcpyHostToDevice, d->stream) == cudaSuccess &&
         cudaMemcpyAsync(d->d_ncc, ncc_subpix, sizeof(double) * ng, cudaMemcpyHostToDevice, d->stream) == cudaSuccess &&
         cudaMemcpyAsync(d->d_origx, ox.data(), sizeof(double) * n, cudaMemcpyHostToDevice, d->stream) == cudaSuccess &&
         cudaMemcpyAsync(d->d_origy, oy.data(), sizeof(double) * n, cudaMemcpyHostToDevice, d->stream) == cudaSuccess &&
         cudaMemsetAsync(d->d_done, 0, sizeof(unsigned), d->stream) == cudaSuccess &&
         // (on the fit's stream, which does not order with the legacy stream)
         cudaStreamSynchronize(d->stream) == cudaSuccess;
  }
  if (!ok) {
    ptk_disto_destroy(d);
    return PTK_ERR_CUDA;
  }
  *out = d;
  return PTK_OK;
}

int ptk_disto_destroy(ptk_disto* d) {
  if (!d) return PTK_OK;
  cudaFree(d->d_refx);
  cudaFree(d->d_refy);
  cudaFree(d->d_pairs);
  cudaFree(d->d_dx);
  cudaFree(d->d_dy);
  cudaFree(d->d_dx0);
  cudaFree(d->d_dy0);
  cudaFree(d->d_ncc);
  cudaFree(d->d_origx);
  cudaFree(d->d_origy);
  cudaFree(d->d_partial);
  cudaFree(d->d_sum);
  cudaFree(d->d_done);
  cudaFree(d->d_fvec);
  cudaFree(d->d_pos);
  if (d->stream) cudaStreamDestroy(d->stream);
  delete d;
  return PTK_OK;
}

const char* ptk_disto_last_error(ptk_disto* d) { return d ? d->err.c_str() : "null handle"; }

int ptk_disto_objective(ptk_disto* d, const double* params14, double* value) {
  if (!d || !params14 || !value) return dfail(d, PTK_ERR_ARG, "null argument");
  return disto_eval(d, params14, 0, value, nullptr);
}

int ptk_disto_residuals(ptk_disto* d, const double* params14, double* value, double* fvec) {
  if (!d || !params14 || !value || !fvec) return dfail(d, PTK_ERR_ARG, "null argument");
  return disto_eval(d, params14, 0, value, fvec);
}

int ptk_disto_fit(ptk_disto* d, double* params14, const double* perturb14, int algo, int num_iter,
                  double* index_ini, double* index_end, double* history) {
  if (!d || !params14 || !perturb14 || !index_ini || !index_end) return dfail(d, PTK_ERR_ARG, "null argument");
  if (algo != PTK_DISTO_POWELL && algo != PTK_DISTO_POWELL_ITER && algo != PTK_DISTO_LEVMAR)
    return dfail(d, PTK_ERR_ARG, "optim_algo: POWELL, POWELL_ITER or LEVMAR");
  if (algo == PTK_DISTO_POWELL_ITER && num_iter < 0) return dfail(d, PTK_ERR_ARG, "powell_num_iter < 0");
  std::vector<double> X(params14, params14 + 14), DX(perturb14, perturb14 + 14);
  if (X[0] < 0.0) X[0] = 0.5 * (double)d->dimx;
  if (X[1] < 0.0) X[1] = 0.5 * (double)d->dimy;
  if (X[8] < 0.0) X[8] = 0.5 * (double)d->dimx;
  if (X[9] < 0.0) X[9] = 0.5 * (double)d->dimy;
  const int use_orig = algo == PTK_DISTO_POWELL_ITER ? 1 : 0;
  int rc = PTK_OK;
  auto f = [&](const std::vector<double>& x, double* v) {
    rc = disto_eval(d, x.data(), use_orig, v, nullptr);
    return rc == PTK_OK;
  };
  const double nb = (double)d->nimg1;
  double v = 0.0;
  if (!f(X, &v)) return rc;
  *index_ini = v / nb;
  if (algo == PTK_DISTO_POWELL_ITER) {
    for (int it = 1; it <= num_iter; ++it) {
      if (!powell_minimize(f, X, DX, 1e-12)) return rc;
      if (!f(X, &v)) return rc;
      if (history) {
        history[(size_t)(it - 1) * 15] = v / nb;
        for (int k = 0; k < 14; ++k) history[(size_t)(it - 1) * 15 + 1 + k] = X[k];
      }
      const Disto Xd = make_disto(X.data());
      k_disto_reanchor<<<(d->n + 127) / 128, 128, 0, d->stream>>>(data_of(d, 1), Xd, d->d_origx, d->d_origy, d->d_dx,
                                                                  d->d_dy, d->d_dx0, d->d_dy0);
      cudaError_t e = cudaStreamSynchronize(d->stream);
      if (e == cudaSuccess) e = cudaGetLastError();
      if (e != cudaSuccess) return dfail(d, PTK_ERR_CUDA, std::string("re-anchoring: ") + cudaGetErrorString(e));
    }
  } else if (algo == PTK_DISTO_LEVMAR) {
    // all 14 parameters free, as the reference passes the whole vector to lmdif1
    const long long m = (long long)d->nimg1 * d->npairs;
    if (m < 14) return dfail(d, PTK_ERR_ARG, "LEVMAR needs at least 14 residuals (images x pairs)");
    if (m > (1LL << 31) / 14) return dfail(d, PTK_ERR_LIMIT, "LEVMAR: residuals x 14 exceed the host Jacobian limit");
    std::vector<double> fvec((size_t)m);
    auto fcn = [&](const double* x, double* fv) {
      double val = 0.0;
      rc = disto_eval(d, x, 0, &val, fv);
      return rc == PTK_OK;
    };
    int nfev = 0;
    const int info = lmdif::lmdif1(fcn, (int)m, 14, X.data(), fvec.data(), DBL_EPSILON, &nfev);
    if (info < 0) return rc;
    d->lm_info = info;
    d->lm_nfev = nfev;
    if (history) {  // one row: final index, then the parameters (as one POWELL_ITER row)
      if (!f(X, &v)) return rc;
      history[0] = v / nb;
      for (int k = 0; k < 14; ++k) history[1 + k] = X[k];
    }
  } else if (!powell_minimize(f, X, DX, 1e-12)) {
    return rc;
  }
  if (!f(X, &v)) return rc;
  *index_end = v / nb;
  for (int k = 0; k < 14; ++k) params14[k] = X[k];
  return PTK_OK;
}

int ptk_disto_levmar_info(ptk_disto* d, int* info, int* nfev, const char** text) {
  if (!d || !info) return dfail(d, PTK_ERR_ARG, "null argument");
  *info = d->lm_info;
  if (nfev) *nfev = d->lm_nfev;
  if (text) *text = d->lm_info >= 0 ? lmdif::info_text(d->lm_info) : "no LEVMAR fit has run";
  return PTK_OK;
}

int ptk_disto_objective_timed(ptk_disto* d, const double* params14, int reps, double* ms_per_eval) {
  if (!d || !params14 || !ms_per_eval || reps < 1) return dfail(d, PTK_ERR_ARG, "null argument or reps < 1");
  const Disto X = make_disto(params14);
  const DistoData dd = data_of(d, 0);
  const long long npts = (long long)(d->nimg1 + 1) * d->n;
  cudaEvent_t ev[2];
  if (cudaEventCreate(&ev[0]) != cudaSuccess) return dfail(d, PTK_ERR_CUDA, "cudaEventCreate");
  if (cudaEventCreate(&ev[1]) != cudaSuccess) {
    cudaEventDestroy(ev[0]);
    return dfail(d, PTK_ERR_CUDA, "cudaEventCreate");
  }
  cudaEventRecord(ev[0], d->stream);
  for (int k = 0; k < reps; ++k) {
    k_disto_points<<<(unsigned)((npts + kDThreads - 1) / kDThreads), kDThreads, 0, d->stream>>>(dd, X, d->d_pos);
    k_disto_residuals<<<kDBlocks, kDThreads, 0, d->stream>>>(dd, d->d_pos, nullptr, d->d_partial, d->d_done,
                                                             d->d_sum);
  }
  cudaEventRecord(ev[1], d->stream);
  cudaError_t e = cudaEventSynchronize(ev[1]);
  float ms = 0.0f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, ev[0], ev[1]);
  if (e == cudaSuccess) e = cudaGetLastError();
  cudaEventDestroy(ev[0]);
  cudaEventDestroy(ev[1]);
  if (e != cudaSuccess) return dfail(d, PTK_ERR_CUDA, std::string("timed objective: ") + cudaGetErrorString(e));
  *ms_per_eval = (double)ms / reps;
  return PTK_OK;
}

int ptk_disto_tracked(ptk_disto* d, double* dx, double* dy) {
  if (!d || !dx || !dy) return dfail(d, PTK_ERR_ARG, "null argument");
  const size_t ng = (size_t)d->nimg1 * d->n;
  cudaError_t e = cudaMemcpyAsync(dx, d->d_dx, sizeof(double) * ng, cudaMemcpyDeviceToHost, d->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dy, d->d_dy, sizeof(double) * ng, cudaMemcpyDeviceToHost, d->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(d->stream);
  if (e != cudaSuccess) return dfail(d, PTK_ERR_CUDA, cudaGetErrorString(e));
  return PTK_OK;
}

}  // extern "C"
