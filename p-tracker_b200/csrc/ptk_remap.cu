// Distortion-correction remap on sm_100a.
//
// The reference models lens distortion with undistor
// (src/distortion_correction.cpp:20-61: Brown radial K1-K3 and tangential
// P1-P3 about (xc, yc), then a two-axis parallax scaling) and applies it to
// point coordinates only.  The tracking path here corrects whole frames: the
// corrected pixel (x, y) takes the distorted frame's value at the point xd
// with undistor(xd) = (x, y).  xd is found by 8 Newton steps from xd = (x, y)
// with a forward-difference Jacobian (step 1e-3 px), then sampled with the
// reference's cubic interpolant (src/interpol.cpp:42-86) and rounded half up.
//
// The inverse map depends only on the 14 parameters, so it is built once per
// parameter set into a resident FP64 map (16 bytes per pixel: 336 MB at
// 5616x3744, kept in HBM) and each frame is then a single gather pass.  This
// file is compiled with -fmad=false; the cos/sin of the two parallax angles
// come from the host.  With both, the device repeats the CPU restatement's
// FP64 operations exactly.
#include "ptk_internal.cuh"
#include "ptk_undistor.cuh"

namespace ptk {

namespace {

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

}  // namespace

__global__ void k_remap_build(Disto X, double2* map, int dimx, int dimy) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x >= dimx || y >= dimy) return;
  const double xu = (double)x, yu = (double)y;
  double xd = xu, yd = yu;
  const double h = 1e-3;
  for (int it = 0; it < 8; ++it) {
    double fx, fy, fx1, fy1, fx2, fy2;
    undistor_d(X, xd, yd, &fx, &fy);
    undistor_d(X, xd + h, yd, &fx1, &fy1);
    undistor_d(X, xd, yd + h, &fx2, &fy2);
    const double j11 = (fx1 - fx) / h, j21 = (fy1 - fy) / h;
    const double j12 = (fx2 - fx) / h, j22 = (fy2 - fy) / h;
    const double rx = fx - xu, ry = fy - yu;
    const double det = j11 * j22 - j12 * j21;
    xd = xd - (j22 * rx - j12 * ry) / det;
    yd = yd - (j11 * ry - j21 * rx) / det;
  }
  map[(size_t)y * dimx + x] = make_double2(xd, yd);
}

// One output row per blockIdx.y; a thread per output pixel.  The 4x4 support
// is gathered through the read-only path; rows of neighbouring threads are
// adjacent, so each warp's 16 loads touch a few cache lines.
__global__ void k_remap_apply(const double2* __restrict__ map, const uint16_t* __restrict__ src,
                              uint16_t* __restrict__ dst, int pitch, int dimx, int dimy) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x >= dimx || y >= dimy) return;
  const double2 m = map[(size_t)y * dimx + x];
  const int ix = (int)floor(m.x), iy = (int)floor(m.y);
  uint16_t out = 0;
  if (ix >= 1 && iy >= 1 && ix + 2 < dimx && iy + 2 < dimy) {
    const double x01 = m.x - (double)ix, y01 = m.y - (double)iy;
    double arr[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int xx = ix - 1 + i;
      const double q0 = (double)__ldg(&src[(size_t)(iy - 1) * pitch + xx]);
      const double q1 = (double)__ldg(&src[(size_t)iy * pitch + xx]);
      const double q2 = (double)__ldg(&src[(size_t)(iy + 1) * pitch + xx]);
      const double q3 = (double)__ldg(&src[(size_t)(iy + 2) * pitch + xx]);
      arr[i] = cubic1(q0, q1, q2, q3, y01);
    }
    double r = floor(cubic1(arr[0], arr[1], arr[2], arr[3], x01) + 0.5);
    r = r < 0.0 ? 0.0 : (r > 65535.0 ? 65535.0 : r);
    out = (uint16_t)r;
  }
  dst[(size_t)y * pitch + x] = out;
}

void launch_remap_build(const double* params14, const double* trig4, double2* map, int dimx, int dimy,
                        cudaStream_t s) {
  Disto X;
  for (int i = 0; i < 14; ++i) X.p[i] = params14[i];
  for (int i = 0; i < 4; ++i) X.trig[i] = trig4[i];
  dim3 grid((dimx + 127) / 128, dimy);
  k_remap_build<<<grid, 128, 0, s>>>(X, map, dimx, dimy);
}

void launch_remap_apply(const double2* map, const uint16_t* src, uint16_t* dst, int pitch, int dimx, int dimy,
                        cudaStream_t s) {
  dim3 grid((dimx + 127) / 128, dimy);
  k_remap_apply<<<grid, 128, 0, s>>>(map, src, dst, pitch, dimx, dimy);
}

}  // namespace ptk
