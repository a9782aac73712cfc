// Grey frames from unpacked RAW sensor mosaics on sm_100a: the demosaic
// modes of read_raw_image (src/p-tracker.cpp:288-372) and its optional grey
// level rescale (:374-383).
//
//   -1   floor of the mean of the 2x2 block whose top-left is the pixel,
//   -2   floor of the 1-2-1 x 1-2-1 (/16) weighted mean of the 3x3 block
//        centred on it,
//   -20  the raw value (achromatic sensors).
//
// The stencil addresses the flat raw array at (left + x + i) +
// raw_width * (top + y + j), as the reference does; the host checks that
// every index lies in the array.  The reference forms these means in double
// from 0.25 / 0.125 / 0.0625 weights: every product and partial sum is exact
// in double (at most 16 + 4 significant bits), so the floor of the mean is
// the integer sum shifted right by 2 or 4, which is what the kernel computes.
// The rescale, floor((v - MinGray) * (65535.0 / (MaxGray - MinGray))), is
// done in double with one correctly rounded division and one product, as on
// the CPU (this file is compiled with -fmad=false).
//
// One pass reads the mosaic (2 bytes per pixel, the 3x3 neighbours come from
// L1) and writes the frame (2 bytes per pixel), two pixels per thread, rows
// grid-strided over a grid of a few CTAs per SM; each CTA folds its pixels'
// minimum and maximum into one atomicMin/atomicMax.  The rescale, when
// asked for, is a second pass over the frame that reads the extremes from
// device memory, so nothing returns to the host in between.
#include "ptk_internal.cuh"

namespace ptk {

namespace {

constexpr int kRawThreads = 128;  // 2 pixels each: 256 columns per CTA row

template <int MODE>
__device__ __forceinline__ unsigned raw_pixel(const uint16_t* __restrict__ raw, long long idx, int w) {
  if (MODE == -20) return __ldg(raw + idx);
  if (MODE == -1) {
    const unsigned s = (unsigned)__ldg(raw + idx) + __ldg(raw + idx + 1) + __ldg(raw + idx + w + 1) +
                       __ldg(raw + idx + w);
    return s >> 2;
  }
  const uint16_t* r0 = raw + idx - w;
  const uint16_t* r1 = raw + idx;
  const uint16_t* r2 = raw + idx + w;
  const unsigned s = (unsigned)__ldg(r0 - 1) + 2u * __ldg(r0) + __ldg(r0 + 1) + 2u * __ldg(r1 - 1) + 4u * __ldg(r1) +
                     2u * __ldg(r1 + 1) + __ldg(r2 - 1) + 2u * __ldg(r2) + __ldg(r2 + 1);
  return s >> 4;
}

template <int MODE>
__global__ void __launch_bounds__(kRawThreads) k_raw_demosaic(const uint16_t* __restrict__ raw, int raw_width,
                                                              int left, int top, uint16_t* __restrict__ dst,
                                                              int pitch, int dimx, int dimy, unsigned* min_max) {
  unsigned mn = 0xffffffffu, mx = 0u;
  const int x = (blockIdx.x * kRawThreads + threadIdx.x) * 2;
  if (x < dimx) {
    for (int y = blockIdx.y; y < dimy; y += gridDim.y) {
      const long long idx = (long long)(left + x) + (long long)raw_width * (top + y);
      const unsigned a = raw_pixel<MODE>(raw, idx, raw_width);
      mn = min(mn, a);
      mx = max(mx, a);
      uint16_t* row = dst + (size_t)y * pitch;
      if (x + 1 < dimx) {
        const unsigned b = raw_pixel<MODE>(raw, idx + 1, raw_width);
        mn = min(mn, b);
        mx = max(mx, b);
        *reinterpret_cast<unsigned*>(row + x) = a | (b << 16);  // x even, rows 128-byte aligned
      } else {
        row[x] = (uint16_t)a;
      }
    }
  }
  mn = __reduce_min_sync(0xffffffffu, mn);
  mx = __reduce_max_sync(0xffffffffu, mx);
  __shared__ unsigned s_mn[kRawThreads / 32], s_mx[kRawThreads / 32];
  if ((threadIdx.x & 31) == 0) {
    s_mn[threadIdx.x >> 5] = mn;
    s_mx[threadIdx.x >> 5] = mx;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < kRawThreads / 32; ++k) {
      mn = min(mn, s_mn[k]);
      mx = max(mx, s_mx[k]);
    }
    if (mn != 0xffffffffu) {
      atomicMin(min_max, mn);
      atomicMax(min_max + 1, mx);
    }
  }
}

__global__ void __launch_bounds__(kRawThreads) k_raw_rescale(uint16_t* __restrict__ dst, int pitch, int dimx,
                                                             int dimy, const unsigned* min_max) {
  const unsigned mn = min_max[0], mx = min_max[1];
  if (mx <= mn) return;  // all pixels equal: left as they are
  const double fact = 65535.0 / (double)(int)(mx - mn);
  const int x = (blockIdx.x * kRawThreads + threadIdx.x) * 2;
  if (x >= dimx) return;
  for (int y = blockIdx.y; y < dimy; y += gridDim.y) {
    uint16_t* row = dst + (size_t)y * pitch;
    const int n = x + 1 < dimx ? 2 : 1;
    for (int k = 0; k < n; ++k) {
      const double v = (double)((int)row[x + k] - (int)mn) * fact;
      row[x + k] = (uint16_t)(unsigned)floor(v);
    }
  }
}

}  // namespace

int raw_stencil_lo(int mode) { return mode == -2 ? -1 : 0; }
int raw_stencil_hi(int mode) { return mode == -20 ? 0 : 1; }

void launch_raw_demosaic(const uint16_t* raw, int raw_width, int left, int top, int mode, int rescale, uint16_t* dst,
                         int pitch, int dimx, int dimy, unsigned* min_max, int num_sms, cudaStream_t s) {
  cudaMemsetAsync(min_max, 0xff, sizeof(unsigned), s);
  cudaMemsetAsync(min_max + 1, 0, sizeof(unsigned), s);
  const int gx = (dimx + 2 * kRawThreads - 1) / (2 * kRawThreads);
  int gy = (num_sms * 16 + gx - 1) / gx;  // 16 CTAs of 128 threads per SM
  if (gy > dimy) gy = dimy;
  const dim3 grid(gx, gy);
  if (mode == -1)
    k_raw_demosaic<-1><<<grid, kRawThreads, 0, s>>>(raw, raw_width, left, top, dst, pitch, dimx, dimy, min_max);
  else if (mode == -2)
    k_raw_demosaic<-2><<<grid, kRawThreads, 0, s>>>(raw, raw_width, left, top, dst, pitch, dimx, dimy, min_max);
  else
    k_raw_demosaic<-20><<<grid, kRawThreads, 0, s>>>(raw, raw_width, left, top, dst, pitch, dimx, dimy, min_max);
  if (rescale) k_raw_rescale<<<grid, kRawThreads, 0, s>>>(dst, pitch, dimx, dimy, min_max);
}

}  // namespace ptk
