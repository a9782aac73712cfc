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
// One pass reads the mosaic (2 bytes per pixel, plus the halo rows of 8-row
// strips, which L2 serves) and writes the frame (2 bytes per pixel) - 8
// pixels per thread with 16-byte accesses when the mosaic rows start 16-byte
// aligned, else 2 per thread - and each CTA folds its pixels' minimum and
// maximum into one atomicMin/atomicMax.  The rescale, when
// asked for, is a second pass over the frame that reads the extremes from
// device memory, so nothing returns to the host in between.
#include "ptk_internal.cuh"

namespace ptk {

namespace {

constexpr int kRawThreads = 128;  // demosaic: 2 pixels each (256 columns per CTA); rescale: 8 pixels each
constexpr int kRawRows = 8;       // rows of one demosaic CTA's strip

// Horizontal sums of one mosaic row for the thread's two pixels a (column c)
// and b (column c + 1), c the flat index of pixel a in that row:
// -1: v[c] + v[c+1], v[c+1] + v[c+2];  -2: v[c-1] + 2 v[c] + v[c+1], v[c] + 2 v[c+1] + v[c+2];
// -20: v[c], v[c+1].  `two` = pixel b exists.
template <int MODE>
__device__ __forceinline__ void raw_hsum(const uint16_t* __restrict__ raw, long long c, bool two, unsigned& ha,
                                         unsigned& hb) {
  if (MODE == -20) {
    ha = __ldg(raw + c);
    hb = two ? __ldg(raw + c + 1) : 0u;
  } else if (MODE == -1) {
    const unsigned v0 = __ldg(raw + c), v1 = __ldg(raw + c + 1);
    ha = v0 + v1;
    hb = two ? v1 + __ldg(raw + c + 2) : 0u;
  } else {
    const unsigned vm = __ldg(raw + c - 1), v0 = __ldg(raw + c), v1 = __ldg(raw + c + 1);
    ha = vm + 2u * v0 + v1;
    hb = two ? v0 + 2u * v1 + __ldg(raw + c + 2) : 0u;
  }
}

// One CTA = 256 columns x kRawRows rows.  Each thread requests the
// horizontal sums of all mosaic rows its two columns of the strip need (the
// strip plus the stencil's halo rows) before any arithmetic, so a thread has
// some 40 loads in flight instead of one chain of dependent rows; each CTA
// folds its pixels' min/max into two atomics.
template <int MODE>
__global__ void __launch_bounds__(kRawThreads) k_raw_demosaic(const uint16_t* __restrict__ raw, int raw_width,
                                                              int left, int top, uint16_t* __restrict__ dst,
                                                              int pitch, int dimx, int dimy, unsigned* min_max) {
  unsigned mn = 0xffffffffu, mx = 0u;
  const int x = (blockIdx.x * kRawThreads + threadIdx.x) * 2;
  const int y0 = blockIdx.y * kRawRows;
  const int y1 = min(dimy, y0 + kRawRows);
  if (x < dimx) {
    const bool two = x + 1 < dimx;
    const long long w = raw_width;
    // rows of the stencil relative to the pixel's row: -1 .. 1 (-2), 0 .. 1 (-1), 0 (-20)
    constexpr int kLo = MODE == -2 ? -1 : 0, kHi = MODE == -20 ? 0 : 1;
    constexpr int kIn = kRawRows + kHi - kLo;  // mosaic rows the strip reads
    const long long c = (long long)(left + x) + w * (top + y0 + kLo);  // flat index, first mosaic row
    // every mosaic row of the strip is requested before any arithmetic
    unsigned ha[kIn], hb[kIn];
#pragma unroll
    for (int r = 0; r < kIn; ++r) {
      ha[r] = hb[r] = 0u;
      if (y0 + r + kLo <= y1 - 1 + kHi) raw_hsum<MODE>(raw, c + w * r, two, ha[r], hb[r]);
    }
    uint16_t* row = dst + (size_t)y0 * pitch + x;
#pragma unroll
    for (int r = 0; r < kRawRows; ++r) {
      if (y0 + r < y1) {
        unsigned a, b;
        if (MODE == -20) {
          a = ha[r];
          b = hb[r];
        } else if (MODE == -1) {
          a = (ha[r] + ha[r + 1]) >> 2;
          b = (hb[r] + hb[r + 1]) >> 2;
        } else {
          a = (ha[r] + 2u * ha[r + 1] + ha[r + 2]) >> 4;
          b = (hb[r] + 2u * hb[r + 1] + hb[r + 2]) >> 4;
        }
        mn = min(mn, a);
        mx = max(mx, a);
        if (two) {
          mn = min(mn, b);
          mx = max(mx, b);
          *reinterpret_cast<unsigned*>(row) = a | (b << 16);  // x even, rows 128-byte aligned
        } else {
          *row = (uint16_t)a;
        }
      }
      row += pitch;
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

// Fast path when every mosaic row's first frame pixel is 16-byte aligned
// (left margin and raw width multiples of 8, mosaic 16-byte aligned): a thread
// takes 8 columns, reads each mosaic row of its strip with one 16-byte load
// (elements past the checked range one by one, or not at all), gets the left
// and right neighbours from the adjacent lanes (the warp's edge lanes read
// theirs), and writes 8 pixels with one 16-byte store.
constexpr int kVecThreads = 128;  // 8 columns each: 1024 columns per CTA
template <int MODE>
__global__ void __launch_bounds__(kVecThreads) k_raw_demosaic8(const uint16_t* __restrict__ raw, int raw_width,
                                                               int left, int top, uint16_t* __restrict__ dst,
                                                               int pitch, int dimx, int dimy, unsigned* min_max) {
  constexpr int kLo = MODE == -2 ? -1 : 0, kHi = MODE == -20 ? 0 : 1;
  constexpr int kIn = kRawRows + kHi - kLo;
  const int lane = threadIdx.x & 31;
  const int x0 = (blockIdx.x * kVecThreads + threadIdx.x) * 8;
  const int y0 = blockIdx.y * kRawRows;
  const int y1 = min(dimy, y0 + kRawRows);
  const long long w = raw_width;
  const int xlim = dimx - 1 + kHi;  // last mosaic column (relative to left) the host checked
  const long long c0 = (long long)(left + x0) + w * (top + y0 + kLo);
  unsigned mn = 0xffffffffu, mx = 0u;
  // horizontal sums of the strip's mosaic rows for the 8 columns (up to 18 bits)
  uint32_t hs[kIn][8];
#pragma unroll
  for (int r = 0; r < kIn; ++r) {
    uint32_t v[4] = {0u, 0u, 0u, 0u};
    uint32_t vl = 0u, vr = 0u;  // elements x0 - 1 and x0 + 8 (edge lanes only)
    const bool row_ok = y0 + r + kLo <= y1 - 1 + kHi;
    const long long c = c0 + w * r;
    if (row_ok) {
      if (x0 + 7 <= xlim) {
        const uint4 q = __ldg(reinterpret_cast<const uint4*>(raw + c));
        v[0] = q.x;
        v[1] = q.y;
        v[2] = q.z;
        v[3] = q.w;
      } else {
        for (int k = 0; k < 8; ++k)
          if (x0 + k <= xlim) v[k >> 1] |= (uint32_t)__ldg(raw + c + k) << (16 * (k & 1));
      }
      if (MODE == -2 && lane == 0 && x0 - 1 <= xlim) vl = __ldg(raw + c - 1);
      if (MODE != -20 && lane == 31 && x0 + 8 <= xlim) vr = __ldg(raw + c + 8);
    }
    if (MODE == -20) {
#pragma unroll
      for (int k = 0; k < 8; ++k) hs[r][k] = (v[k >> 1] >> (16 * (k & 1))) & 0xffffu;
      continue;
    }
    const uint32_t from_left = __shfl_up_sync(0xffffffffu, v[3] >> 16, 1);
    const uint32_t from_right = __shfl_down_sync(0xffffffffu, v[0] & 0xffffu, 1);
    if (lane != 0) vl = from_left;
    if (lane != 31) vr = from_right;
    uint32_t e[10];  // elements x0 - 1 .. x0 + 8
    e[0] = vl;
#pragma unroll
    for (int k = 0; k < 8; ++k) e[k + 1] = (v[k >> 1] >> (16 * (k & 1))) & 0xffffu;
    e[9] = vr;
#pragma unroll
    for (int k = 0; k < 8; ++k) hs[r][k] = MODE == -1 ? e[k + 1] + e[k + 2] : e[k] + 2u * e[k + 1] + e[k + 2];
  }
  if (x0 < dimx) {
    uint16_t* out = dst + (size_t)y0 * pitch + x0;
#pragma unroll
    for (int r = 0; r < kRawRows; ++r) {
      if (y0 + r < y1) {
        uint32_t px[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          if (MODE == -20) px[k] = hs[r][k];
          else if (MODE == -1) px[k] = (hs[r][k] + hs[r + 1][k]) >> 2;
          else px[k] = (hs[r][k] + 2u * hs[r + 1][k] + hs[r + 2][k]) >> 4;
          if (x0 + k < dimx) {
            mn = min(mn, px[k]);
            mx = max(mx, px[k]);
          }
        }
        if (x0 + 7 < dimx) {
          *reinterpret_cast<uint4*>(out) = make_uint4(px[0] | (px[1] << 16), px[2] | (px[3] << 16),
                                                      px[4] | (px[5] << 16), px[6] | (px[7] << 16));
        } else {
          for (int k = 0; x0 + k < dimx; ++k) out[k] = (uint16_t)px[k];
        }
      }
      out += pitch;
    }
  }
  mn = __reduce_min_sync(0xffffffffu, mn);
  mx = __reduce_max_sync(0xffffffffu, mx);
  __shared__ unsigned s_mn[kVecThreads / 32], s_mx[kVecThreads / 32];
  if (lane == 0) {
    s_mn[threadIdx.x >> 5] = mn;
    s_mx[threadIdx.x >> 5] = mx;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < kVecThreads / 32; ++k) {
      mn = min(mn, s_mn[k]);
      mx = max(mx, s_mx[k]);
    }
    if (mn != 0xffffffffu) {
      atomicMin(min_max, mn);
      atomicMax(min_max + 1, mx);
    }
  }
}

__device__ __forceinline__ unsigned rescale1(unsigned v, unsigned mn, double fact) {
  return (unsigned)floor((double)((int)v - (int)mn) * fact);
}

// Rescale: 8 pixels per thread (16-byte accesses; rows are 128-byte
// aligned), the row's last dimx % 8 pixels one by one; a CTA row per frame row.
__global__ void __launch_bounds__(kRawThreads) k_raw_rescale(uint16_t* __restrict__ dst, int pitch, int dimx,
                                                             int dimy, const unsigned* min_max) {
  const unsigned mn = min_max[0], mx = min_max[1];
  if (mx <= mn) return;  // all pixels equal: left as they are
  const double fact = 65535.0 / (double)(int)(mx - mn);
  const int x = (blockIdx.x * kRawThreads + threadIdx.x) * 8;
  if (x >= dimx) return;
  for (int y = blockIdx.y; y < dimy; y += gridDim.y) {
    uint16_t* row = dst + (size_t)y * pitch;
    if (x + 8 <= dimx) {
      uint4 v = *reinterpret_cast<const uint4*>(row + x);
      unsigned* u = reinterpret_cast<unsigned*>(&v);
#pragma unroll
      for (int k = 0; k < 4; ++k)
        u[k] = rescale1(u[k] & 0xffffu, mn, fact) | (rescale1(u[k] >> 16, mn, fact) << 16);
      *reinterpret_cast<uint4*>(row + x) = v;
    } else {
      for (int k = x; k < dimx; ++k) row[k] = (uint16_t)rescale1(row[k], mn, fact);
    }
  }
}

}  // namespace

int raw_stencil_lo(int mode) { return mode == -2 ? -1 : 0; }
int raw_stencil_hi(int mode) { return mode == -20 ? 0 : 1; }

void launch_raw_demosaic(const uint16_t* raw, int raw_width, int left, int top, int mode, int rescale, uint16_t* dst,
                         int pitch, int dimx, int dimy, unsigned* min_max, int num_sms, cudaStream_t s) {
  (void)num_sms;
  cudaMemsetAsync(min_max, 0xff, sizeof(unsigned), s);
  cudaMemsetAsync(min_max + 1, 0, sizeof(unsigned), s);
  if (left % 8 == 0 && raw_width % 8 == 0 && reinterpret_cast<uintptr_t>(raw) % 16 == 0) {
    const dim3 gv((dimx + 8 * kVecThreads - 1) / (8 * kVecThreads), (dimy + kRawRows - 1) / kRawRows);
    if (mode == -1)
      k_raw_demosaic8<-1><<<gv, kVecThreads, 0, s>>>(raw, raw_width, left, top, dst, pitch, dimx, dimy, min_max);
    else if (mode == -2)
      k_raw_demosaic8<-2><<<gv, kVecThreads, 0, s>>>(raw, raw_width, left, top, dst, pitch, dimx, dimy, min_max);
    else
      k_raw_demosaic8<-20><<<gv, kVecThreads, 0, s>>>(raw, raw_width, left, top, dst, pitch, dimx, dimy, min_max);
  } else {
    const dim3 grid((dimx + 2 * kRawThreads - 1) / (2 * kRawThreads), (dimy + kRawRows - 1) / kRawRows);
    if (mode == -1)
      k_raw_demosaic<-1><<<grid, kRawThreads, 0, s>>>(raw, raw_width, left, top, dst, pitch, dimx, dimy, min_max);
    else if (mode == -2)
      k_raw_demosaic<-2><<<grid, kRawThreads, 0, s>>>(raw, raw_width, left, top, dst, pitch, dimx, dimy, min_max);
    else
      k_raw_demosaic<-20><<<grid, kRawThreads, 0, s>>>(raw, raw_width, left, top, dst, pitch, dimx, dimy, min_max);
  }
  if (rescale) {
    const int rx = (dimx + 8 * kRawThreads - 1) / (8 * kRawThreads);
    const int ry = dimy < 65535 ? dimy : 65535;  // one frame row per CTA row (grid-strided beyond)
    k_raw_rescale<<<dim3(rx, ry), kRawThreads, 0, s>>>(dst, pitch, dimx, dimy, min_max);
  }
}

}  // namespace ptk
