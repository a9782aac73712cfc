// Register-tiled exact search (the plain form's fast kernel).
//
// Same results as k_search (every candidate's S1 = sum I1, S11 = sum I1^2 and
// S01 = sum I0*I1 exact, same ranking and tie rule), computed with far fewer
// instructions per pattern-pixel-candidate:
//
//  * The rotated pattern of a work item is scattered once into a dense
//    column-major FP64 map over its bounding box:
//        map(x, y) = sum over points at (x, y) of (I0 + 2^20)
//    i.e. the reference pixel sum plus 2^20 x the multiplicity M(x, y).
//  * For each map column, every thread (one x offset u, 8 consecutive y
//    offsets) streams its current-frame column in blocks of 8 values and
//    accumulates sum map(x, y) * I1(x+u, y+v) with FP64 FMAs, 8 rows x 8
//    candidates per chunk.  All operands and partial sums are integers below
//    2^51, so every FMA is exact:  acc = S01 + 2^20 S1.  Two 8-value register
//    blocks alternate (no register moves); the next block is loaded between
//    the two halves of a chunk's FMAs, hiding shared-memory latency.
//  * S1 and S11 come from the column's maximal runs of constant multiplicity:
//    a run's window sum is formed once and slid over the 8 candidates with
//    one add and one subtract per step (exact integer arithmetic).
//  * If a column has more runs than the per-column list holds (sparse custom
//    patterns), the work item computes S1 and S11 entry by entry instead.
//
// Thread layout: 256 threads; lane = x offset, warp w = y offsets
// 8 (w mod 4) .. 8 (w mod 4) + 7 of a 32x32 candidate tile, over the map
// columns of parity w / 4; the two column halves are summed through shared
// memory at the end.  The patch pitch is a template constant so every
// shared-memory address in the inner loop is a register plus an immediate.
#include <climits>

#include "ptk_internal.cuh"

namespace ptk {

namespace {

constexpr int kTT = 8;               // candidates per thread (along y) = rows per chunk
constexpr int kTiledThreads = 256;   // 2 column halves x 4 warps x 8 rows
constexpr int kRunsPerCol = 8;
constexpr int kMultShift = 20;       // map entry = I0 sum + multiplicity * 2^20
constexpr double kMult = 1048576.0;

__device__ __forceinline__ short2 rotate_round_t(short2 p, double c, double s) {
  const double px = (double)p.x, py = (double)p.y;
  const double xr = __dadd_rn(__dmul_rn(c, px), __dmul_rn(s, py));
  const double yr = __dadd_rn(__dmul_rn(-s, px), __dmul_rn(c, py));
  return make_short2((short)round(xr), (short)round(yr));
}

// exact uint16 -> double: bits of 2^52 + v, minus 2^52
__device__ __forceinline__ double u16d(unsigned v) {
  return __hiloint2double(0x43300000, (int)v) - 4503599627370496.0;
}

__device__ __forceinline__ bool better_t(double ncc, int idx, double bn, int bi) {
  return ncc > 0.0 && (ncc > bn || (ncc == bn && idx < bi));
}

struct TiledGeom {
  int mw, mh;  // map columns / rows (rows padded for the chunk loop)
  int ph;      // patch rows (the pitch is the template constant)
};

__host__ __device__ inline TiledGeom tiled_geom(int max_r) {
  TiledGeom t;
  const int box = 2 * max_r + 1;
  t.mw = box;
  t.mh = ((box + kTT - 1) / kTT) * kTT + 2 * kTT;
  t.ph = t.mh + kTileV + 2 * kTT;
  return t;
}

__host__ __device__ inline int tiled_pitch(int max_r) { return 2 * max_r + 1 + kTileU - 1 <= 128 ? 128 : 256; }

__host__ __device__ inline size_t tiled_map_bytes(int max_r) {
  const TiledGeom t = tiled_geom(max_r);
  size_t b = (size_t)t.mw * t.mh * 8;
  const size_t partial = (size_t)(kTiledThreads / 2) * kTT * 24;  // column-half partial sums
  return b < partial ? partial : b;
}

__host__ __device__ inline size_t tiled_smem(int max_r) {
  const TiledGeom t = tiled_geom(max_r);
  size_t b = tiled_map_bytes(max_r);
  b += (size_t)t.mw * kRunsPerCol * 4;  // runs
  b += (size_t)t.mw * 4 * 2;            // column extent + run count
  b = (b + 15) & ~(size_t)15;
  b += (size_t)tiled_pitch(max_r) * t.ph * 2;  // patch
  return b + 16;
}

}  // namespace

template <int PITCH>
__global__ void __launch_bounds__(kTiledThreads, 2) k_search_tiled(SearchLaunch p, int max_r) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_item, s_bbox[4], s_overflow;
  __shared__ double s_rn[kTiledThreads / 32];
  __shared__ int s_ri[kTiledThreads / 32];
  const TiledGeom G = tiled_geom(max_r);
  const size_t map_bytes = tiled_map_bytes(max_r);
  double* s_map = reinterpret_cast<double*>(smem);
  int* s_runs = reinterpret_cast<int*>(smem + map_bytes);
  int* s_ext = s_runs + G.mw * kRunsPerCol;  // packed (lo | hi << 16), empty column: lo > hi
  int* s_nrun = s_ext + G.mw;
  const size_t pofs = (map_bytes + (size_t)G.mw * kRunsPerCol * 4 + (size_t)G.mw * 8 + 15) & ~(size_t)15;
  uint16_t* s_patch = reinterpret_cast<uint16_t*>(smem + pofs);
  // partial sums of the second column half reuse the map region after the FMAs
  double* s_pacc = reinterpret_cast<double*>(smem);
  unsigned long long* s_p11 = reinterpret_cast<unsigned long long*>(smem + (size_t)(kTiledThreads / 2) * kTT * 8);
  unsigned* s_p1 = reinterpret_cast<unsigned*>(smem + (size_t)(kTiledThreads / 2) * kTT * 16);

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int half = warp >> 2;       // column parity handled by this warp
  const int rb = kTT * (warp & 3);  // first y offset (within the tile) of this thread
  const int pidx = tid & (kTiledThreads / 2 - 1);
  const int count = *p.list_count;
  const int per_grain = p.nrot * p.tiles_u * p.tiles_v;
  long long total = (long long)count * per_grain;
  if (total > p.max_items) total = p.max_items;
  const int NU = p.left + p.right + 1, NV = p.up + p.down + 1;
  const GrainsDev& g = p.g;

  for (;;) {
    if (tid == 0) s_item = atomicAdd(p.work_next, 1);
    __syncthreads();
    const int item = s_item;
    if (item >= total) break;
    const int li = item / per_grain;
    const int rem = item - li * per_grain;
    const int r = rem / (p.tiles_u * p.tiles_v);
    const int t = rem - r * (p.tiles_u * p.tiles_v);
    const int tu = t / p.tiles_v, tv = t - tu * p.tiles_v;
    const int gi = p.list[li];
    const int b = g.pstart[gi], P = g.pstart[gi + 1] - b;
    if (g.masked[gi] || (g.flags[gi] & 2) || P <= 0 || P > kMaxPatternPoints) {
      if (tid == 0) p.best[item] = SearchBest{0.0, INT_MAX, 0};
      __syncthreads();
      continue;
    }
    const double total_rot = (g.refrot[gi] + g.drot[gi]) + p.steps[r];
    double s1, c1;
    sincos(total_rot, &s1, &c1);
    const int gdx = (int)round(g.dx[gi]);
    const int gdy = (int)round(g.dy[gi]);

    // (a) bounding box of the rotated pattern
    if (tid == 0) {
      s_bbox[0] = INT_MAX;
      s_bbox[1] = INT_MIN;
      s_bbox[2] = INT_MAX;
      s_bbox[3] = INT_MIN;
      s_overflow = 0;
    }
    __syncthreads();
    int xmn = INT_MAX, xmx = INT_MIN, ymn = INT_MAX, ymx = INT_MIN;
    for (int i = tid; i < P; i += kTiledThreads) {
      const short2 q = rotate_round_t(g.pat[b + i], c1, s1);
      xmn = min(xmn, (int)q.x);
      xmx = max(xmx, (int)q.x);
      ymn = min(ymn, (int)q.y);
      ymx = max(ymx, (int)q.y);
    }
    for (int o = 16; o > 0; o >>= 1) {
      xmn = min(xmn, __shfl_xor_sync(0xffffffffu, xmn, o));
      xmx = max(xmx, __shfl_xor_sync(0xffffffffu, xmx, o));
      ymn = min(ymn, __shfl_xor_sync(0xffffffffu, ymn, o));
      ymx = max(ymx, __shfl_xor_sync(0xffffffffu, ymx, o));
    }
    if (lane == 0) {
      atomicMin(&s_bbox[0], xmn);
      atomicMax(&s_bbox[1], xmx);
      atomicMin(&s_bbox[2], ymn);
      atomicMax(&s_bbox[3], ymx);
    }
    __syncthreads();
    const int bx0 = s_bbox[0], bx1 = s_bbox[1], by0 = s_bbox[2], by1 = s_bbox[3];
    const int bw = bx1 - bx0 + 1, bh = by1 - by0 + 1;
    const int u0 = -p.left + tu * kTileU, u1 = min(u0 + kTileU - 1, p.right);
    const int v0 = -p.up + tv * kTileV, v1 = min(v0 + kTileV - 1, p.down);
    const int X0 = g.refx[gi] + gdx + bx0 + u0;
    const int Y0 = g.refy[gi] + gdy + by0 + v0;
    const int needw = bw + (u1 - u0), needh = bh + (v1 - v0);
    const bool oob = X0 < 0 || Y0 < 0 || X0 + needw > p.cur.dimx || Y0 + needh > p.cur.dimy;
    const int mh = ((bh + kTT - 1) / kTT) * kTT + 2 * kTT;  // rows of this item's map
    const bool fits = bw <= G.mw && mh <= G.mh && bw + kTileU - 1 <= PITCH;
    if (oob || !fits) {
      if (tid == 0) {
        if (oob) atomicOr(&g.flags[gi], 1);
        else atomicOr(&g.flags[gi], 4);  // does not fit the tiled layout (not expected: host sizes it)
        p.best[item] = SearchBest{0.0, INT_MAX, 0};
      }
      __syncthreads();
      continue;
    }

    // (b) zero the map, (c) scatter I0 + 2^20 per point
    for (int e = tid; e < bw * mh; e += kTiledThreads) s_map[e] = 0.0;
    __syncthreads();
    for (int i = tid; i < P; i += kTiledThreads) {
      const short2 q = rotate_round_t(g.pat[b + i], c1, s1);
      atomicAdd(&s_map[(q.x - bx0) * mh + (q.y - by0)], (double)g.w0[b + i] + kMult);
    }
    // (e) stage the patch: rows [0, needh) x columns [0, needw); the rest
    // (reached only by zero weights or by candidates outside the zone) is zero
    const int ph = mh + kTileV + 2 * kTT;
    for (int e = tid; e < PITCH * ph; e += kTiledThreads) {
      const int yy = e / PITCH, xx = e - yy * PITCH;
      uint16_t v = 0;
      if (yy < needh && xx < needw) v = p.cur.pix[(size_t)(Y0 + yy) * p.cur.pitch + (X0 + xx)];
      s_patch[e] = v;
    }
    __syncthreads();
    // (d) per column: extent of non-zero rows and runs of constant multiplicity
    for (int x = tid; x < bw; x += kTiledThreads) {
      const double* col = s_map + x * mh;
      int lo = INT_MAX, hi = -1, nr = 0, cur_m = 0, start = 0;
      for (int y = 0; y <= bh; ++y) {
        const int m = y < bh ? (int)(col[y] * (1.0 / kMult)) : 0;
        if (m != 0) {
          lo = min(lo, y);
          hi = y;
        }
        if (m != cur_m) {
          if (cur_m != 0) {
            if (nr < kRunsPerCol) s_runs[x * kRunsPerCol + nr] = start | ((y - 1) << 8) | (cur_m << 16);
            ++nr;
          }
          cur_m = m;
          start = y;
        }
      }
      s_ext[x] = hi < 0 ? 1 : (lo | (hi << 16));
      s_nrun[x] = nr;
      if (nr > kRunsPerCol) atomicOr(&s_overflow, 1);
    }
    __syncthreads();

    // (f) candidates: x offset u0 + lane, y offsets v0 + rb + 0..7, map columns of parity `half`
    double acc[kTT];
    unsigned S1[kTT];
    unsigned long long S11[kTT];
#pragma unroll
    for (int k = 0; k < kTT; ++k) {
      acc[k] = 0.0;
      S1[k] = 0;
      S11[k] = 0;
    }
    const bool overflow = s_overflow != 0;
    for (int x = half; x < bw; x += 2) {
      const int ext = s_ext[x];
      const int lo = ext & 0xffff, hi = ext >> 16;
      if (lo > hi) continue;
      // column of this thread from row lo + rb, in blocks of 8 rows
      const uint16_t* cp = s_patch + (lo + rb) * PITCH + x + lane;
      const double* wp = s_map + x * mh + lo;
      double A[kTT], B[kTT];
#pragma unroll
      for (int k = 0; k < kTT; ++k) A[k] = u16d(cp[k * PITCH]);
#pragma unroll
      for (int k = 0; k < kTT; ++k) B[k] = u16d(cp[(kTT + k) * PITCH]);
      // chunk c uses (A, B) = row blocks c, c+1; block c+2 is loaded into A
      // between the FMAs that read A and those that read only B
      int nchunk = (hi - lo) / kTT + 1;
      for (;;) {
        {
          double w[kTT];
#pragma unroll
          for (int j = 0; j < kTT; ++j) w[j] = wp[j];
#pragma unroll
          for (int j = 0; j < kTT; ++j)
#pragma unroll
            for (int k = 0; k < kTT; ++k)
              if (j + k < kTT) acc[k] = fma(w[j], A[j + k], acc[k]);
          cp += kTT * PITCH;
#pragma unroll
          for (int k = 0; k < kTT; ++k) A[k] = u16d(cp[(kTT + k) * PITCH]);
#pragma unroll
          for (int j = 0; j < kTT; ++j)
#pragma unroll
            for (int k = 0; k < kTT; ++k)
              if (j + k >= kTT) acc[k] = fma(w[j], B[j + k - kTT], acc[k]);
          wp += kTT;
        }
        if (--nchunk == 0) break;
        {
          double w[kTT];
#pragma unroll
          for (int j = 0; j < kTT; ++j) w[j] = wp[j];
#pragma unroll
          for (int j = 0; j < kTT; ++j)
#pragma unroll
            for (int k = 0; k < kTT; ++k)
              if (j + k < kTT) acc[k] = fma(w[j], B[j + k], acc[k]);
          cp += kTT * PITCH;
#pragma unroll
          for (int k = 0; k < kTT; ++k) B[k] = u16d(cp[(kTT + k) * PITCH]);
#pragma unroll
          for (int j = 0; j < kTT; ++j)
#pragma unroll
            for (int k = 0; k < kTT; ++k)
              if (j + k >= kTT) acc[k] = fma(w[j], A[j + k - kTT], acc[k]);
          wp += kTT;
        }
        if (--nchunk == 0) break;
      }
      const uint16_t* colp = s_patch + rb * PITCH + x + lane;
      if (!overflow) {
        const int nr = s_nrun[x];
        for (int q = 0; q < nr; ++q) {
          const int rr = s_runs[x * kRunsPerCol + q];
          const int a = rr & 0xff, e = (rr >> 8) & 0xff;
          const unsigned m = (unsigned)(rr >> 16);
          unsigned sm = 0;
          unsigned long long s2 = 0;
          for (int y = a; y <= e; ++y) {
            const unsigned val = colp[y * PITCH];
            sm += val;
            s2 += (unsigned long long)(val * val);
          }
#pragma unroll
          for (int k = 0; k < kTT; ++k) {
            if (k > 0) {
              const unsigned vin = colp[(e + k) * PITCH];
              const unsigned vout = colp[(a + k - 1) * PITCH];
              sm = sm + vin - vout;
              s2 = s2 + (unsigned long long)(vin * vin) - (unsigned long long)(vout * vout);
            }
            S1[k] += m * sm;
            S11[k] += (unsigned long long)m * s2;
          }
        }
      } else {
        // entry by entry: every non-zero map entry of the column with its multiplicity
        const double* wcol = s_map + x * mh;
        for (int y = lo; y <= hi; ++y) {
          const unsigned m = (unsigned)(int)(wcol[y] * (1.0 / kMult));
          if (!m) continue;
#pragma unroll
          for (int k = 0; k < kTT; ++k) {
            const unsigned val = colp[(y + k) * PITCH];
            S1[k] += m * val;
            S11[k] += (unsigned long long)m * (unsigned long long)(val * val);
          }
        }
      }
    }
    // sum the two column halves (the map is no longer needed)
    __syncthreads();
    if (half == 1) {
#pragma unroll
      for (int k = 0; k < kTT; ++k) {
        s_pacc[k * (kTiledThreads / 2) + pidx] = acc[k];
        s_p11[k * (kTiledThreads / 2) + pidx] = S11[k];
        s_p1[k * (kTiledThreads / 2) + pidx] = S1[k];
      }
    }
    __syncthreads();
    double bn = 0.0;
    int bi = INT_MAX;
    if (half == 0) {
      const long long Pl = P, S0 = g.s0[gi];
      const double den1 = (double)(Pl * g.s00[gi] - S0 * S0);
      const int u = u0 + lane;
#pragma unroll
      for (int k = 0; k < kTT; ++k) {
        const double a = acc[k] + s_pacc[k * (kTiledThreads / 2) + pidx];
        const unsigned s1k = S1[k] + s_p1[k * (kTiledThreads / 2) + pidx];
        const unsigned long long s11k = S11[k] + s_p11[k * (kTiledThreads / 2) + pidx];
        const int v = v0 + rb + k;
        if (u > u1 || v > v1) continue;
        const long long s01 = __double2ll_rn(a) - ((long long)s1k << kMultShift);
        const long long num = Pl * s01 - S0 * (long long)s1k;
        const long long d2 = Pl * (long long)s11k - (long long)s1k * (long long)s1k;
        const double ncc = (double)num / sqrt(den1 * (double)d2);
        const int idx = (r * NU + (u + p.left)) * NV + (v + p.up);
        if (better_t(ncc, idx, bn, bi)) {
          bn = ncc;
          bi = idx;
        }
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      const double on = __shfl_xor_sync(0xffffffffu, bn, o);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (better_t(on, oi, bn, bi)) {
        bn = on;
        bi = oi;
      }
    }
    if (lane == 0) {
      s_rn[warp] = bn;
      s_ri[warp] = bi;
    }
    __syncthreads();
    if (tid == 0) {
      double fn = 0.0;
      int fi = INT_MAX;
      for (int k = 0; k < kTiledThreads / 32; ++k)
        if (better_t(s_rn[k], s_ri[k], fn, fi)) {
          fn = s_rn[k];
          fi = s_ri[k];
        }
      p.best[item] = SearchBest{fn, fi, 0};
    }
    __syncthreads();
  }
}

size_t search_tiled_smem(int max_r) { return tiled_smem(max_r); }

int search_tiled_occupancy(size_t smem, int max_r) {
  int blocks = 0;
  if (tiled_pitch(max_r) == 128) {
    ensure_smem((const void*)k_search_tiled<128>, smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_search_tiled<128>, kTiledThreads, smem);
  } else {
    ensure_smem((const void*)k_search_tiled<256>, smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_search_tiled<256>, kTiledThreads, smem);
  }
  return blocks;
}

void launch_search_tiled(const SearchLaunch& p, int max_r, int grid, size_t smem, cudaStream_t s) {
  search_tiled_occupancy(smem, max_r);
  if (tiled_pitch(max_r) == 128) k_search_tiled<128><<<grid, kTiledThreads, smem, s>>>(p, max_r);
  else k_search_tiled<256><<<grid, kTiledThreads, smem, s>>>(p, max_r);
}

}  // namespace ptk
