// Exact integer-pixel + rotation-step NCC search on sm_100a (the plain form).
//
// Reference semantics (src/p-tracker.cpp:659-1016): for every rotation step of
// the zone (outer loop), every x offset u (middle) and y offset v (inner), the
// pattern rotated by refrot + drot + step and rounded is correlated with the
// current frame at refcoord + round(d) + (u, v); the first strict maximum of
// NCC above 0 wins (best_NCC starts at 0.0, `if (best_NCC < NCC_test)`).
//
// Instead of the reference's two FP64 passes per candidate, each candidate
// accumulates three exact integer sums over the P pattern points,
//   S1 = sum I1,  S11 = sum I1^2,  S01 = sum I0 * I1,
// and NCC = (P S01 - S0 S1) / sqrt((P S00 - S0^2)(P S11 - S1^2)), which is the
// reference's C0C1 / sqrt(C0C0 C1C1) with every cancellation done exactly in
// int64 (P <= 16384, 16-bit pixels: all terms stay below 2^61).  Candidates
// are therefore ranked on values within one rounding of the exact NCC.
//
// Work decomposition: one work item = (grain, rotation step, 32x32 candidate
// tile).  A persistent grid pulls items from a device work queue (level 0:
// grains ordered by decreasing pattern size, so heavy items start first;
// levels 1/2: the device-built rescue lists), stages the rotated pattern and
// the current-frame patch in shared memory, evaluates up to 1024 candidates
// (lane = x offset, 4 y offsets per thread) and writes the item's best
// (NCC, order index).  k_finalize reduces items per grain in the reference's
// iteration order and applies the stage's acceptance rule.
#include <climits>

#include "ptk_internal.cuh"

namespace ptk {

// rotate_pixel_pattern (src/p-tracker.cpp:615-621): FP64 without FMA
// contraction, then round half away from zero.
__device__ __forceinline__ short2 rotate_round(short2 p, double c, double s) {
  const double px = (double)p.x, py = (double)p.y;
  const double xr = __dadd_rn(__dmul_rn(c, px), __dmul_rn(s, py));
  const double yr = __dadd_rn(__dmul_rn(-s, px), __dmul_rn(c, py));
  return make_short2((short)round(xr), (short)round(yr));
}

__device__ __forceinline__ long long warp_sum_ll(long long v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// ---------------------------------------------------------------------------
// do_precomputations (src/p-tracker.cpp:624-656): pattern0_rotated, the
// reference pixels under it, and exact S0 / S00 from which mean0 and C0C0
// follow.
__global__ void k_precompute(GrainsDev g, FrameDev ref) {
  const int gi = blockIdx.x;
  const int b = g.pstart[gi], P = g.pstart[gi + 1] - b;
  double s0r, c0r;
  sincos(g.refrot[gi], &s0r, &c0r);
  const int rx = g.refx[gi], ry = g.refy[gi];
  long long S0 = 0, S00 = 0;
  int oob = 0;
  // four points per thread at a time, so that their pixel loads are in flight
  // together (the integer sums do not depend on the order)
  const int nt = blockDim.x;
  for (int i0 = threadIdx.x; i0 < P; i0 += 4 * nt) {
    unsigned v[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int i = i0 + u * nt;
      v[u] = 0;
      if (i >= P) continue;
      const short2 q = rotate_round(g.pat[b + i], c0r, s0r);
      g.pat0[b + i] = q;
      const int x = rx + q.x, y = ry + q.y;
      if (x < 0 || y < 0 || x >= ref.dimx || y >= ref.dimy) oob = 1;
      else v[u] = ref.pix[(size_t)y * ref.pitch + x];
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int i = i0 + u * nt;
      if (i >= P) continue;
      g.w0[b + i] = (uint16_t)v[u];
      S0 += v[u];
      S00 += (long long)v[u] * v[u];
    }
  }
  __shared__ long long red[2][32];
  __shared__ int s_oob;
  if (threadIdx.x == 0) s_oob = 0;
  __syncthreads();
  if (oob) atomicOr(&s_oob, 1);
  S0 = warp_sum_ll(S0);
  S00 = warp_sum_ll(S00);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) {
    red[0][w] = S0;
    red[1][w] = S00;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    long long a = 0, c = 0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
      a += red[0][k];
      c += red[1][k];
    }
    g.s0[gi] = a;
    g.s00[gi] = c;
    g.mean0[gi] = (double)a / (double)P;
    g.c0c0[gi] = (double)((long long)P * c - a * a) / (double)P;
    if (s_oob || P <= 0) g.flags[gi] |= 2;
    else g.flags[gi] &= ~2;
  }
}

// reset() + backup() of every grain at the start of the pixel stage
// (src/p-tracker.cpp:478-479) and zeroing of the list counters.
__global__ void k_stage_begin(GrainsDev g, int* counts) {
  const int gi = blockIdx.x * blockDim.x + threadIdx.x;
  if (gi == 0) {
    counts[1] = 0;
    counts[2] = 0;
    counts[4] = counts[5] = counts[6] = 0;  // exact re-search lists of BF16 levels
  }
  if (gi >= g.n) return;
  g.ncc[gi] = 0.0;
  g.ncc_rescue[gi] = 0.0;
  g.ncc_subpix[gi] = 0.0;
  g.dx_prev[gi] = g.dx[gi];
  g.dy_prev[gi] = g.dy[gi];
  g.drot_prev[gi] = g.drot[gi];
  const int f = g.flags[gi] & 2;
  g.flags[gi] = f;
  g.status[gi] = (g.masked[gi] ? PTK_ST_MASKED : 0) | (f ? PTK_ST_OUT_OF_BOUNDS : 0);
}

// ---------------------------------------------------------------------------
// Shared-memory layout of one search CTA (dynamic):
//   int      off[max_points]   patch offset of each rotated pattern point
//   uint16_t w[max_points]     reference pixel of each point (I0)
//   uint16_t patch[...]        current-frame patch, row-major, width PW
size_t search_smem_bytes(int max_points, int max_patch_elems) {
  size_t b = (size_t)max_points * 4 + (size_t)max_points * 2;
  b = (b + 15) & ~(size_t)15;
  return b + (size_t)max_patch_elems * 2 + 16;
}

struct Cand {
  double ncc;
  int idx;
};

// Reference order: a later candidate replaces the running best only if its
// NCC is strictly larger, so among equal values the smallest index wins; NaN
// and values <= 0 never win (best_NCC starts at 0.0).
__device__ __forceinline__ bool better(double ncc, int idx, double bn, int bi) {
  return ncc > 0.0 && (ncc > bn || (ncc == bn && idx < bi));
}

__global__ void __launch_bounds__(kSearchThreads) k_search(SearchLaunch p) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_item;
  __shared__ int s_bbox[4];
  __shared__ double s_rn[kSearchThreads / 32];
  __shared__ int s_ri[kSearchThreads / 32];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int count = *p.list_count;
  const int per_grain = p.nrot * p.tiles_u * p.tiles_v;
  long long total = (long long)count * per_grain;
  if (total > p.max_items) total = p.max_items;
  const int NU = p.left + p.right + 1, NV = p.up + p.down + 1;

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
    const GrainsDev& g = p.g;

    const int b = g.pstart[gi], P = g.pstart[gi + 1] - b;
    const bool skip = g.masked[gi] || (g.flags[gi] & 2) || P <= 0 || P > kMaxPatternPoints;
    if (skip) {
      if (tid == 0) p.best[item] = SearchBest{0.0, INT_MAX, 0};
      __syncthreads();
      continue;
    }
    int* s_off = reinterpret_cast<int*>(smem);
    uint16_t* s_w = reinterpret_cast<uint16_t*>(smem + (size_t)P * 4);
    // patch follows the two per-point arrays (sized for this grain's P)
    size_t pofs = ((size_t)P * 6 + 15) & ~(size_t)15;
    uint16_t* s_patch = reinterpret_cast<uint16_t*>(smem + pofs);

    // total_rot = refrot + drot + step (src/p-tracker.cpp:687)
    const double total_rot = (g.refrot[gi] + g.drot[gi]) + p.steps[r];
    double s1, c1;
    sincos(total_rot, &s1, &c1);
    const int gdx = (int)round(g.dx[gi]);
    const int gdy = (int)round(g.dy[gi]);

    if (tid == 0) {
      s_bbox[0] = INT_MAX;
      s_bbox[1] = INT_MIN;
      s_bbox[2] = INT_MAX;
      s_bbox[3] = INT_MIN;
    }
    __syncthreads();
    int xmn = INT_MAX, xmx = INT_MIN, ymn = INT_MAX, ymx = INT_MIN;
    for (int i = tid; i < P; i += kSearchThreads) {
      const short2 q = rotate_round(g.pat[b + i], c1, s1);
      s_off[i] = ((int)q.y << 16) | ((int)q.x & 0xffff);  // packed, decoded below
      s_w[i] = g.w0[b + i];
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

    // candidates of this tile
    const int u0 = -p.left + tu * kTileU, u1 = min(u0 + kTileU - 1, p.right);
    const int v0 = -p.up + tv * kTileV, v1 = min(v0 + kTileV - 1, p.down);
    const int X0 = g.refx[gi] + gdx + bx0 + u0;
    const int Y0 = g.refy[gi] + gdy + by0 + v0;
    const int PW = (bx1 - bx0) + (u1 - u0) + 1;
    const int PH = (by1 - by0) + (v1 - v0) + 1;
    const bool oob = X0 < 0 || Y0 < 0 || X0 + PW > p.cur.dimx || Y0 + PH > p.cur.dimy;
    if (oob) {
      if (tid == 0) {
        atomicOr(&g.flags[gi], 1);
        p.best[item] = SearchBest{0.0, INT_MAX, 0};
      }
      __syncthreads();
      continue;
    }
    // stage the patch (rows of PW pixels) and turn points into patch offsets
    for (int e = tid; e < PW * PH; e += kSearchThreads) {
      const int yy = e / PW, xx = e - yy * PW;
      s_patch[e] = p.cur.pix[(size_t)(Y0 + yy) * p.cur.pitch + (X0 + xx)];
    }
    for (int i = tid; i < P; i += kSearchThreads) {
      const int pk = s_off[i];
      const int qx = (int)(short)(pk & 0xffff), qy = pk >> 16;
      s_off[i] = (qy - by0) * PW + (qx - bx0);
    }
    __syncthreads();

    // each thread: x offset u = u0 + lane, y offsets v0 + warp + 8k
    const int u = u0 + lane;
    int base[4];
    bool valid[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int vl = warp + 8 * k;
      valid[k] = (u <= u1) && (v0 + vl <= v1);
      base[k] = valid[k] ? vl * PW + lane : 0;
    }
    unsigned S1[4] = {0, 0, 0, 0};
    unsigned long long S11[4] = {0, 0, 0, 0}, S01[4] = {0, 0, 0, 0};
#pragma unroll 2
    for (int i = 0; i < P; ++i) {
      const int o = s_off[i];
      const unsigned w = s_w[i];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const unsigned val = s_patch[o + base[k]];
        S1[k] += val;
        S11[k] += (unsigned long long)(val * val);
        S01[k] += (unsigned long long)w * val;
      }
    }
    // NCC per candidate and the thread's best in order
    const long long Pl = P, S0 = g.s0[gi];
    const double den1 = (double)(Pl * g.s00[gi] - S0 * S0);
    double bn = 0.0;
    int bi = INT_MAX;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (!valid[k]) continue;
      const long long num = Pl * (long long)S01[k] - S0 * (long long)S1[k];
      const long long d2 = Pl * (long long)S11[k] - (long long)S1[k] * (long long)S1[k];
      const double ncc = (double)num / sqrt(den1 * (double)d2);
      const int v = v0 + warp + 8 * k;
      const int idx = (r * NU + (u + p.left)) * NV + (v + p.up);
      if (better(ncc, idx, bn, bi)) {
        bn = ncc;
        bi = idx;
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      const double on = __shfl_xor_sync(0xffffffffu, bn, o);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (better(on, oi, bn, bi)) {
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
      for (int k = 0; k < kSearchThreads / 32; ++k)
        if (better(s_rn[k], s_ri[k], fn, fi)) {
          fn = s_rn[k];
          fi = s_ri[k];
        }
      p.best[item] = SearchBest{fn, fi, 0};
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Per-grain reduction over its work items and the stage's acceptance rule:
//   level 0 (follow_pattern_pixel, src/p-tracker.cpp:732-742)
//   level 1 (follow_pattern_rescue_pixel, :868-880)
//   level 2 (follow_pattern_super_rescue_pixel, :1005-1015)
__global__ void k_finalize(FinalizeLaunch p) {
  const int li = blockIdx.x * blockDim.x + threadIdx.x;
  if (li >= *p.list_count) return;
  const int gi = p.list[li];
  GrainsDev& g = p.g;
  if (g.masked[gi]) return;
  if ((g.flags[gi] & 7) != 0) {  // footprint leaves the frame (or the tile layout): not searched
    g.status[gi] |= PTK_ST_OUT_OF_BOUNDS;
    return;
  }
  const int per_grain = p.nrot * p.tiles;
  double bn = 0.0;
  int bi = INT_MAX;
  for (int k = 0; k < per_grain; ++k) {
    const SearchBest sb = p.best[(size_t)li * per_grain + k];
    if (better(sb.ncc, sb.idx, bn, bi)) {
      bn = sb.ncc;
      bi = sb.idx;
    }
  }
  // decode idx = (r * NU + (u + left)) * NV + (v + up)
  int bu = 0, bv = 0;
  double bdrot = 0.0;
  if (bi != INT_MAX) {
    const int ru = bi / p.nv;
    const int r = ru / p.nu;
    bv = (bi - ru * p.nv) - p.up;
    bu = (ru - r * p.nu) - p.left;
    bdrot = p.steps[r];
  }
  const int gdx = (int)round(g.dx[gi]);
  const int gdy = (int)round(g.dy[gi]);
  bool accept;
  if (p.level == 0) {
    g.upix[gi] = 0.0;
    g.vpix[gi] = 0.0;
    g.rot_inc[gi] = 0.0;
    g.ncc[gi] = bn;
    g.ncc_rescue[gi] = bn;
    accept = !(bn < p.NCC_min);
  } else if (p.level == 1) {
    g.ncc_rescue[gi] = bn;
    accept = !(bn < p.NCC_min_super);
  } else {
    g.ncc_rescue[gi] = bn;
    accept = bn > p.NCC_min_super;
  }
  if (!accept && p.redo) {  // decided by the exact re-search of this level
    p.out_list[atomicAdd(p.out_count, 1)] = gi;
    return;
  }
  if (p.level == 0) {
    if (!accept) {
      p.out_list[atomicAdd(p.out_count, 1)] = gi;
      g.status[gi] |= PTK_ST_RESCUED;
    }
  } else if (p.level == 1) {
    if (!accept) {
      p.out_list[atomicAdd(p.out_count, 1)] = gi;
      g.status[gi] |= PTK_ST_SUPER_RESCUED | PTK_ST_FAILED;
    }
  } else if (accept) {
    g.status[gi] &= (uint8_t)~PTK_ST_FAILED;
  }
  if (accept) {
    const double rest_dx = g.dx[gi] - gdx;
    const double rest_dy = g.dy[gi] - gdy;
    g.upix[gi] = (double)bu - rest_dx;
    g.vpix[gi] = (double)bv - rest_dy;
    g.rot_inc[gi] = bdrot;
    g.dx[gi] = (double)(gdx + bu);
    g.dy[gi] = (double)(gdy + bv);
    g.drot[gi] += bdrot;
  }
}

// Increments of the frame and, when requested, the reference change
// (src/p-tracker.cpp:577-611).
__global__ void k_end_frame(GrainsDev g, int swap_reference) {
  const int gi = blockIdx.x * blockDim.x + threadIdx.x;
  if (gi >= g.n) return;
  g.upix[gi] = g.dx[gi] - g.dx_prev[gi];
  g.vpix[gi] = g.dy[gi] - g.dy_prev[gi];
  g.rot_inc[gi] = g.drot[gi] - g.drot_prev[gi];
  if (swap_reference) {
    double actual = (double)g.refx[gi] + g.dx[gi];
    g.refx[gi] = (int)round(actual);
    g.dx[gi] = actual - (double)g.refx[gi];
    actual = (double)g.refy[gi] + g.dy[gi];
    g.refy[gi] = (int)round(actual);
    g.dy[gi] = actual - (double)g.refy[gi];
    g.refrot[gi] += g.drot[gi];
    g.drot[gi] = 0.0;
  }
}

// Widening of 8-bit frames to the 16-bit device layout (values unchanged).
__global__ void k_widen_u8(const uint8_t* src, size_t src_pitch, uint16_t* dst, int dst_pitch, int dimx, int dimy) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x < dimx && y < dimy) dst[(size_t)y * dst_pitch + x] = src[(size_t)y * src_pitch + x];
}

// ---------------------------------------------------------------------------
void launch_precompute(const GrainsDev& g, const FrameDev& ref, cudaStream_t s) {
  if (g.n > 0) k_precompute<<<g.n, 256, 0, s>>>(g, ref);
}

void launch_stage_begin(const GrainsDev& g, int* counts, cudaStream_t s) {
  const int n = g.n > 0 ? g.n : 1;
  k_stage_begin<<<(n + 255) / 256, 256, 0, s>>>(g, counts);
}

static void search_attr(size_t smem) { ensure_smem((const void*)k_search, smem); }

void launch_search(const SearchLaunch& p, int grid, size_t smem, cudaStream_t s) {
  search_attr(smem);
  k_search<<<grid, kSearchThreads, smem, s>>>(p);
}

int search_occupancy(size_t smem) {
  search_attr(smem);
  int blocks = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_search, kSearchThreads, smem);
  return blocks;
}

void launch_finalize(const FinalizeLaunch& p, int n_grains, cudaStream_t s) {
  const int n = n_grains > 0 ? n_grains : 1;
  k_finalize<<<(n + 127) / 128, 128, 0, s>>>(p);
}

void launch_end_frame(const GrainsDev& g, int swap_reference, cudaStream_t s) {
  const int n = g.n > 0 ? g.n : 1;
  k_end_frame<<<(n + 255) / 256, 256, 0, s>>>(g, swap_reference);
}

void launch_widen_u8(const uint8_t* src, size_t src_pitch, uint16_t* dst, int dst_pitch, int dimx, int dimy,
                     cudaStream_t s) {
  dim3 grid((dimx + 255) / 256, dimy);
  k_widen_u8<<<grid, 256, 0, s>>>(src, src_pitch, dst, dst_pitch, dimx, dimy);
}

}  // namespace ptk
