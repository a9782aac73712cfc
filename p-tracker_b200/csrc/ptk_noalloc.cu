// Pixel-stage search for callers that cannot allocate device memory.
//
// Some callers of this library cannot call cudaMalloc: a plug-in living inside
// a host application whose own allocator owns every byte of device memory, or
// a capture or real-time loop where an allocation (which may synchronise the
// device) is not allowed.  ptk_search_pixel_noalloc serves them: it runs the
// same exact integer-pixel + rotation-step NCC search as ptk_search(level 0)
// on buffers the caller already owns, and keeps its own scratch (work-queue
// head, rotation steps, per-work-item bests) in one file-scope device array of
// fixed size, kScratchBytes.  Every GPU that loads the library holds that
// array until the process exits.
//
// The array is shared by all calls on a device and keeps the previous call's
// contents; the work-queue head is cleared at the start of every call.  Calls
// whose work overlaps on the GPU (for instance on two streams) race on the
// array and give wrong results: serialise them.
//
// Host code must not pass the array's name to a kernel: on the host it is a
// stand-in symbol, not a device address.  The first call on each device, with
// that device current, looks the address up with cudaGetSymbolAddress and
// caches it; make that first call before any stream capture on that device.
#include <climits>
#include <cmath>
#include <mutex>
#include <vector>

#include "ptk_internal.cuh"

namespace ptk {
namespace {

// 4 MiB: 256 B queue head, 32 KiB of rotation steps (4096 doubles), and
// (4 MiB - 33024 B) / 16 B = 260,080 per-work-item records.
constexpr size_t kScratchBytes = 4u << 20;
constexpr size_t kStepsOffset = 256;
constexpr int kMaxSteps = 4096;
constexpr size_t kItemsOffset = kStepsOffset + sizeof(double) * kMaxSteps;
constexpr long long kMaxItems = (long long)((kScratchBytes - kItemsOffset) / sizeof(SearchBest));

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

struct NoallocLaunch {
  const uint16_t* ref;
  const uint16_t* cur;
  int pitch;  // elements
  int dimx, dimy;
  int n;
  const int32_t* refx;
  const int32_t* refy;
  const double* refrot;
  const double* drot;
  const double* dx;
  const double* dy;
  const int32_t* pstart;
  const short2* pat;
  int max_points, span;
  int left, right, up, down, nrot, tiles_u, tiles_v;
  unsigned char* scratch;  // device address of g_noalloc_scratch
};

__device__ __forceinline__ short2 rot_round(short2 p, double c, double s) {
  const double px = (double)p.x, py = (double)p.y;
  const double xr = __dadd_rn(__dmul_rn(c, px), __dmul_rn(s, py));
  const double yr = __dadd_rn(__dmul_rn(-s, px), __dmul_rn(c, py));
  return make_short2((short)round(xr), (short)round(yr));
}

__device__ __forceinline__ bool better_cand(double ncc, int idx, double bn, int bi) {
  return ncc > 0.0 && (ncc > bn || (ncc == bn && idx < bi));
}

// One work item = (grain, rotation step, 32x32 candidate tile), pulled from a
// queue whose head lives in the scratch array.  Unlike the context path, the
// reference side (pattern rotated by refrot, I0, S0, S00) is recomputed per
// item from the reference frame, so no per-grain precompute buffer is needed.
__global__ void __launch_bounds__(kSearchThreads) k_search_noalloc(NoallocLaunch p) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_item, s_bad;
  __shared__ int s_bbox[4];
  __shared__ long long s_red[2][kSearchThreads / 32];
  __shared__ double s_rn[kSearchThreads / 32];
  __shared__ int s_ri[kSearchThreads / 32];
  int* head = reinterpret_cast<int*>(p.scratch);
  const double* steps = reinterpret_cast<const double*>(p.scratch + kStepsOffset);
  SearchBest* best = reinterpret_cast<SearchBest*>(p.scratch + kItemsOffset);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int per_grain = p.nrot * p.tiles_u * p.tiles_v;
  const long long total = (long long)p.n * per_grain;
  const int NU = p.left + p.right + 1, NV = p.up + p.down + 1;
  int* s_off = reinterpret_cast<int*>(smem);
  uint16_t* s_w = reinterpret_cast<uint16_t*>(smem + (size_t)p.max_points * 4);
  uint16_t* s_patch = reinterpret_cast<uint16_t*>(smem + (((size_t)p.max_points * 6 + 15) & ~(size_t)15));
  for (;;) {
    if (tid == 0) s_item = atomicAdd(head, 1);
    __syncthreads();
    const int item = s_item;
    if (item >= total) break;
    const int gi = item / per_grain;
    const int rem = item - gi * per_grain;
    const int r = rem / (p.tiles_u * p.tiles_v);
    const int t = rem - r * (p.tiles_u * p.tiles_v);
    const int tu = t / p.tiles_v, tv = t - tu * p.tiles_v;
    const int b = p.pstart[gi], P = p.pstart[gi + 1] - b;
    if (P <= 0 || P > p.max_points) {
      if (tid == 0) best[item] = SearchBest{0.0, -2, 0};  // -2: pattern outside the stated limits
      __syncthreads();
      continue;
    }
    double sr, cr, s1, c1;
    sincos(p.refrot[gi], &sr, &cr);
    sincos((p.refrot[gi] + p.drot[gi]) + steps[r], &s1, &c1);
    const int gdx = (int)round(p.dx[gi]), gdy = (int)round(p.dy[gi]);
    const int rx = p.refx[gi], ry = p.refy[gi];
    if (tid == 0) {
      s_bbox[0] = INT_MAX;
      s_bbox[1] = INT_MIN;
      s_bbox[2] = INT_MAX;
      s_bbox[3] = INT_MIN;
      s_bad = 0;
    }
    __syncthreads();
    long long S0 = 0, S00 = 0;
    int xmn = INT_MAX, xmx = INT_MIN, ymn = INT_MAX, ymx = INT_MIN, bad = 0;
    const int half = (p.span - kTileU) / 2;
    for (int i = tid; i < P; i += kSearchThreads) {
      const short2 pt = p.pat[b + i];
      const short2 q0 = rot_round(pt, cr, sr);
      const int x0 = rx + q0.x, y0 = ry + q0.y;
      unsigned v0 = 0;
      if (x0 < 0 || y0 < 0 || x0 >= p.dimx || y0 >= p.dimy) bad |= 1;
      else v0 = p.ref[(size_t)y0 * p.pitch + x0];
      s_w[i] = (uint16_t)v0;
      S0 += v0;
      S00 += (long long)v0 * v0;
      const short2 q = rot_round(pt, c1, s1);
      if (q.x < -half || q.x > half || q.y < -half || q.y > half) bad |= 2;  // beyond max_radius: a caller limit
      s_off[i] = ((int)q.y << 16) | ((int)q.x & 0xffff);
      xmn = min(xmn, (int)q.x);
      xmx = max(xmx, (int)q.x);
      ymn = min(ymn, (int)q.y);
      ymx = max(ymx, (int)q.y);
    }
    for (int o = 16; o > 0; o >>= 1) {
      S0 += __shfl_xor_sync(0xffffffffu, S0, o);
      S00 += __shfl_xor_sync(0xffffffffu, S00, o);
      xmn = min(xmn, __shfl_xor_sync(0xffffffffu, xmn, o));
      xmx = max(xmx, __shfl_xor_sync(0xffffffffu, xmx, o));
      ymn = min(ymn, __shfl_xor_sync(0xffffffffu, ymn, o));
      ymx = max(ymx, __shfl_xor_sync(0xffffffffu, ymx, o));
    }
    if (bad) atomicOr(&s_bad, bad);
    if (lane == 0) {
      s_red[0][warp] = S0;
      s_red[1][warp] = S00;
      atomicMin(&s_bbox[0], xmn);
      atomicMax(&s_bbox[1], xmx);
      atomicMin(&s_bbox[2], ymn);
      atomicMax(&s_bbox[3], ymx);
    }
    __syncthreads();
    S0 = 0;
    S00 = 0;
    for (int k = 0; k < kSearchThreads / 32; ++k) {
      S0 += s_red[0][k];
      S00 += s_red[1][k];
    }
    const int bx0 = s_bbox[0], bx1 = s_bbox[1], by0 = s_bbox[2], by1 = s_bbox[3];
    const int u0 = -p.left + tu * kTileU, u1 = min(u0 + kTileU - 1, p.right);
    const int v0 = -p.up + tv * kTileV, v1 = min(v0 + kTileV - 1, p.down);
    const int X0 = rx + gdx + bx0 + u0, Y0 = ry + gdy + by0 + v0;
    const int PW = (bx1 - bx0) + (u1 - u0) + 1, PH = (by1 - by0) + (v1 - v0) + 1;
    if (s_bad & 2) {
      if (tid == 0) best[item] = SearchBest{0.0, -2, 0};  // -2: a rotated offset exceeds max_radius
      __syncthreads();
      continue;
    }
    const bool oob = s_bad || X0 < 0 || Y0 < 0 || X0 + PW > p.dimx || Y0 + PH > p.dimy;
    if (oob) {
      if (tid == 0) best[item] = SearchBest{0.0, -1, 0};  // -1: footprint leaves the frame
      __syncthreads();
      continue;
    }
    for (int e = tid; e < PW * PH; e += kSearchThreads) {
      const int yy = e / PW, xx = e - yy * PW;
      s_patch[e] = p.cur[(size_t)(Y0 + yy) * p.pitch + (X0 + xx)];
    }
    for (int i = tid; i < P; i += kSearchThreads) {
      const int pk = s_off[i];
      const int qx = (int)(short)(pk & 0xffff), qy = pk >> 16;
      s_off[i] = (qy - by0) * PW + (qx - bx0);
    }
    __syncthreads();
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
    const long long Pl = P;
    const double den1 = (double)(Pl * S00 - S0 * S0);
    double bn = 0.0;
    int bi = INT_MAX;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (!valid[k]) continue;
      const long long num = Pl * (long long)S01[k] - S0 * (long long)S1[k];
      const long long d2 = Pl * (long long)S11[k] - (long long)S1[k] * (long long)S1[k];
      const double ncc = (double)num / sqrt(den1 * (double)d2);
      const int idx = (r * NU + (u + p.left)) * NV + (v0 + warp + 8 * k + p.up);
      if (better_cand(ncc, idx, bn, bi)) {
        bn = ncc;
        bi = idx;
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      const double on = __shfl_xor_sync(0xffffffffu, bn, o);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (better_cand(on, oi, bn, bi)) {
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
        if (better_cand(s_rn[k], s_ri[k], fn, fi)) {
          fn = s_rn[k];
          fi = s_ri[k];
        }
      best[item] = SearchBest{fn, fi, 0};
    }
    __syncthreads();
  }
}

// The rotation-step list, produced by the reference's own double loop
// (src/p-tracker.cpp:684-686); IEEE additions give the host's values bit for bit.
__global__ void k_steps_noalloc(double inc, int num, int nrot, unsigned char* scratch) {
  double* steps = reinterpret_cast<double*>(scratch + kStepsOffset);
  const double rotmax = fabs(inc * num);
  int k = 0;
  for (double d = -rotmax; d <= rotmax && k < nrot; d += inc) steps[k++] = d;
}

// Per grain, in the reference's iteration order (first strict maximum above
// 0 wins, src/p-tracker.cpp:718-723).
__global__ void k_finalize_noalloc(NoallocLaunch p, double* best_ncc, int32_t* best_u, int32_t* best_v,
                                   double* best_drot) {
  const int gi = blockIdx.x * blockDim.x + threadIdx.x;
  if (gi >= p.n) return;
  const double* steps = reinterpret_cast<const double*>(p.scratch + kStepsOffset);
  const SearchBest* best = reinterpret_cast<const SearchBest*>(p.scratch + kItemsOffset);
  const int per_grain = p.nrot * p.tiles_u * p.tiles_v;
  double bn = 0.0;
  int bi = INT_MAX;
  int err = 0;
  for (int k = 0; k < per_grain; ++k) {
    const SearchBest sb = best[(size_t)gi * per_grain + k];
    if (sb.idx < 0) err = (err == -2 || sb.idx == -2) ? -2 : -1;  // a caller-limit error outranks the frame edge
    else if (better_cand(sb.ncc, sb.idx, bn, bi)) {
      bn = sb.ncc;
      bi = sb.idx;
    }
  }
  if (err) {
    best_ncc[gi] = __longlong_as_double(0x7ff8000000000000ll);
    best_u[gi] = err == -1 ? INT_MIN : INT_MIN + 1;
    best_v[gi] = best_u[gi];
    best_drot[gi] = 0.0;
    return;
  }
  int u = 0, v = 0;
  double dr = 0.0;
  if (bi != INT_MAX) {
    const int NU = p.left + p.right + 1, NV = p.up + p.down + 1;
    const int ru = bi / NV;
    const int r = ru / NU;
    v = (bi - ru * NV) - p.up;
    u = (ru - r * NU) - p.left;
    dr = steps[r];
  }
  best_ncc[gi] = bn;
  best_u[gi] = u;
  best_v[gi] = v;
  best_drot[gi] = dr;
}

// Device address of the scratch array, looked up once per device, and the
// dynamic shared memory the search kernel has been enabled for there.
std::mutex g_mutex;
constexpr int kMaxDevices = 64;
unsigned char* g_addr[kMaxDevices] = {};
size_t g_smem[kMaxDevices] = {};

}  // namespace
}  // namespace ptk

using namespace ptk;

extern "C" int ptk_search_pixel_noalloc(const uint16_t* ref_pix, const uint16_t* cur_pix, size_t pitch_bytes,
                                        int dimx, int dimy, int n_grains, const int32_t* refx,
                                        const int32_t* refy, const double* refrot, const double* drot,
                                        const double* dx, const double* dy, const int32_t* pattern_starts,
                                        const int16_t* pattern_xy, int max_points, int max_radius,
                                        const ptk_zone* zone, int rotations, double* best_ncc, int32_t* best_u,
                                        int32_t* best_v, double* best_drot, void* stream) {
  if (!ref_pix || !cur_pix || !refx || !refy || !refrot || !drot || !dx || !dy || !pattern_starts || !pattern_xy ||
      !zone || !best_ncc || !best_u || !best_v || !best_drot || n_grains < 0 || dimx < 4 || dimy < 4 ||
      pitch_bytes < (size_t)dimx * 2 || pitch_bytes % 2 != 0)
    return PTK_ERR_ARG;
  if (zone->left < 0 || zone->right < 0 || zone->up < 0 || zone->down < 0) return PTK_ERR_ARG;
  if (max_points < 1 || max_points > kMaxPatternPoints || max_radius < 0 || max_radius > 4096) return PTK_ERR_LIMIT;
  if (n_grains == 0) return PTK_OK;
  // rotation steps exactly as the reference's loop (src/p-tracker.cpp:684-686)
  double inc = zone->inc_rot;
  int num = zone->num_rot;
  if (rotations == 0) {
    inc = 1.0;
    num = 0;
  }
  if (!(inc > 0.0)) return PTK_ERR_ARG;
  int nrot = 0;
  const double rotmax = std::fabs(inc * num);
  for (double d = -rotmax; d <= rotmax; d += inc) {
    if (nrot == kMaxSteps) return PTK_ERR_LIMIT;
    ++nrot;
  }
  const int nu = zone->left + zone->right + 1, nv = zone->up + zone->down + 1;
  const int tiles_u = (nu + kTileU - 1) / kTileU, tiles_v = (nv + kTileV - 1) / kTileV;
  const long long items = (long long)n_grains * nrot * tiles_u * tiles_v;
  if (items > kMaxItems) return PTK_ERR_LIMIT;  // more work items than the fixed scratch holds
  const int span = 2 * (max_radius + 1) + kTileU;
  const size_t smem = (((size_t)max_points * 6 + 15) & ~(size_t)15) + (size_t)span * span * 2 + 16;
  if (smem > 226 * 1024) return PTK_ERR_LIMIT;  // leaves room for the kernel's static shared memory

  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return PTK_ERR_CUDA;
  unsigned char* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_addr[dev]) {
      void* ptr = nullptr;
      if (cudaGetSymbolAddress(&ptr, g_noalloc_scratch) != cudaSuccess || !ptr) return PTK_ERR_CUDA;
      g_addr[dev] = static_cast<unsigned char*>(ptr);
    }
    if (smem > g_smem[dev]) {
      if (cudaFuncSetAttribute(k_search_noalloc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
          cudaSuccess)
        return PTK_ERR_CUDA;
      g_smem[dev] = smem;
    }
    scratch = g_addr[dev];
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // Every enqueue below reports its own status (cudaLaunchKernel, not the
  // triple-chevron launch followed by cudaGetLastError), so an error left
  // pending by the caller's earlier work is neither reported as this call's
  // failure nor cleared.
  // the queue head must start at zero; the step list is rebuilt on the device
  if (cudaMemsetAsync(scratch, 0, sizeof(int), s) != cudaSuccess) return PTK_ERR_CUDA;
  {
    void* args[] = {&inc, &num, &nrot, &scratch};
    if (cudaLaunchKernel((const void*)k_steps_noalloc, dim3(1), dim3(1), args, 0, s) != cudaSuccess)
      return PTK_ERR_CUDA;
  }
  NoallocLaunch p;
  p.ref = ref_pix;
  p.cur = cur_pix;
  p.pitch = (int)(pitch_bytes / 2);
  p.dimx = dimx;
  p.dimy = dimy;
  p.n = n_grains;
  p.refx = refx;
  p.refy = refy;
  p.refrot = refrot;
  p.drot = drot;
  p.dx = dx;
  p.dy = dy;
  p.pstart = pattern_starts;
  p.pat = reinterpret_cast<const short2*>(pattern_xy);
  p.max_points = max_points;
  p.span = span;
  p.left = zone->left;
  p.right = zone->right;
  p.up = zone->up;
  p.down = zone->down;
  p.nrot = nrot;
  p.tiles_u = tiles_u;
  p.tiles_v = tiles_v;
  p.scratch = scratch;
  int sms = 148, occ = 1;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_search_noalloc, kSearchThreads, smem);
  {
    void* args[] = {&p};
    if (cudaLaunchKernel((const void*)k_search_noalloc, dim3(sms * (occ > 0 ? occ : 1)), dim3(kSearchThreads), args,
                         smem, s) != cudaSuccess)
      return PTK_ERR_CUDA;
  }
  {
    void* args[] = {&p, &best_ncc, &best_u, &best_v, &best_drot};
    if (cudaLaunchKernel((const void*)k_finalize_noalloc, dim3((n_grains + 127) / 128), dim3(128), args, 0, s) !=
        cudaSuccess)
      return PTK_ERR_CUDA;
  }
  return PTK_OK;
}
