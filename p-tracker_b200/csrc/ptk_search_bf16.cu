// BF16 tensor-core integer-pixel + rotation-step search (the precision form)
// on sm_100a.
//
// Same result contract as the exact search (src/p-tracker.cpp:659-1016): the
// grain moves to the first strict NCC maximum above 0 over (rotation step,
// x offset, y offset), ranked on exact integer sums.  The tensor cores only
// decide WHERE to look; every value that reaches the acceptance rule is exact.
//
//  1. k_weights_bf16: per grain and rotation step r, the pattern rotated as
//     the exact search rotates it (rotate_pixel_pattern), scattered into two
//     maps over the footprint: W_r, the centred reference values
//     I0_i - mean0 (coinciding points add up), and M_r, the multiplicity of
//     each footprint pixel.  Both are stored in BF16 (M_r exactly).
//  2. k_search_bf16 (tcgen05): for every rotation step r and candidate
//     c = (u, v) of a 32 x 32 tile, two correlations with the current frame I1,
//         D_r(c) = sum_x W_r(x) I1(x + c)              (the NCC's cross term)
//         S_r(c) = sum_x M_r(x) (I1(x + c) - m)^2      (m = rint(mean0))
//     in BF16 with FP32 accumulation in tensor memory, and per candidate the
//     ranking score max_r D_r / sqrt(S_r).  Because the window's variance
//     under the rotated footprint is S_r minus a non-negative mean term,
//     D_r / sqrt(S_r) is a lower bound of NCC_r * sqrt(C0C0) that no footprint
//     difference between rotation steps can inflate, and it is tight when the
//     window's mean is close to the reference pattern's.  The best candidates
//     of each tile (within a few percent of its best score) are written out.
//  3. k_rescore_bf16 (CUDA cores, exact integers): every rotation step at each
//     kept candidate, with the exact search's sums and NCC expression, giving
//     per-candidate best records in the reference's order; the level's usual
//     finalize applies the acceptance rule to them.
//
// Tensor-core formulation of step 2 (one work item = one 32 x 32 candidate
// tile of one grain, persistent CTAs, one per SM, 512 threads):
//   * A operands (M = 128 = 4 x-shifts j by 32 rotation slots r, K = 16
//     footprint columns): W_r and M_r, stored in the grain's scratch slot as
//     [footprint row][8-column block][rotation][8 values] (512 bytes per row
//     block).  In shared memory each row has 3 zero blocks in front, so row
//     m = 32 j + r of a core-matrix group reads block (a + j): consecutive
//     8-row groups are 128 bytes apart (SBO) and the two K halves 512 bytes
//     apart (LBO), i.e. the x-shift by 8 j columns costs nothing but the
//     descriptor.  Rows are brought in with bulk async copies (cp.async.bulk,
//     no multicast), one per footprint row and operand: the rotation slots
//     beyond the level's steps come along and feed accumulator lanes that
//     are never read.
//   * B operands (N = 256 = 32 y offsets by 8 x offsets, K = 16 image
//     columns): the current frame minus m, and its square, in a Hankel
//     layout - per image row and 8-column block, 8 entries of 16 bytes, entry
//     s holding the 8 pixels that start s columns into the block - so the 8 x
//     offsets of a core matrix are 16 bytes apart, K halves 128 bytes apart
//     (LBO) and y offsets one image row apart (SBO).
//   * For footprint row y and chunk c, D[32 j + r][8 v + s] accumulates
//     W_r(y, f) * I(y + v, f + 24 - 8 j + s): candidate x offset 24 - 8 j + s
//     (S likewise with M_r and the squares).  Two MMAs (M=128, N=256, K=16)
//     cover the whole 32 x 32 x 32 tile for one row and chunk; a grain's tile
//     takes 2 MMAs per footprint row and chunk touching a block that holds a
//     point of some rotation step (the weights kernel records each row's
//     first and last such block), issued by one thread per strip of rows and
//     committed to an mbarrier.  D occupies tensor-memory
//     columns 0..255, S columns 256..511.
//   * The epilogue reads both accumulators with tcgen05.ld (warp w: lanes
//     32 (w % 4).., columns 64 (w / 4)..), divides per rotation lane, takes
//     the maximum over rotation lanes per candidate with a warp max-reduction
//     and keeps the best candidates.
//
// Pattern rotation (all kernels) is rotate_pixel_pattern's
// (src/p-tracker.cpp:615-621) result bit for bit: an FP32 estimate decides the
// rounding, and the FP64 expression is evaluated whenever the estimate lies
// within 1e-3 of a half-integer (the estimate's error is below 2e-5 for the
// offsets allowed here).
//
// Limits (else the exact kernels run): pattern extent within +-47 px
// (footprint side <= 95), at most 32 rotation steps, no offset repeated more
// than 63 times within a pattern.

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include <climits>
#include <mutex>

#include "ptk_internal.cuh"

namespace ptk {

namespace {

constexpr int kThreads = 512;     // 16 warps
constexpr int kWarps = kThreads / 32;
constexpr int kNRot = 32;         // rotation slots of the A operands
constexpr int kMaxFoot = 96;      // footprint side limit (2 * half + 1 < 96)
constexpr int kTmemCols = 512;    // D in columns 0..255, S in 256..511 (128 lanes x FP32)
constexpr int kSmemBudget = 224 * 1024;  // one CTA per SM
// Kept candidates: the tile's best score and those within kKeepRel of it (up
// to `keep`).  Over 959 grains of the 50-frame 5616x3744 sequence (small
// grains with edge-dominated patterns, accumulated reference rotations) the
// exact best lay at most 1.9 % below the tile's best score.  The bound is
// looser for mediocre matches (the window's mean further from the pattern's),
// so tiles whose best score, as an NCC lower bound, is below kGoodMatch keep
// candidates within kKeepRelWeak.
constexpr float kKeepRel = 0.03f;
constexpr float kKeepRelWeak = 0.10f;
constexpr float kGoodMatch = 0.9f;
constexpr long kWaitLimit = 1L << 22;
constexpr int kStageBoxRows = 8;  // image rows per TMA box of the strip staging
// after an error: the waits for the CTA's own copies and MMAs still in flight
// (they complete unless the device is broken) get a longer bound
constexpr long kDrainLimit = 1L << 26;
// operand rows in flight: W_r and M_r of one footprint row per ring buffer
constexpr int kRing = 8;       // barrier slots
constexpr int kRingUsed = 4;   // buffers
// weights kernel: 512 threads, 108 KB of 32-bit maps (two blocks per SM, as
// its registers allow)
constexpr int kWThreads = 512;
constexpr int kWSmem = 108 * 1024;

// A and B operand formats: BF16 x BF16 -> FP32, both K-major, M = 128, N = 256.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(256 >> 3) << 17) |
                            ((uint32_t)(128 >> 4) << 24);

struct Geom {
  int half;  // footprint covers offsets [-half, half] in x and y
  int fw;    // footprint side
  int nbf;   // 8-column blocks of the footprint
  int nch;   // 16-column MMA chunks (footprint + 24 columns of shift)
  int wb;    // weight blocks per row in shared memory (3 leading zero blocks)
  int hb;    // Hankel blocks per image row
  int rp;    // bytes per staged image row (8 hb + 16 pixels from a 16-byte boundary: one TMA box row)
  int rs;    // footprint rows per strip (Hankel rows filled at once, plus 31)
  int nb;    // operand-row ring buffers
};

__host__ __device__ inline Geom geom_of(int half, int nb = kRingUsed) {
  Geom g;
  g.half = half;
  g.fw = 2 * half + 1;
  g.nbf = (g.fw + 7) / 8;
  g.nch = (g.nbf + 3 + 1) / 2;
  g.wb = 2 * g.nch + 3;
  g.hb = 2 * g.nch;
  g.rp = 16 * g.hb + 32;
  // the operand-row ring, then two Hankel buffers and the staged image rows
  // with 31 rows of halo (staged in boxes of 8 rows: up to 7 more)
  const int halo_row = 2 * g.hb * 128 + g.rp;
  int rs = (kSmemBudget - nb * 2 * g.wb * 512 - (kStageBoxRows - 1) * g.rp) / halo_row - 31;
  if (rs > g.fw) rs = g.fw;
  g.rs = rs < 1 ? 1 : rs;
  g.nb = nb;
  return g;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// tcgen05 shared-memory matrix descriptor: K-major, no swizzle, version 1.
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((saddr & 0x3FFFFu) >> 4);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

__device__ __forceinline__ void mma_bf16(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(dtmem),
      "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}

// Bounded wait on an mbarrier phase; false when the limit ran out.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, long limit = kWaitLimit) {
  uint32_t done = 0;
  for (long it = 0; it < limit && !done; ++it) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
  }
  return done != 0;
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
}

// One box of a 5-D tensor map global -> shared (TMA, tiled, no multicast):
// coordinates innermost first; elements outside the tensor are filled with
// zeros and count toward the transaction bytes.
__device__ __forceinline__ void tma_load_5d(uint32_t dst, const CUtensorMap* tmap, int c0, int c1, int c2, int c3,
                                            int c4, uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, "
      "%6}], [%7];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(tmap)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(mbar)
      : "memory");
}

// One box of a 2-D tensor map global -> shared (TMA, tiled, no multicast);
// x must be a multiple of 8 pixels (16 bytes); rows or columns outside the
// frame come back as zeros.
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* tmap, int x, int y, uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
          "r"(dst),
      "l"(reinterpret_cast<uint64_t>(tmap)), "r"(x), "r"(y), "r"(mbar)
      : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
        "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
        "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ uint32_t tmem_ld1(uint32_t taddr) {
  uint32_t v;
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];" : "=r"(v) : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
  return v;
}

// rotate_pixel_pattern (src/p-tracker.cpp:615-621): FP64 without contraction,
// round half away from zero - identical to the exact search's rotation.
__device__ __forceinline__ short2 rotate_round_b(short2 p, double c, double s) {
  const double px = (double)p.x, py = (double)p.y;
  const double xr = __dadd_rn(__dmul_rn(c, px), __dmul_rn(s, py));
  const double yr = __dadd_rn(__dmul_rn(-s, px), __dmul_rn(c, py));
  return make_short2((short)round(xr), (short)round(yr));
}

// Small integer <-> float without the conversion pipe (|v| < 2^22).
__device__ __forceinline__ float small_i2f(int v) { return __int_as_float(0x4B400000 + v) - 12582912.0f; }

// rotate_round_b's result for |p.x|, |p.y| <= 1024: the FP32 estimate
// (error < 3e-4 at that size) rounds to nearest unless it lies within 1e-3 of
// a half-integer, where the FP64 expression decides.
__device__ __forceinline__ short2 rotate_round_fast(short2 p, float cf, float sf, double c, double s) {
  const float pxf = small_i2f(p.x), pyf = small_i2f(p.y);
  const float xf = fmaf(cf, pxf, sf * pyf);
  const float yf = fmaf(cf, pyf, -(sf * pxf));
  const float mx = xf + 12582912.0f, my = yf + 12582912.0f;  // rint in the low mantissa bits
  const float rx = mx - 12582912.0f, ry = my - 12582912.0f;
  if (fabsf(xf - rx) < 0.499f && fabsf(yf - ry) < 0.499f)
    return make_short2((short)(__float_as_int(mx) - 0x4B400000), (short)(__float_as_int(my) - 0x4B400000));
  return rotate_round_b(p, c, s);
}

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}

// float <-> int keys whose signed order is the float order (finite values)
__device__ __forceinline__ int f2key(float f) {
  const int i = __float_as_int(f);
  return i >= 0 ? i : i ^ 0x7FFFFFFF;
}
__device__ __forceinline__ float key2f(int k) { return __int_as_float(k >= 0 ? k : k ^ 0x7FFFFFFF); }

__device__ __forceinline__ bool better_b(double ncc, int idx, double bn, int bi) {
  return ncc > 0.0 && (ncc > bn || (ncc == bn && idx < bi));
}

}  // namespace

// ---------------------------------------------------------------------------
// 1. BF16 operands of every rotation step of a grain (one block per list
//    entry): the pattern rotated by each step, scattered into one 32-bit map
//    per step holding, per footprint pixel, the sum of the reference values
//    I0 of the points landing there (low 24 bits, exact) and their number
//    (high 8 bits), with integer shared-memory atomics.  Written to the
//    grain's slot as W_r = sum I0 - count * mean0 and M_r = count, each
//    [footprint row][8-column block][rotation][8 values], M after W.  As many
//    rotations per pass as maps fit in shared memory.
__global__ void __launch_bounds__(kWThreads) k_weights_bf16(Bf16Launch p) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ double2 s_cs[kNRot];
  __shared__ float2 s_csf[kNRot];
  const int li = blockIdx.x;
  if (li >= *p.list_count) return;
  const GrainsDev& g = p.g;
  const int gi = p.list[li];
  const int b = g.pstart[gi], P = g.pstart[gi + 1] - b;
  if (g.masked[gi] || (g.flags[gi] & 2) || P <= 0 || P > kMaxPatternPoints) return;
  const Geom G = geom_of(p.half[gi]);
  if (G.fw >= kMaxFoot) return;  // excluded by the host's geometry check
  const int tid = threadIdx.x;
  const int rows = G.fw * G.nbf;
  // [W / M][footprint row][8-column block][live rotation step][8 values]:
  // only the level's nrot steps are stored; the search kernel's tensor map
  // zero-fills the other rotation slots of its A operands
  uint4* slotW = reinterpret_cast<uint4*>(p.wslots) + p.wofs[gi];
  uint4* slotM = slotW + (size_t)rows * p.nrot;
  static_assert((kMaxFoot - 1 + 7) / 8 <= 12, "8-column blocks per footprint row");
  __shared__ unsigned char s_occ[kMaxFoot * 12];  // [row][8-column block]: a point in some rotation step
  for (int e = tid; e < rows; e += kWThreads) s_occ[e] = 0;
  const double base_rot = g.refrot[gi] + g.drot[gi];  // total_rot = base_rot + step, as the exact search
  if (tid < p.nrot) {
    double sr, cr;
    sincos(base_rot + p.steps[tid], &sr, &cr);
    s_cs[tid] = make_double2(cr, sr);
    s_csf[tid] = make_float2((float)cr, (float)sr);
    // kept for this level's search and rescore kernels, which rotate by the same steps
    p.rot_cs[(size_t)gi * kNRot + tid] = make_double2(cr, sr);
  }
  const float mean0 = (float)g.mean0[gi];
  // per rotation step a map of fw rows of fwp = 8 nbf words (the columns past
  // fw stay zero), so that a block's 8 words are two 16-byte loads
  const int fwp = 8 * G.nbf, fw2 = G.fw * fwp;
  const int nb_max = max(1, min(p.nrot, kWSmem / (4 * fw2)));
  unsigned* map = reinterpret_cast<unsigned*>(smem);
  for (int r0 = 0; r0 < p.nrot; r0 += nb_max) {
    const int nb = min(nb_max, p.nrot - r0);
    for (int e = tid; e < nb * fw2 / 4; e += kWThreads) reinterpret_cast<uint4*>(map)[e] = make_uint4(0, 0, 0, 0);
    __syncthreads();
    // four points per thread at a time: their loads are in flight together
    for (int i0 = tid; i0 < P; i0 += 4 * kWThreads) {
      short2 q0[4];
      unsigned add[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int i = i0 + u * kWThreads;
        q0[u] = i < P ? g.pat[b + i] : make_short2(0, 0);
        // at most 255 points share a pixel (bf16_supported): the sum stays below 2^24
        add[u] = i < P ? (unsigned)g.w0[b + i] + (1u << 24) : 0u;
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        if (i0 + u * kWThreads >= P) break;
        // rotate_round_fast with the point's conversions hoisted out of the
        // step loop and the map address advanced per step
        const float pxf = small_i2f(q0[u].x), pyf = small_i2f(q0[u].y);
        unsigned* mk = map + G.half * (fwp + 1);  // offset (0, 0) of step r0
#pragma unroll 3
        for (int k = 0; k < nb; ++k, mk += fw2) {
          const float2 cf = s_csf[r0 + k];
          const float xf = fmaf(cf.x, pxf, cf.y * pyf);
          const float yf = fmaf(cf.x, pyf, -(cf.y * pxf));
          const float mx = xf + 12582912.0f, my = yf + 12582912.0f;
          int qx = __float_as_int(mx) - 0x4B400000, qy = __float_as_int(my) - 0x4B400000;
          // the float rounding is the FP64 one unless a coordinate lies within
          // 0.001 of a half-integer (the inputs are finite)
          if (!(fmaxf(fabsf(xf - (mx - 12582912.0f)), fabsf(yf - (my - 12582912.0f))) < 0.499f)) {
            const double2 cd = s_cs[r0 + k];
            const short2 q = rotate_round_b(q0[u], cd.x, cd.y);
            qx = q.x;
            qy = q.y;
          }
          // |q| <= round(|p|) <= ceil(max |offset|) = half - 1 in each
          // coordinate, for every rotation: always inside the footprint
          atomicAdd(mk + qy * fwp + qx, add[u]);
        }
      }
    }
    __syncthreads();
    // thread t converts rotation step k = t % nb of the blocks t / nb, t / nb + per, ...
    // (consecutive threads write consecutive 16-byte rows of the slot)
    const int per = kWThreads / nb;
    if (tid < per * nb) {
      const int k = tid % nb;
      int rem = tid / nb;
      int y = rem / G.nbf, af = rem - y * G.nbf;
      const int dy = per / G.nbf, daf = per - dy * G.nbf;
      const unsigned* mapk = map + k * fw2;
      for (; rem < rows; rem += per) {
        const uint4* src = reinterpret_cast<const uint4*>(mapk + y * fwp + 8 * af);
        const uint4 c0 = src[0], c1 = src[1];
        const unsigned c[8] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w};
        float v[8], m[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const float n = (float)(c[j] >> 24);
          m[j] = n;
          v[j] = (float)(c[j] & 0xFFFFFFu) - n * mean0;
        }
        if ((c[0] | c[1] | c[2] | c[3] | c[4] | c[5] | c[6] | c[7]) >> 24) s_occ[rem] = 1;
        const size_t at = (size_t)rem * p.nrot + r0 + k;
        slotW[at] = make_uint4(pack_bf16x2(v[0], v[1]), pack_bf16x2(v[2], v[3]), pack_bf16x2(v[4], v[5]),
                               pack_bf16x2(v[6], v[7]));
        slotM[at] = make_uint4(pack_bf16x2(m[0], m[1]), pack_bf16x2(m[2], m[3]), pack_bf16x2(m[4], m[5]),
                               pack_bf16x2(m[6], m[7]));
        af += daf;
        y += dy;
        if (af >= G.nbf) {
          af -= G.nbf;
          ++y;
        }
      }
    }
    __syncthreads();
  }
  // per footprint row: the first and last 8-column block holding a point of
  // any rotation step (an empty row: first > last)
  unsigned char* rng = reinterpret_cast<unsigned char*>(slotM + (size_t)rows * p.nrot);
  if (tid < G.fw) {
    int lo = 255, hi = 0;
    for (int a = G.nbf - 1; a >= 0; --a)
      if (s_occ[tid * G.nbf + a]) {
        lo = a;
        hi = max(hi, a);
      }
    rng[2 * tid] = (unsigned char)lo;
    rng[2 * tid + 1] = (unsigned char)hi;
  }
}

// ---------------------------------------------------------------------------
// 2. Tensor-core cross terms and second moments, and the kept candidates of
//    every tile.
// RING: operand-row buffers (a compile-time constant, so the ring indexing
// of the MMA-issuing thread folds; launched for 2, 3, 4 and 6).
template <int RING>
__global__ void __launch_bounds__(kThreads, 1) k_search_bf16(Bf16Launch p) {
  extern __shared__ __align__(128) unsigned char smem_bf[];
  unsigned char* smem = smem_bf;
  __shared__ __align__(8) unsigned long long s_mbar;   // MMA completion
  __shared__ __align__(8) unsigned long long s_full[kRing];  // operand row copied into a ring buffer
  __shared__ __align__(8) unsigned long long s_free[kRing];  // the MMAs reading a ring buffer completed
  __shared__ __align__(8) unsigned long long s_probe;  // failure-path test: nothing ever arrives on it
  __shared__ __align__(8) unsigned long long s_stage;  // a strip's image rows staged (TMA)
  __shared__ int s_stage_out;                          // stagings issued and not yet waited for (0 or 1)
  // operand rows through the ring (thread 0): uses of each buffer copied and
  // consumed so far (a buffer's barriers complete one phase per use)
  __shared__ unsigned s_iss[kRing], s_con[kRing];
  __shared__ uint32_t s_tmem;
  __shared__ int s_li, s_err, s_bb[4];
  __shared__ double2 s_cs[kNRot];
  __shared__ float2 s_csf[kNRot];
  __shared__ float s_cv[kWarps * kBf16KeepMax];
  __shared__ int s_ci[kWarps * kBf16KeepMax];
  __shared__ int s_kept[kBf16KeepMax], s_nkept;  // the tile's kept candidates (packed u, v) and their count
  __shared__ float s_rel;
  __shared__ unsigned char s_rng[2 * kMaxFoot];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t mbar = smem_u32(&s_mbar);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar));
    for (int k = 0; k < kRing; ++k) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s_full[k])));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s_free[k])));
    }
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s_probe)));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s_stage)));
    s_stage_out = 0;
    asm volatile("fence.mbarrier_init.release.cluster;");
    s_err = 0;
    for (int k = 0; k < kRing; ++k) s_iss[k] = s_con[k] = 0u;
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = s_tmem;
  uint32_t parity = 0;  // thread 0: parity of the next MMA-completion phase of s_mbar
  uint32_t sparity = 0;  // thread 0: parity of the next staging phase of s_stage
  if (tid == 0 && (smem_u32(smem_bf) & 127u)) {
    // the operand rows' TMA boxes land on 512-byte multiples from here: the
    // dynamic shared memory must start 128-byte aligned (never seen otherwise)
    s_err = 1;
    atomicOr(p.error, 1);
  }
  if (p.probe_wait > 0 && tid == 0) {
    // Failure-path test: a bounded wait that runs out (no copy or MMA has been
    // issued yet), reported exactly as a real one.
    if (!mbar_wait(smem_u32(&s_probe), 0u, p.probe_wait)) {
      s_err = 1;
      atomicOr(p.error, 1);
    }
  }
  int zhalf = -1;  // footprint geometry whose zero blocks the operand rows hold
  int pf_next = -1;   // thread 0: the next work item, taken before this one's epilogue (-1: none)
  bool pf = false;    // thread 0: its first operand rows and image strip are already on their way

  const GrainsDev& g = p.g;
  const int count = *p.list_count;
  const int tiles = p.tiles_u * p.tiles_v;
  const int keep = p.keep;

  for (;;) {
    __syncthreads();  // every thread is done with the previous grain's shared state
    if (tid == 0) {
      s_li = pf_next >= 0 ? pf_next : atomicAdd(p.work_next, 1);
      pf_next = -1;
      s_bb[0] = s_bb[2] = INT_MAX;
      s_bb[1] = s_bb[3] = INT_MIN;
    }
    __syncthreads();
    // work item = (list entry, tile): the tiles of a large zone (rescues)
    // spread over CTAs instead of running one after another in one
    const int item = s_li;
    const int li = item / tiles, t_item = item - li * tiles;
    if (li >= count || s_err) break;
    const int gi = p.list[li];
    const int b = g.pstart[gi], P = g.pstart[gi + 1] - b;
    int2* topk_g = p.topk + (size_t)li * tiles * kBf16KeepMax;
    if (g.masked[gi] || (g.flags[gi] & 2) || P <= 0 || P > kMaxPatternPoints) {
      if (tid < kBf16KeepMax) topk_g[(size_t)t_item * kBf16KeepMax + tid] = make_int2(INT_MIN, INT_MIN);
      if (tid == 0) p.tile_top[item] = -INFINITY;
      continue;
    }
    // rotation cos/sin (total_rot = base_rot + step, as the exact search) and
    // the grain's footprint geometry
    if (tid < p.nrot) {  // the weights kernel's cos / sin of this grain's steps
      const double2 cs = p.rot_cs[(size_t)gi * kNRot + tid];
      s_cs[tid] = cs;
      s_csf[tid] = make_float2((float)cs.x, (float)cs.y);
    }
    const Geom G = geom_of(p.half[gi], RING);
    const float mean0 = (float)g.mean0[gi];
    const float c00_rsqrt = g.c0c0[gi] > 0.0 ? (float)(1.0 / sqrt(g.c0c0[gi])) : 0.0f;
    const int gdx = (int)round(g.dx[gi]), gdy = (int)round(g.dy[gi]);
    const size_t wrows = (size_t)G.fw * G.nbf * p.nrot;
    const uint4* slotW = reinterpret_cast<const uint4*>(p.wslots) + p.wofs[gi];
    const uint4* slotM = slotW + wrows;
    if (tid < 2 * G.fw) s_rng[tid] = reinterpret_cast<const unsigned char*>(slotM + wrows)[tid];
    const CUtensorMap* tmap = p.tmaps + gi;  // this grain's operand rows, rotation slots zero-filled to 32
    const CUtensorMap* fmap = p.frame_tmaps + (G.hb >> 1);  // the frame's map for this Hankel width
    if (tid == 0) {
      asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(tmap) : "memory");
      asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(fmap) : "memory");
    }
    // ring buffer k: W row at k * 2 wb * 512, M row wb * 512 after it
    const size_t hbytes = (size_t)(G.rs + 31) * G.hb * 128;
    unsigned char* sA = smem;
    unsigned char* sHa = sA + (size_t)G.nb * 2 * G.wb * 512;
    unsigned char* sHs = sHa + hbytes;
    unsigned char* sR = sHs + hbytes;
    const uint32_t abase = smem_u32(sA), habase = smem_u32(sHa), hsbase = smem_u32(sHs);
    const uint32_t rbase = smem_u32(sR);
    // zero blocks of every operand row (3 in front, the rest after the footprint);
    // the copies never write them, so they stay valid while the geometry does
    // (grains come in decreasing pattern size)
    if (G.half != zhalf) {
      for (int e = tid; e < 2 * G.nb * (G.wb - G.nbf) * kNRot; e += kThreads) {
        const int row = e / ((G.wb - G.nbf) * kNRot), rem = e - row * ((G.wb - G.nbf) * kNRot);
        const int zb = rem >> 5, r = rem & 31;
        const int a = zb < 3 ? zb : zb + G.nbf;
        reinterpret_cast<uint4*>(sA)[((size_t)row * G.wb + a) * kNRot + r] = make_uint4(0, 0, 0, 0);
      }
      zhalf = G.half;
    }
    __syncthreads();
    // Bounding box of the rotated patterns: +-(half - 1) bounds it; the exact
    // union over the rotation steps (which decides out-of-frame grains, as in
    // the exact search) is computed only when that bound reaches the edge.
    int bbx0 = 1 - G.half, bbx1 = G.half - 1, bby0 = 1 - G.half, bby1 = G.half - 1;
    bool exact_bb = false;
    const float sub = 8388608.0f + rintf(mean0);  // pixel v -> (2^23 + v) - sub = v - m, exactly

    for (int t = t_item; t <= t_item; ++t) {
      const int tu = t / p.tiles_v, tv = t - tu * p.tiles_v;
      const int u0 = -p.left + tu * kTileU, u1 = min(u0 + kTileU - 1, p.right);
      const int v0 = -p.up + tv * kTileV, v1 = min(v0 + kTileV - 1, p.down);
      int2* topk = topk_g + (size_t)t * kBf16KeepMax;
      {  // the union of the rotated footprints over the tile's candidates must stay in the frame
        const int X = g.refx[gi] + gdx, Y = g.refy[gi] + gdy;
        bool oob = X + bbx0 + u0 < 0 || Y + bby0 + v0 < 0 || X + bbx1 + u1 >= p.cur.dimx ||
                   Y + bby1 + v1 >= p.cur.dimy;
        if (oob && !exact_bb) {
          int xmn = INT_MAX, xmx = INT_MIN, ymn = INT_MAX, ymx = INT_MIN;
          for (int i = tid; i < P; i += kThreads) {
            const short2 q0 = g.pat[b + i];
            for (int r = 0; r < p.nrot; ++r) {
              const short2 q = rotate_round_fast(q0, s_csf[r].x, s_csf[r].y, s_cs[r].x, s_cs[r].y);
              xmn = min(xmn, (int)q.x);
              xmx = max(xmx, (int)q.x);
              ymn = min(ymn, (int)q.y);
              ymx = max(ymx, (int)q.y);
            }
          }
          for (int o = 16; o > 0; o >>= 1) {
            xmn = min(xmn, __shfl_xor_sync(0xffffffffu, xmn, o));
            xmx = max(xmx, __shfl_xor_sync(0xffffffffu, xmx, o));
            ymn = min(ymn, __shfl_xor_sync(0xffffffffu, ymn, o));
            ymx = max(ymx, __shfl_xor_sync(0xffffffffu, ymx, o));
          }
          if (lane == 0) {
            atomicMin(&s_bb[0], xmn);
            atomicMax(&s_bb[1], xmx);
            atomicMin(&s_bb[2], ymn);
            atomicMax(&s_bb[3], ymx);
          }
          __syncthreads();
          bbx0 = s_bb[0];
          bbx1 = s_bb[1];
          bby0 = s_bb[2];
          bby1 = s_bb[3];
          exact_bb = true;
          oob = X + bbx0 + u0 < 0 || Y + bby0 + v0 < 0 || X + bbx1 + u1 >= p.cur.dimx || Y + bby1 + v1 >= p.cur.dimy;
        }
        if (oob) {
          if (tid == 0) {
            atomicOr(&g.flags[gi], 1);
            p.tile_top[(size_t)li * tiles + t] = -INFINITY;
          }
          if (tid < kBf16KeepMax) topk[tid] = make_int2(INT_MIN, INT_MIN);
          continue;
        }
      }
      // image origin of footprint column 0 at candidate (u0, v0)
      const int Xi = g.refx[gi] + gdx - G.half + u0, Yi = g.refy[gi] + gdy - G.half + v0;
      // A strip's image rows (columns Xa .. Xa + 8 hb + 15, rows from Yi + ys)
      // are staged in shared memory by TMA boxes of 8 rows from the frame's
      // tensor map for this Hankel width, issued by thread 0 - for the next
      // strip during the current strip's MMAs.  Rows and columns outside the
      // frame come back as zeros: they only meet candidates outside the zone
      // or footprint pixels whose weights are zero in every rotation step.
      const int nwin = 8 * G.hb;
      const int Xa = Xi & ~7, xoff = Xi - Xa;
      auto stage_rows_at = [&](int xa, int yi, int ys_) {  // thread 0
        const int boxes = (min(G.rs, G.fw - ys_) + 31 + kStageBoxRows - 1) / kStageBoxRows;
        const uint32_t sb = smem_u32(&s_stage);
        mbar_expect_tx(sb, (uint32_t)(boxes * kStageBoxRows * G.rp));
        for (int j = 0; j < boxes; ++j)
          tma_load_2d(rbase + (uint32_t)(j * kStageBoxRows * G.rp), fmap, xa, yi + ys_ + j * kStageBoxRows, sb);
        s_stage_out = 1;
      };
      auto stage_rows = [&](int ys_) { stage_rows_at(Xa, Yi, ys_); };
      auto wait_rows = [&]() {  // thread 0 (a wait that gives up leaves the staging to the drain)
        if (mbar_wait(smem_u32(&s_stage), sparity)) {
          s_stage_out = 0;
          sparity ^= 1u;
        } else {
          s_err = 1;
          atomicOr(p.error, 1);
        }
      };
      // Operand rows stream through the ring (thread 0): row y of the tile goes
      // to buffer y % nb; its copy waits for the MMAs of the row that used the
      // buffer before (nb rows earlier), and is issued nb - 1 rows ahead of its
      // MMAs, so the copies overlap the fills and MMAs.
      const int NB = G.nb;
      auto issue_row_of = [&](const CUtensorMap* tm, int y) -> bool {  // thread 0
        const int k = y % NB;
        const unsigned use = s_iss[k];
        if (use > 0 && !mbar_wait(smem_u32(&s_free[k]), (use - 1) & 1u)) return false;
        const uint32_t full = smem_u32(&s_full[k]);
        mbar_expect_tx(full, (uint32_t)(2 * G.nbf * 512));
        const uint32_t dst = abase + (uint32_t)(k * 2 * G.wb * 512 + 3 * 512);
        // footprint row y of W (coordinate 4 = 0) and of M (1): nbf blocks of
        // 32 rotation slots x 8 values, 512 bytes per block
        tma_load_5d(dst, tm, 0, 0, 0, y, 0, full);
        tma_load_5d(dst + (uint32_t)(G.wb * 512), tm, 0, 0, 0, y, 1, full);
        s_iss[k] = use + 1;
        return true;
      };
      auto issue_row = [&](int y) -> bool { return issue_row_of(tmap, y); };
      if (tid == 0 && !pf) {  // (a prefetched item's first rows and strip were issued during the last epilogue)
        for (int y = 0; y < min(NB - 1, G.fw); ++y)
          if (!issue_row(y)) {
            s_err = 1;
            atomicOr(p.error, 1);
            break;
          }
        if (!s_err) stage_rows(0);
      }
      pf = false;
      uint32_t acc = 0u;  // the tile's first MMA into each accumulator overwrites it
      for (int ys = 0; ys < G.fw; ys += G.rs) {
        const int nr = min(G.rs, G.fw - ys);
        if (tid == 0 && s_stage_out) wait_rows();  // this strip's rows (staged during the previous MMAs)
        __syncthreads();
        if (s_err) break;
        // Hankel image rows ys .. ys + nr + 30 of I - m and of (I - m)^2.
        // Entry (block a, shift s) of a row is the 8-pixel window starting at
        // column x = 8 a + s, stored at byte 16 x: a warp fills one row, 25
        // windows per pass, lane x reading pixel x and taking pixels
        // x + 1 .. x + 7 from the next lanes, so the 16-byte stores of a pass
        // are contiguous.  The pixels come from the staged rows.
        for (int rho = warp; rho < nr + 31; rho += kWarps) {
          const uint16_t* srow = reinterpret_cast<const uint16_t*>(sR + (size_t)rho * G.rp) + xoff;
          unsigned char* drow = sHa + (size_t)rho * G.hb * 128;
          unsigned char* qrow = sHs + (size_t)rho * G.hb * 128;
          for (int x0 = 0; x0 < nwin; x0 += 25) {
            const int x = x0 + lane;
            const float f = x < nwin + 7 ? __int_as_float(0x4B000000 | (int)srow[x]) - sub : 0.0f;
            const float f1 = __shfl_down_sync(0xffffffffu, f, 1);
            const uint32_t p0 = pack_bf16x2(f, f1);
            const uint32_t q0 = pack_bf16x2(f * f, f1 * f1);
            const uint32_t p2 = __shfl_down_sync(0xffffffffu, p0, 2);
            const uint32_t p4 = __shfl_down_sync(0xffffffffu, p0, 4);
            const uint32_t p6 = __shfl_down_sync(0xffffffffu, p0, 6);
            const uint32_t q2 = __shfl_down_sync(0xffffffffu, q0, 2);
            const uint32_t q4 = __shfl_down_sync(0xffffffffu, q0, 4);
            const uint32_t q6 = __shfl_down_sync(0xffffffffu, q0, 6);
            if (lane < 25 && x < nwin) {
              *reinterpret_cast<uint4*>(drow + 16 * x) = make_uint4(p0, p2, p4, p6);
              *reinterpret_cast<uint4*>(qrow + 16 * x) = make_uint4(q0, q2, q4, q6);
            }
          }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        // the staged rows are consumed: bring in the next strip's during these MMAs
        if (tid == 0 && !s_err && ys + G.rs < G.fw) stage_rows(ys + G.rs);
        bool committed = false;  // thread 0: MMAs of this strip committed to s_mbar
        if (tid == 0 && !s_err) {
          for (int yl = 0; yl < nr; ++yl) {
            const int y = ys + yl;
            const int k = y % NB;
            const unsigned use = s_con[k];
            if (!mbar_wait(smem_u32(&s_full[k]), use & 1u)) {
              s_err = 1;
              atomicOr(p.error, 1);
              break;
            }
            s_con[k] = use + 1;
            asm volatile("tcgen05.fence::after_thread_sync;");
            // chunk c reads footprint blocks 2c - 3 .. 2c + 1 (over the 4 x-shifts):
            // the chunks touching the row's occupied blocks [lo, hi]
            const int lo = s_rng[2 * y], hi = s_rng[2 * y + 1];
            const int c1 = min(G.nch - 1, (hi + 3) >> 1);
            const uint32_t wrow = abase + (uint32_t)(k * 2 * G.wb * 512), mrow = wrow + (uint32_t)(G.wb * 512);
            for (int c = lo >> 1; c <= c1; ++c) {
              const uint32_t ao = (uint32_t)(2 * c * 512);
              const uint32_t bo = (uint32_t)((yl * G.hb + 2 * c) * 128);
              mma_bf16(tmem, make_desc(wrow + ao, 512, 128), make_desc(habase + bo, 128, (uint32_t)(G.hb * 128)),
                       acc);
              mma_bf16(tmem + 256u, make_desc(mrow + ao, 512, 128),
                       make_desc(hsbase + bo, 128, (uint32_t)(G.hb * 128)), acc);
              acc = 1u;
            }
            mma_commit(smem_u32(&s_free[k]));
            if (y + NB - 1 < G.fw && !issue_row(y + NB - 1)) {
              s_err = 1;
              atomicOr(p.error, 1);
              break;
            }
          }
          // also after an error: the MMAs issued before it are then tracked by this phase
          mma_commit(mbar);
          committed = true;
        }
        // one thread waits for the MMAs; the others rest at the barrier
        if (tid == 0 && committed) {
          if (!mbar_wait(mbar, parity)) {
            s_err = 1;
            atomicOr(p.error, 1);
          }
          parity ^= 1u;
          asm volatile("tcgen05.fence::before_thread_sync;");
        }
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;");
        if (s_err) break;
      }
      if (s_err) break;

      // Prefetch (thread 0): the next work item is taken now and, when its
      // grain has this footprint geometry (same shared-memory layout, zero
      // blocks in place) and its tile lies in the frame by the +-(half - 1)
      // bound (so that it is searched, not skipped), its first operand rows
      // and its first strip's image rows are issued into the ring and the
      // staging rows, which this tile no longer reads, to land during this
      // tile's epilogue.
      if (tid == 0) {
        pf_next = atomicAdd(p.work_next, 1);
        const int li2 = pf_next / tiles, t2 = pf_next - li2 * tiles;
        if (li2 < count) {
          const int gi2 = p.list[li2];
          const int P2 = g.pstart[gi2 + 1] - g.pstart[gi2];
          if (!(g.masked[gi2] || (g.flags[gi2] & 2) || P2 <= 0 || P2 > kMaxPatternPoints) && p.half[gi2] == G.half) {
            const int tu2 = t2 / p.tiles_v, tv2 = t2 - tu2 * p.tiles_v;
            const int u0b = -p.left + tu2 * kTileU, u1b = min(u0b + kTileU - 1, p.right);
            const int v0b = -p.up + tv2 * kTileV, v1b = min(v0b + kTileV - 1, p.down);
            const int X2 = g.refx[gi2] + (int)round(g.dx[gi2]), Y2 = g.refy[gi2] + (int)round(g.dy[gi2]);
            const int e = G.half - 1;
            if (X2 - e + u0b >= 0 && Y2 - e + v0b >= 0 && X2 + e + u1b < p.cur.dimx && Y2 + e + v1b < p.cur.dimy) {
              const CUtensorMap* tm2 = p.tmaps + gi2;
              asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(tm2) : "memory");
              pf = true;
              for (int y = 0; y < min(NB - 1, G.fw); ++y)
                if (!issue_row_of(tm2, y)) {
                  s_err = 1;
                  atomicOr(p.error, 1);
                  break;
                }
              if (!s_err) stage_rows_at((X2 - G.half + u0b) & ~7, Y2 - G.half + v0b, 0);
            }
          }
        }
      }

      // ---- epilogue: per rotation lane D / sqrt(S), max over rotations, keep the best candidates
      const int q = warp & 3, h = warp >> 2;  // TMEM lane quadrant (x shift j) and column quarter
      float sc[2];
#pragma unroll
      for (int ch = 0; ch < 2; ++ch) {
        uint32_t dv[32], sv[32];
        const uint32_t ta = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(64 * h + 32 * ch);
        tmem_ld32(ta, dv);
        tmem_ld32(ta + 256u, sv);
        int mine = INT_MIN;
#pragma unroll
        for (int k = 0; k < 32; ++k) {
          const float d = __uint_as_float(dv[k]), s2 = __uint_as_float(sv[k]);
          const int key = (lane < p.nrot && s2 > 0.0f) ? f2key(d * rsqrtf(s2)) : INT_MIN;
          const int m = __reduce_max_sync(0xffffffffu, key);
          if (lane == k) mine = m;
        }
        // this lane's candidate: accumulator column 64 h + 32 ch + lane
        const int ul = 24 - 8 * q + (lane & 7), vl = 8 * h + 4 * ch + (lane >> 3);
        sc[ch] = (u0 + ul <= u1 && v0 + vl <= v1 && mine != INT_MIN) ? key2f(mine) : -INFINITY;
      }
      // per-warp best `keep` (down to kKeepRelWeak below the warp's best: the
      // tile's best is at least as high), then the block's best `keep` among them
      float wtop = -INFINITY;
      for (int k = 0; k < keep; ++k) {
        const int bc = sc[1] > sc[0] ? 1 : (sc[0] > -INFINITY ? 0 : -1);
        const float bv = bc == 1 ? sc[1] : sc[0];
        const int key = (bc >= 0) ? f2key(bv) : INT_MIN;
        const int mkey = __reduce_max_sync(0xffffffffu, key);
        if (k == 0) wtop = key2f(mkey);
        if (mkey == INT_MIN || (k > 0 && wtop > 0.0f && key2f(mkey) < wtop * (1.0f - kKeepRelWeak))) {
          if (lane == 0)
            for (int r = k; r < keep; ++r) {
              s_cv[warp * kBf16KeepMax + r] = -INFINITY;
              s_ci[warp * kBf16KeepMax + r] = -1;
            }
          break;
        }
        const unsigned who = __ballot_sync(0xffffffffu, key == mkey && bc >= 0);
        const int wl = who ? __ffs(who) - 1 : -1;
        int packed = -1;
        if (lane == wl) {
          const int ul = 24 - 8 * q + (lane & 7), vl = 8 * h + 4 * bc + (lane >> 3);
          packed = (ul << 8) | vl;
          if (bc == 0) sc[0] = -INFINITY;
          else sc[1] = -INFINITY;
        }
        packed = __shfl_sync(0xffffffffu, packed, wl >= 0 ? wl : 0);
        if (lane == 0) {
          s_cv[warp * kBf16KeepMax + k] = wl >= 0 ? key2f(mkey) : -INFINITY;
          s_ci[warp * kBf16KeepMax + k] = wl >= 0 ? packed : -1;
        }
      }
      __syncthreads();
      if (warp == 0) {
        // 16 warps x 8 entries: this lane holds entries lane + 32 i
        const bool used = (lane & (kBf16KeepMax - 1)) < keep;
        float cv[4];
        int ci[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          cv[i] = used ? s_cv[lane + 32 * i] : -INFINITY;
          ci[i] = used ? s_ci[lane + 32 * i] : -1;
        }
        float top = -INFINITY, rel = kKeepRel;
        for (int k = 0; k < kBf16KeepMax; ++k) {
          float bv = cv[0];
          int bi = ci[0], bsel = 0;
#pragma unroll
          for (int i = 1; i < 4; ++i)
            if (cv[i] > bv) {
              bv = cv[i];
              bi = ci[i];
              bsel = i;
            }
          const int key = bi >= 0 ? f2key(bv) : INT_MIN;
          const int mkey = __reduce_max_sync(0xffffffffu, key);
          if (k == 0) {
            top = key2f(mkey);
            if (lane == 0) p.tile_top[(size_t)li * tiles + t] = mkey == INT_MIN ? -INFINITY : top;
            // D / sqrt(S) <= NCC sqrt(C0C0)
            if (!(top * c00_rsqrt >= kGoodMatch)) rel = kKeepRelWeak;
          }
          // candidates scoring more than `rel` below the tile's best are not rescored
          const bool near = !(top > 0.0f) || key2f(mkey) >= top * (1.0f - rel);
          if (k >= keep || !near || mkey == INT_MIN) {
            if (lane == 0) {
              for (int r = k; r < kBf16KeepMax; ++r) topk[r] = make_int2(INT_MIN, INT_MIN);
              s_nkept = k;
              s_rel = rel;
            }
            break;
          }
          const unsigned who = __ballot_sync(0xffffffffu, key == mkey && bi >= 0);
          const int wl = who ? __ffs(who) - 1 : -1;
          int packed = -1;
          if (lane == wl) {
            packed = bi;
#pragma unroll
            for (int i = 0; i < 4; ++i)
              if (i == bsel) {
                cv[i] = -INFINITY;
                ci[i] = -1;
              }
          }
          packed = __shfl_sync(0xffffffffu, packed, wl >= 0 ? wl : 0);
          if (lane == 0) {
            topk[k] = (wl >= 0 && packed >= 0) ? make_int2(u0 + (packed >> 8), v0 + (packed & 0xff))
                                               : make_int2(INT_MIN, INT_MIN);
            s_kept[k] = (wl >= 0 && packed >= 0) ? packed : -1;
            if (k == kBf16KeepMax - 1) {
              s_nkept = kBf16KeepMax;
              s_rel = rel;
            }
          }
        }
      }
      __syncthreads();
      // rotation steps to rescore at each kept candidate: those whose score lies
      // within the tile's keep margin of that candidate's best step.  A
      // candidate's 32 rotation lanes sit in TMEM lane quadrant 3 - (u >> 3),
      // column 8 v + (u & 7); the warp of that quadrant reads them back.
      if (warp < 4) {
        unsigned* rot_g = p.topk_rot + ((size_t)li * tiles + t) * kBf16KeepMax;
        const int nk = s_nkept;
        const float rel_t = s_rel;
        for (int k = 0; k < nk; ++k) {
          const int pk = s_kept[k];
          if (pk < 0 || 3 - ((pk >> 8) >> 3) != warp) continue;
          const int ul = pk >> 8, vl = pk & 0xff;
          const uint32_t col = (uint32_t)(8 * vl + (ul & 7));
          const uint32_t ta = tmem + ((uint32_t)(32 * warp) << 16) + col;
          const float d = __uint_as_float(tmem_ld1(ta)), s2 = __uint_as_float(tmem_ld1(ta + 256u));
          const bool ok = lane < p.nrot && s2 > 0.0f;
          const float sv = ok ? d * rsqrtf(s2) : -INFINITY;
          const float best = key2f(__reduce_max_sync(0xffffffffu, ok ? f2key(sv) : INT_MIN));
          const unsigned m = __ballot_sync(0xffffffffu, ok && (!(best > 0.0f) || sv >= best * (1.0f - rel_t)));
          if (lane == 0) rot_g[k] = m;
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;");
      __syncthreads();
    }
    if (s_err) break;
  }
  __syncthreads();
  if (s_err && tid == 0) {
    // Before the tensor memory is freed and the CTA exits: the bulk copies still
    // in flight (at most one per ring buffer: a copy into a buffer is issued
    // only after the previous one was consumed) and the last committed MMA phase
    // (a no-op when it completed, or when none was committed), with the longer
    // drain bound.
    for (int k = 0; k < kRing; ++k)
      for (unsigned u = s_con[k]; u < s_iss[k]; ++u) mbar_wait(smem_u32(&s_full[k]), u & 1u, kDrainLimit);
    if (s_stage_out) mbar_wait(smem_u32(&s_stage), sparity, kDrainLimit);  // the image rows still in flight
    mbar_wait(mbar, parity ^ 1u, kDrainLimit);
  }
  asm volatile("tcgen05.fence::after_thread_sync;");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
}
// ---------------------------------------------------------------------------
// 3. Exact rescoring of the kept candidates of a tile, at the rotation steps
//    the search marked for each (those within the keep margin of the
//    candidate's best step), with the exact search's integer sums and NCC
//    expression; tiles of a multi-tile zone whose best score is more than the
//    weak keep margin below the grain's best tile are not rescored.  One block per (grain, tile); a work unit is one rotation
//    step for two candidates that both need it (or one), taken by one warp
//    whose lanes share the pattern points; per candidate the best record over
//    its rotation steps in the reference's order.
__global__ void __launch_bounds__(256, 4) k_rescore_bf16(Bf16Launch p) {
  constexpr int kW = 8;
  __shared__ double s_bn[kBf16KeepMax][kW];
  __shared__ int s_bi[kBf16KeepMax][kW];
  __shared__ int s_base[kBf16KeepMax], s_uv[kBf16KeepMax];
  __shared__ int s_nk, s_nu;
  __shared__ int s_unit[kNRot * kBf16KeepMax / 2];  // rotation | first candidate << 8 | second << 16 (255: none)
  const int item = blockIdx.x;
  const int tiles = p.tiles_u * p.tiles_v;
  const int li = item / tiles;
  if (li >= *p.list_count) return;
  const int gi = p.list[li];
  const GrainsDev& g = p.g;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  SearchBest* rec = p.rescored + (size_t)item * kBf16KeepMax;
  if (*p.error) {
    // a search CTA gave up a wait and left tiles without kept candidates: no
    // candidate anywhere, so the level's finalize hands every grain to the
    // exact re-search
    if (tid < kBf16KeepMax) rec[tid] = SearchBest{0.0, INT_MAX, 0};
    return;
  }
  const int b = g.pstart[gi], P = g.pstart[gi + 1] - b;
  const bool skip = g.masked[gi] || (g.flags[gi] & 7) || P <= 0 || P > kMaxPatternPoints;
  const int NU = p.left + p.right + 1, NV = p.up + p.down + 1;
  if (tid == 0) {  // the kept candidates, compacted: anchor pixel index and order index without the rotation
    int nk = 0, nu = 0;
    // a tile whose best score lies further below the grain's best tile than
    // the weak keep margin cannot hold the exact best (the keep rule's bound)
    bool far = false;
    if (tiles > 1) {
      const float* tt = p.tile_top + (size_t)li * tiles;
      float best = -INFINITY;
      for (int k = 0; k < tiles; ++k) best = fmaxf(best, tt[k]);
      far = best > 0.0f && tt[item - li * tiles] < best * (1.0f - kKeepRelWeak);
    }
    if (!skip && !far) {
      const int2* cand = p.topk + (size_t)item * kBf16KeepMax;
      const unsigned* rots = p.topk_rot + (size_t)item * kBf16KeepMax;
      const int gdx = (int)round(g.dx[gi]), gdy = (int)round(g.dy[gi]);
      unsigned rm[kBf16KeepMax];
      for (int k = 0; k < p.keep && k < kBf16KeepMax; ++k) {
        const int2 c = cand[k];
        if (c.x == INT_MIN) continue;
        s_base[nk] = (g.refy[gi] + gdy + c.y) * p.cur.pitch + (g.refx[gi] + gdx + c.x);
        s_uv[nk] = (c.x + p.left) * NV + (c.y + p.up);
        rm[nk] = rots[k];
        ++nk;
      }
      // units: per rotation step, the candidates that need it, two at a time
      for (int r = 0; r < p.nrot; ++r) {
        int first = -1;
        for (int k = 0; k < nk; ++k) {
          if (!((rm[k] >> r) & 1u)) continue;
          if (first < 0) {
            first = k;
          } else {
            s_unit[nu++] = r | (first << 8) | (k << 16);
            first = -1;
          }
        }
        if (first >= 0) s_unit[nu++] = r | (first << 8) | (255 << 16);
      }
    }
    s_nk = nk;
    s_nu = nu;
  }
  if (tid < kBf16KeepMax * kW) {
    s_bn[tid / kW][tid % kW] = 0.0;
    s_bi[tid / kW][tid % kW] = INT_MAX;
  }
  __syncthreads();
  const int nk = s_nk;
  if (nk == 0) {
    if (tid < kBf16KeepMax) rec[tid] = SearchBest{0.0, INT_MAX, 0};
    return;
  }
  const long long Pl = P, S0 = g.s0[gi];
  const double den1 = (double)(Pl * g.s00[gi] - S0 * S0);
  const int pitch = p.cur.pitch;
  const int nu = s_nu;
  for (int u = warp; u < nu; u += kW) {
    const int unit = s_unit[u];
    const int r = unit & 0xff, k0 = (unit >> 8) & 0xff, k1 = (unit >> 16) & 0xff;
    const double2 cs = p.rot_cs[(size_t)gi * kNRot + r];  // the weights kernel's cos / sin of the step
    const double sr = cs.y, cr = cs.x;
    const float cf = (float)cr, sf = (float)sr;
    const bool two = k1 != 255;
    const uint16_t* pa = p.cur.pix + s_base[k0];
    const uint16_t* pb = p.cur.pix + s_base[two ? k1 : k0];
    unsigned s1a = 0, s1b = 0;
    unsigned long long s11a = 0, s11b = 0, s01a = 0, s01b = 0;
#pragma unroll 4
    for (int i = lane; i < P; i += 32) {
      const short2 q = rotate_round_fast(g.pat[b + i], cf, sf, cr, sr);
      const int o = (int)q.y * pitch + (int)q.x;
      const unsigned w = g.w0[b + i];
      const unsigned va = __ldg(pa + o);
      s1a += va;
      s11a += (unsigned long long)(va * va);
      s01a += (unsigned long long)(w * va);
      if (two) {
        const unsigned vb = __ldg(pb + o);
        s1b += vb;
        s11b += (unsigned long long)(vb * vb);
        s01b += (unsigned long long)(w * vb);
      }
    }
    unsigned long long a0 = s1a, c0 = s11a, d0 = s01a, a1 = s1b, c1 = s11b, d1 = s01b;
    for (int o = 16; o > 0; o >>= 1) {
      a0 += __shfl_xor_sync(0xffffffffu, a0, o);
      c0 += __shfl_xor_sync(0xffffffffu, c0, o);
      d0 += __shfl_xor_sync(0xffffffffu, d0, o);
      a1 += __shfl_xor_sync(0xffffffffu, a1, o);
      c1 += __shfl_xor_sync(0xffffffffu, c1, o);
      d1 += __shfl_xor_sync(0xffffffffu, d1, o);
    }
    if (lane < 2 && (lane == 0 || two)) {
      const int k = lane == 0 ? k0 : k1;
      const long long S1 = (long long)(lane == 0 ? a0 : a1), S11 = (long long)(lane == 0 ? c0 : c1);
      const long long S01 = (long long)(lane == 0 ? d0 : d1);
      const long long num = Pl * S01 - S0 * S1;
      const long long d2 = Pl * S11 - S1 * S1;
      const double ncc = (double)num / sqrt(den1 * (double)d2);
      const int idx = r * NU * NV + s_uv[k];
      if (better_b(ncc, idx, s_bn[k][warp], s_bi[k][warp])) {
        s_bn[k][warp] = ncc;
        s_bi[k][warp] = idx;
      }
    }
  }
  __syncthreads();
  if (tid < kBf16KeepMax) {
    double fn = 0.0;
    int fi = INT_MAX;
    for (int w = 0; w < kW; ++w)
      if (better_b(s_bn[tid][w], s_bi[tid][w], fn, fi)) {
        fn = s_bn[tid][w];
        fi = s_bi[tid][w];
      }
    rec[tid] = SearchBest{fn, fi, 0};
  }
}

// ---------------------------------------------------------------------------
size_t bf16_weight_entries(int half) {
  const Geom G = geom_of(half);
  // W, M, per-row block ranges (2 fw <= 190 bytes, padded to keep slots 512-byte aligned)
  return 2 * (size_t)G.fw * G.nbf * kNRot + kNRot;
}

// The weights kernel counts the points landing on a pixel in 8 bits: a
// rotated pattern puts at most 4 distinct offsets on one pixel, each repeated
// at most max_dup times.
bool bf16_supported(int max_r, int nrot, int max_dup) {
  return 2 * max_r + 1 < kMaxFoot && nrot >= 1 && nrot <= kNRot && 4 * max_dup <= 255;
}

// A ring of `ring` operand-row buffers leaves strips of at least one row for
// every footprint up to half-extent max_half within the shared-memory budget.
bool bf16_ring_ok(int max_half, int ring) {
  if (ring != 2 && ring != 3 && ring != 4 && ring != 6) return false;  // the instantiated kernels
  const Geom G = geom_of(max_half, ring);
  const int halo_row = 2 * G.hb * 128 + G.rp;
  return (kSmemBudget - ring * 2 * G.wb * 512 - (kStageBoxRows - 1) * G.rp) / halo_row - 31 >= 1;
}

void prepare_search_bf16() {
  ensure_smem((const void*)k_search_bf16<2>, kSmemBudget);
  ensure_smem((const void*)k_search_bf16<3>, kSmemBudget);
  ensure_smem((const void*)k_search_bf16<4>, kSmemBudget);
  ensure_smem((const void*)k_search_bf16<6>, kSmemBudget);
  ensure_smem((const void*)k_weights_bf16, kWSmem);
}

// Tensor maps of the grains' operand slots for a level with `nrot` rotation
// steps (host): per grain a 5-D BF16 tensor {8 values, nrot steps, nbf blocks,
// fw rows, W/M} at its slot, read one footprint row at a time as a box
// {8, 32, nbf, 1, 1} - the 32 - nrot slots beyond the tensor come back as
// zeros, in the shared-memory layout of the A operands.  Returns false when
// the driver's encoder is unavailable or refuses a map.
static PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  });
  return encode;
}

bool bf16_encode_tmaps(const int* half, const size_t* wofs, int n, unsigned char* wslots, int nrot,
                       CUtensorMap* out) {
  const PFN_cuTensorMapEncodeTiled_v12000 encode = tmap_encoder();
  if (!encode || nrot < 1 || nrot > kNRot) return false;
  const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
  for (int i = 0; i < n; ++i) {
    const Geom G = geom_of(half[i]);
    if (G.fw >= kMaxFoot) {  // never searched by the BF16 kernels (bf16_supported): a small valid map
      const cuuint64_t d1[5] = {8, 1, 1, 1, 1};
      const cuuint64_t s1[4] = {16, 16, 16, 16};
      const cuuint32_t b1[5] = {8, 1, 1, 1, 1};
      if (encode(&out[i], CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, wslots + wofs[i] * 16, d1, s1, b1, estr,
                 CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                 CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return false;
      continue;
    }
    const cuuint64_t dims[5] = {8, (cuuint64_t)nrot, (cuuint64_t)G.nbf, (cuuint64_t)G.fw, 2};
    const cuuint64_t strides[4] = {16, 16ull * nrot, 16ull * nrot * G.nbf, 16ull * nrot * G.nbf * G.fw};
    const cuuint32_t box[5] = {8, (cuuint32_t)kNRot, (cuuint32_t)G.nbf, 1, 1};
    if (encode(&out[i], CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, wslots + wofs[i] * 16, dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return false;
  }
  return true;
}

// Tensor maps of one frame buffer (host): the u16 image {dimx, dimy} at its
// row pitch, read as boxes of 8 rows x (8 hb + 16) pixels, one map per Hankel
// width hb = 2 nch at out[nch] (nch = 2 .. kBf16FrameMaps - 1, which covers
// every footprint below kMaxFoot; out[0] and out[1] repeat nch = 2).  Pixels
// outside the frame read as zeros.
bool bf16_encode_frame_tmaps(const uint16_t* pix, int dimx, int dimy, int pitch, CUtensorMap* out) {
  const PFN_cuTensorMapEncodeTiled_v12000 encode = tmap_encoder();
  if (!encode || dimx < 1 || dimy < 1 || pitch < dimx) return false;
  static_assert((kMaxFoot - 1 + 7) / 8 / 2 + 2 < kBf16FrameMaps, "one frame map per Hankel width");
  const cuuint64_t dims[2] = {(cuuint64_t)dimx, (cuuint64_t)dimy};
  const cuuint64_t strides[1] = {2ull * pitch};
  const cuuint32_t estr[2] = {1, 1};
  for (int k = 0; k < kBf16FrameMaps; ++k) {
    const int hb = 2 * (k < 2 ? 2 : k);
    const cuuint32_t box[2] = {(cuuint32_t)(8 * hb + 16), (cuuint32_t)kStageBoxRows};
    if (encode(&out[k], CU_TENSOR_MAP_DATA_TYPE_UINT16, 2, const_cast<uint16_t*>(pix), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return false;
  }
  return true;
}

void launch_search_bf16(const Bf16Launch& p, int grid, cudaStream_t s, cudaEvent_t* ev, cudaEvent_t frame_ready) {
  const int items = p.max_items;
  if (ev) cudaEventRecord(ev[0], s);
  k_weights_bf16<<<p.max_items / (p.tiles_u * p.tiles_v), kWThreads, kWSmem, s>>>(p);
  // the weights need only the reference frame: the current one may still be uploading until here
  if (frame_ready) cudaStreamWaitEvent(s, frame_ready, cudaEventWaitExternal);
  if (ev) cudaEventRecord(ev[1], s);
  switch (p.ring) {
    case 2: k_search_bf16<2><<<grid, kThreads, kSmemBudget, s>>>(p); break;
    case 3: k_search_bf16<3><<<grid, kThreads, kSmemBudget, s>>>(p); break;
    case 6: k_search_bf16<6><<<grid, kThreads, kSmemBudget, s>>>(p); break;
    default: k_search_bf16<4><<<grid, kThreads, kSmemBudget, s>>>(p); break;
  }
  if (ev) cudaEventRecord(ev[2], s);
  k_rescore_bf16<<<items, 256, 0, s>>>(p);
  if (ev) cudaEventRecord(ev[3], s);
}

}  // namespace ptk
