// Internal declarations shared by the kernels and the host runtime of the
// sm_100a tracking path.  Not part of the public ABI (include/ptk.h).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/ptk.h"

namespace ptk {

// Largest pattern (points per grain) the search and subpixel kernels stage in
// shared memory.  A disc of radius 50 has 7845 points.
constexpr int kMaxPatternPoints = 16384;
// Candidate tile of one search work item: 32 x-offsets (one per lane) by up
// to 32 y-offsets (8 warps x 4 rows).
constexpr int kTileU = 32;
constexpr int kTileV = 32;
constexpr int kSearchThreads = 256;
constexpr int kSubpixThreads = 128;

// Device view of the grain state, structure of arrays (one entry per grain).
struct GrainsDev {
  int n;
  int* refx;
  int* refy;
  double* refrot;
  double* radius;
  double* dx;
  double* dy;
  double* drot;
  double* dx_prev;
  double* dy_prev;
  double* drot_prev;
  double* upix;
  double* vpix;
  double* rot_inc;
  double* ncc;
  double* ncc_rescue;
  double* ncc_subpix;
  double* mean0;     // mean of the reference pattern pixels
  double* c0c0;      // sum of squared deviations of the reference pattern pixels
  long long* s0;     // exact sum of reference pattern pixels
  long long* s00;    // exact sum of their squares
  uint8_t* masked;
  uint8_t* status;   // PTK_ST_* bits
  int* flags;        // per-stage scratch flag (bit 0: footprint out of frame)
  const int* pstart; // CSR offsets into the pattern arrays, n + 1 entries
  const short2* pat; // pattern offsets (grain_type_2D::pattern)
  short2* pat0;      // pattern rotated by refrot and rounded (pattern0_rotated)
  uint16_t* w0;      // reference pixel at each pattern0_rotated point
};

struct FrameDev {
  const uint16_t* pix;  // row-major, `pitch` elements per row
  int pitch;
  int dimx, dimy;
};

// Best candidate of one search work item: NCC value and its position in the
// reference's iteration order (rotation-major, then x, then y).
struct SearchBest {
  double ncc;
  int idx;
  int pad;
};

struct SearchLaunch {
  GrainsDev g;
  FrameDev cur;
  const int* list;        // grains to search (ordered by decreasing cost for level 0)
  const int* list_count;  // number of entries in `list` (device)
  int* work_next;         // work-queue head (zeroed before launch)
  const double* steps;    // rotation steps of the zone
  int nrot;
  int left, right, up, down;
  int tiles_u, tiles_v;
  SearchBest* best;       // [list entry][rotation][tile]
  int max_items;          // capacity of `best` in work items
};

struct FinalizeLaunch {
  GrainsDev g;
  const int* list;
  const int* list_count;
  const double* steps;
  int nrot, left, up;
  int nu, nv;  // zone width (left + right + 1) and height (up + down + 1)
  int tiles;   // tiles_u * tiles_v
  const SearchBest* best;
  int level;
  double NCC_min, NCC_min_super;
  int* out_list;   // next-level list (rescue / super-rescue), or the re-search list
  int* out_count;
  int redo;        // 1: rejected grains go to out_list for an exact re-search of this level, unmarked
};

// BF16 tensor-core search: kept candidates per tile (upper bound of `keep`).
constexpr int kBf16KeepMax = 8;
constexpr int kBf16FrameMaps = 9;  // frame tensor maps per frame buffer, one per Hankel width

struct Bf16Launch {
  GrainsDev g;
  FrameDev cur;
  const int* list;
  const int* list_count;
  int* work_next;           // work-queue head over list entries (zeroed before launch)
  const double* steps;
  int nrot;
  int left, right, up, down;
  int tiles_u, tiles_v;
  int keep;                 // candidates per tile rescored exactly (1..kBf16KeepMax)
  int max_items;            // list capacity x tiles: grid of the per-tile kernels
  const int* half;          // per grain: footprint half-extent ceil(max |offset|) + 1
  const size_t* wofs;       // per grain: offset of its weight slot in wslots (16-byte units)
  unsigned char* wslots;    // BF16 weights of the level's rotation steps, per grain
  const CUtensorMap* tmaps; // per grain: tensor map of its operand rows (bf16_encode_tmaps)
  const CUtensorMap* frame_tmaps;  // the current frame's maps per Hankel width (bf16_encode_frame_tmaps)
  double2* rot_cs;          // [grain][32]: cos, sin of each rotation step's total angle (weights kernel)
  int2* topk;               // [list entry][tile][kBf16KeepMax] kept (u, v), INT_MIN when none
  unsigned* topk_rot;       // same layout: bit r = rotation step r is rescored at that candidate
  int ring;                 // operand-row buffers of the search kernel's ring (2..8; the strips take the rest)
  float* tile_top;          // [list entry][tile] the tile's best ranking score (-inf: no candidate)
  SearchBest* rescored;     // [list entry][tile][kBf16KeepMax] exact best per kept candidate
  int* error;               // set when a bounded wait gave up
  int probe_wait;           // failure-path test: > 0 makes the search kernel first wait this many polls on a
                            // barrier nothing arrives on (before any copy or MMA), then report the timeout
};

struct SubpixParams {
  double tol;
  double init_dir[3];
  double disp_max;
  double stiffness;
  int interp;
};

struct LmParams {
  int max_iter;
  double tol;   // step tolerance in pixels (rotation scaled by the grain radius)
  int* iters;   // optional per-grain iteration count
  const int* order;  // grains by decreasing pattern size (one block each), or null for index order
  int max_r;         // largest pattern radius (sizes the staged frame region)
  int* redo_list;    // grains whose refinement left the cell (for Powell), or null to keep every result
  int* redo_count;   // their number (zeroed before the launch)
  double cell_px;    // cell of the integer optimum: |dx|, |dy| <= cell_px
  double cell_rot;   // and |drot| <= cell_rot
};

// Raises `func`'s dynamic shared-memory limit to at least `bytes` on the
// current device.  The attribute belongs to the device that is current when it
// is set, so the largest value set is remembered per (kernel, device), behind a
// mutex: contexts on several devices, or created from several host threads,
// each get the limit their launches need (ptk_api.cu).
cudaError_t ensure_smem(const void* func, size_t bytes);

// ---- host-side launchers (defined in the kernel files) ------------------
void launch_subpix_lm(const GrainsDev& g, const FrameDev& cur, const LmParams& lp, cudaStream_t s);
void launch_grad_f32(const GrainsDev& g, const FrameDev& cur, const double* X, double* f, double* grad,
                     cudaStream_t s);
void launch_precompute(const GrainsDev& g, const FrameDev& ref, cudaStream_t s);
void launch_stage_begin(const GrainsDev& g, int* counts, cudaStream_t s);
void launch_search(const SearchLaunch& p, int grid, size_t smem, cudaStream_t s);
size_t search_smem_bytes(int max_points, int max_patch_elems);
int search_occupancy(size_t smem);
size_t search_tiled_smem(int max_r);
int search_tiled_occupancy(size_t smem, int max_r);
void launch_search_tiled(const SearchLaunch& p, int max_r, int grid, size_t smem, cudaStream_t s);
void launch_finalize(const FinalizeLaunch& p, int n_grains, cudaStream_t s);
bool bf16_supported(int max_r, int nrot, int max_dup);
bool bf16_ring_ok(int max_half, int ring);
constexpr int kBf16RingDefault = 4;
size_t bf16_weight_entries(int half);
bool bf16_encode_tmaps(const int* half, const size_t* wofs, int n, unsigned char* wslots, int nrot,
                       CUtensorMap* out);
bool bf16_encode_frame_tmaps(const uint16_t* pix, int dimx, int dimy, int pitch, CUtensorMap* out);
void prepare_search_bf16();
// ev (optional, 5 events): recorded before the first kernel and after each of the four
// frame_ready (may be null): an event the search waits for after the weights
// kernel (recorded where the current frame's upload completes)
void launch_search_bf16(const Bf16Launch& p, int grid, cudaStream_t s, cudaEvent_t* ev = nullptr,
                        cudaEvent_t frame_ready = nullptr);
void launch_end_frame(const GrainsDev& g, int swap_reference, cudaStream_t s);
void prepare_subpix(int max_points, int max_r);
// order: grains by decreasing pattern size (one block each), or null for index
// order; with list_count, only the first *list_count entries of `order` (a
// device-built list) are refined
void launch_subpix_powell(const GrainsDev& g, const FrameDev& cur, const FrameDev& ref,
                          const SubpixParams& sp, int max_points, int max_r, const int* order, cudaStream_t s,
                          const int* list_count = nullptr);
void launch_objective(const GrainsDev& g, const FrameDev& cur, const SubpixParams& sp, const double* X,
                      double* f, double* grad, int max_points, cudaStream_t s);
void launch_widen_u8(const uint8_t* src, size_t src_pitch, uint16_t* dst, int dst_pitch, int dimx, int dimy,
                     cudaStream_t s);
void launch_remap_build(const double* params14, const double* trig4, double2* map, int dimx, int dimy,
                        cudaStream_t s);
void launch_remap_apply(const double2* map, const uint16_t* src, uint16_t* dst, int pitch, int dimx, int dimy,
                        cudaStream_t s);
// RAW mosaic -> grey frame (ptk_raw.cu): stencil offsets of a mode, and the
// demosaic (+ rescale) launches; min_max = 2 unsigned of device scratch.
int raw_stencil_lo(int mode);
int raw_stencil_hi(int mode);
void launch_raw_demosaic(const uint16_t* raw, int raw_width, int left, int top, int mode, int rescale, uint16_t* dst,
                         int pitch, int dimx, int dimy, unsigned* min_max, int num_sms, cudaStream_t s);

}  // namespace ptk
