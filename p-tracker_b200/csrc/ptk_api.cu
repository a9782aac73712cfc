// Host runtime of the C ABI declared in include/ptk.h.
//
// A context owns: both frames (uint16, row-major, pitch rounded to 64 pixels),
// the grain state as one device block of structure-of-arrays, the patterns in
// CSR form, the rotation-step lists of the three zones, the device-built
// rescue lists, the search scratch, the cached undistortion map, and the CUDA
// graphs of the per-frame pipeline.  Every launch goes to the context stream.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "ptk_internal.cuh"

using namespace ptk;

cudaError_t ptk::ensure_smem(const void* func, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, size_t> set;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(mu);
  size_t& cur = set[{func, dev}];
  if (bytes <= cur) return cudaSuccess;
  e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) cur = bytes;
  return e;
}

namespace {

constexpr int kMaxRotSteps = 4096;
constexpr int kFrameBufs = 3;  // device frame buffers: the two slots and a spare for overlapped uploads
thread_local std::string g_static_error;

// Layout of the grain block: 16 double fields, 2 int64 fields, 3 int32 fields,
// 2 uint8 fields, each n entries, in this order.
enum { D_REFROT, D_RADIUS, D_DX, D_DY, D_DROT, D_DXP, D_DYP, D_DROTP, D_UPIX, D_VPIX, D_ROTINC, D_NCC, D_NCCR, D_NCCS,
       D_MEAN0, D_C0C0, D_COUNT };
enum { L_S0, L_S00, L_COUNT };
enum { I_REFX, I_REFY, I_FLAGS, I_COUNT };
enum { B_MASKED, B_STATUS, B_COUNT };

struct BlockLayout {
  size_t d_off, l_off, i_off, b_off, total;
  explicit BlockLayout(int n) {
    const size_t nn = (size_t)(n > 0 ? n : 1);
    d_off = 0;
    l_off = d_off + D_COUNT * nn * 8;
    i_off = l_off + L_COUNT * nn * 8;
    b_off = i_off + ((I_COUNT * nn * 4 + 15) & ~(size_t)15);
    total = b_off + ((B_COUNT * nn + 15) & ~(size_t)15);
  }
};

}  // namespace

struct ptk_ctx {
  ptk_config cfg{};
  int device{0};
  int num_sms{148};
  cudaStream_t stream{nullptr};
  cudaStream_t own_stream{nullptr};
  cudaStream_t cap_stream{nullptr};
  // Three frame buffers: the reference and current slots' and a spare.  Host
  // uploads into buffer p go to copy_stream[p] and record buf_ready[p].  An
  // upload waits for the buffer's last reader: while free_valid[p], that is a
  // frame graph's record of buf_free[p] (right after its precompute for the
  // reference buffer, at its end for the current one, and nothing since);
  // otherwise all the work queued so far (main_mark).  An upload into a slot
  // may go to the spare buffer instead when the spare is released earlier
  // (the slot then uses the spare, and its old buffer becomes the spare).  A
  // frame's graph waits for the current buffer's upload just before its first
  // kernel that reads it, for the reference buffer's before the graph; every
  // other reader at its entry (sync_cur).
  cudaStream_t copy_stream[kFrameBufs]{};
  cudaEvent_t buf_ready[kFrameBufs]{}, buf_free[kFrameBufs]{}, main_mark{nullptr};
  bool ready_pending[kFrameBufs]{};
  bool free_valid[kFrameBufs]{};
  bool released_early[kFrameBufs]{};  // the latest graph using it released it after its precompute
  int64_t used_by_graph[kFrameBufs]{};  // sequence number of the latest graph that read it
  int64_t graph_seq{0};
  std::string err;
  int64_t launches{0};

  // frames
  int pitch{0};
  uint16_t* d_img[kFrameBufs]{};
  uint16_t* d_tmp{nullptr};
  uint8_t* d_u8{nullptr};
  uint16_t* d_raw{nullptr};  // staging of a host RAW mosaic (ptk_load_frame_raw)
  size_t raw_cap{0};         // elements
  unsigned* d_minmax{nullptr};
  int ref_slot{0}, cur_slot{1}, spare_buf{2};  // frame buffers of the slots, and the spare
  bool loaded[2]{false, false};

  // grains
  int n{0};
  void* d_block{nullptr};
  void* d_snap{nullptr};     // device copy of the grain block (ptk_snapshot_grains)
  void* h_stage{nullptr};    // pinned staging for grain upload / download
  size_t h_stage_bytes{0};
  GrainsDev g{};
  std::vector<double> h_radius;

  // patterns
  std::vector<std::vector<short2>> h_pat;
  int* d_pstart{nullptr};
  short2* d_pat{nullptr};
  short2* d_pat0{nullptr};
  uint16_t* d_w0{nullptr};
  int* d_order{nullptr};
  int max_P{0};
  int max_R{0};
  int max_dup{1};  // largest repeat count of one offset within a pattern
  bool patterns_ok{false};

  // zones
  std::vector<double> steps[3];
  double* d_steps[3]{nullptr, nullptr, nullptr};

  // lists: counts[0] = n (level-0 list), counts[1] rescue, counts[2] super-rescue
  int* d_counts{nullptr};
  int* d_lists{nullptr};  // [rescue n][super n][exact re-search n][LM refinements that left their cell n]
  int* d_work{nullptr};
  SearchBest* d_best{nullptr};
  size_t best_cap{0};

  // BF16 tensor-core search scratch (PTK_SEARCH_BF16)
  int* d_bf_half{nullptr};             // per grain footprint half-extent
  size_t* d_bf_wofs{nullptr};          // per grain weight-slot offset (16-byte units)
  unsigned char* d_bf_wslots{nullptr};  // BF16 weights of every rotation step, per grain
  size_t bf_wslots_bytes{0};
  bool bf_geom_dirty{true};            // patterns changed since the slots were laid out
  std::vector<int> h_bf_half;          // host copies of the slot layout (tensor-map encoding)
  std::vector<size_t> h_bf_wofs;
  CUtensorMap* d_bf_tmaps[3]{nullptr, nullptr, nullptr};  // per level: each grain's operand-row tensor map
  CUtensorMap* d_frame_tmaps{nullptr};  // [frame buffer][kBf16FrameMaps] the BF16 search's image-strip maps
  double2* d_bf_rot_cs{nullptr};                           // per grain: cos / sin of the level's rotation steps
  int bf_tmaps_nrot[3]{0, 0, 0};                           // rotation steps they were encoded for (0: stale)
  int2* d_topk{nullptr};
  unsigned* d_topk_rot{nullptr};  // rotation steps of each kept candidate to rescore
  float* d_tile_top{nullptr};     // best ranking score of each (grain, tile)
  SearchBest* d_rescored{nullptr};
  size_t bf_cap{0};  // (list entries x tiles) the per-tile buffers hold

  // distortion
  double disto[14]{};
  bool have_disto{false};
  double2* d_map{nullptr};
  bool map_valid{false};

  // objective buffers
  double* d_X{nullptr};
  double* d_f{nullptr};
  double* d_gr{nullptr};

  // per-frame graphs, keyed by (reference buffer, current buffer, precompute, swap)
  cudaGraphExec_t graph[kFrameBufs * kFrameBufs * 4]{};
  bool graph_dirty{true};

  // level-0 search shape chosen by ptk_autotune (0: the built-in choice)
  int tune_ring{0};   // BF16 form: operand-row buffers of the search kernel
  int tune_exact{0};  // exact form: 1 register-tiled kernel, 2 direct kernel
  bool tuned{false};
  std::string tune_cache;  // ptk_set_tune_cache: JSON file of chosen shapes ("" = none)

  int iref{0};
  bool need_precompute{true};
  int probe_wait{0};  // failure-path test hook (ptk_test_bf16_wait_timeout)
};

namespace {

int fail(ptk_ctx* c, int code, const std::string& msg) {
  if (c) c->err = msg;
  else g_static_error = msg;
  return code;
}

int cuda_fail(ptk_ctx* c, cudaError_t e, const char* what) {
  return fail(c, PTK_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define CK(call)                                      \
  do {                                                \
    cudaError_t e_ = (call);                          \
    if (e_ != cudaSuccess) return cuda_fail(c, e_, #call); \
  } while (0)

void drop_graphs(ptk_ctx* c) {
  for (auto& ge : c->graph)
    if (ge) {
      cudaGraphExecDestroy(ge);
      ge = nullptr;
    }
  c->graph_dirty = false;
}

void invalidate(ptk_ctx* c) { c->graph_dirty = true; }

// The context stream waits for a current-frame upload still in flight on the
// copy stream (entry of every call that reads the current frame or reuses
// its staging outside a frame's graph).
// After the context stream was synchronised from the host, no queued work
// reads any frame buffer any more (uploads into a buffer stay ordered on its
// copy stream): an upload need not wait for anything else.
void all_released(ptk_ctx* c) {
  for (int b = 0; b < kFrameBufs; ++b) {
    c->free_valid[b] = true;
    c->used_by_graph[b] = 0;
  }
}

// The context stream waits for every pending frame upload; the work that
// follows is no longer a frame graph's alone.
void sync_cur(ptk_ctx* c) {
  // the slots' buffers may be read or written by the work that follows
  c->free_valid[c->ref_slot] = c->free_valid[c->cur_slot] = false;
  for (int p = 0; p < kFrameBufs; ++p)
    if (c->ready_pending[p]) {
      cudaStreamWaitEvent(c->stream, c->buf_ready[p], 0);
      c->ready_pending[p] = false;
    }
}

FrameDev frame(const ptk_ctx* c, int phys) {
  return FrameDev{c->d_img[phys], c->pitch, c->cfg.dimx, c->cfg.dimy};
}

SubpixParams subpix_params(const ptk_ctx* c) {
  SubpixParams sp;
  sp.tol = c->cfg.subpix_tol;
  for (int i = 0; i < 3; ++i) sp.init_dir[i] = c->cfg.initial_direction[i];
  sp.disp_max = c->cfg.subpix_displacement_max;
  sp.stiffness = c->cfg.overflow_stiffness;
  sp.interp = c->cfg.image_interpolator;
  return sp;
}

// Rotation steps exactly as the reference's loops produce them
// (src/p-tracker.cpp:684-686); with `rotations 0` every zone becomes
// inc_rot = 1, num_rot = 0 (src/p-tracker.cpp:1191-1201).
int build_steps(ptk_ctx* c, int level) {
  const ptk_zone& z = c->cfg.zone[level];
  double inc = z.inc_rot;
  int num = z.num_rot;
  if (c->cfg.rotations == 0) {
    inc = 1.0;
    num = 0;
  }
  std::vector<double> s;
  const double rotmax = std::fabs(inc * num);
  if (!(inc > 0.0)) return fail(c, PTK_ERR_ARG, "search zone inc_rot must be > 0 (the reference loops forever)");
  for (double drot = -rotmax; drot <= rotmax; drot += inc) {
    s.push_back(drot);
    if ((int)s.size() > kMaxRotSteps) return fail(c, PTK_ERR_LIMIT, "more than 4096 rotation steps in a zone");
  }
  if (z.left < 0 || z.right < 0 || z.up < 0 || z.down < 0) return fail(c, PTK_ERR_ARG, "negative search zone");
  if ((long long)(z.left + z.right + 1) * (z.up + z.down + 1) * (long long)s.size() > (1ll << 30))
    return fail(c, PTK_ERR_LIMIT, "search zone has more than 2^30 candidates");
  c->steps[level] = s;
  if (c->d_steps[level]) cudaFree(c->d_steps[level]);
  c->d_steps[level] = nullptr;
  cudaError_t e = cudaMalloc(&c->d_steps[level], sizeof(double) * (s.size() ? s.size() : 1));
  if (e != cudaSuccess) return cuda_fail(c, e, "cudaMalloc(steps)");
  e = cudaMemcpyAsync(c->d_steps[level], s.data(), sizeof(double) * s.size(), cudaMemcpyHostToDevice, c->stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "cudaMemcpy(steps)");
  invalidate(c);
  return PTK_OK;
}

void bind_grains(ptk_ctx* c) {
  BlockLayout L(c->n);
  char* base = static_cast<char*>(c->d_block);
  const size_t nn = (size_t)(c->n > 0 ? c->n : 1);
  auto D = [&](int k) { return reinterpret_cast<double*>(base + L.d_off + k * nn * 8); };
  auto Lf = [&](int k) { return reinterpret_cast<long long*>(base + L.l_off + k * nn * 8); };
  auto I = [&](int k) { return reinterpret_cast<int*>(base + L.i_off + k * nn * 4); };
  auto B = [&](int k) { return reinterpret_cast<uint8_t*>(base + L.b_off + k * nn); };
  GrainsDev& g = c->g;
  g.n = c->n;
  g.refrot = D(D_REFROT);
  g.radius = D(D_RADIUS);
  g.dx = D(D_DX);
  g.dy = D(D_DY);
  g.drot = D(D_DROT);
  g.dx_prev = D(D_DXP);
  g.dy_prev = D(D_DYP);
  g.drot_prev = D(D_DROTP);
  g.upix = D(D_UPIX);
  g.vpix = D(D_VPIX);
  g.rot_inc = D(D_ROTINC);
  g.ncc = D(D_NCC);
  g.ncc_rescue = D(D_NCCR);
  g.ncc_subpix = D(D_NCCS);
  g.mean0 = D(D_MEAN0);
  g.c0c0 = D(D_C0C0);
  g.s0 = Lf(L_S0);
  g.s00 = Lf(L_S00);
  g.refx = I(I_REFX);
  g.refy = I(I_REFY);
  g.flags = I(I_FLAGS);
  g.masked = B(B_MASKED);
  g.status = B(B_STATUS);
  g.pstart = c->d_pstart;
  g.pat = c->d_pat;
  g.pat0 = c->d_pat0;
  g.w0 = c->d_w0;
}

int upload_patterns(ptk_ctx* c) {
  const int n = c->n;
  std::vector<int> start(n + 1, 0);
  int maxP = 0;
  double maxnorm = 0.0;
  for (int i = 0; i < n; ++i) {
    const size_t P = c->h_pat[i].size();
    if (P > (size_t)kMaxPatternPoints)
      return fail(c, PTK_ERR_LIMIT, "pattern of grain " + std::to_string(i) + " has more than 16384 points");
    if ((long long)start[i] + (long long)P > (1ll << 30)) return fail(c, PTK_ERR_LIMIT, "too many pattern points");
    start[i + 1] = start[i] + (int)P;
    maxP = std::max(maxP, (int)P);
    for (const short2& q : c->h_pat[i]) maxnorm = std::max(maxnorm, std::sqrt((double)q.x * q.x + (double)q.y * q.y));
  }
  const size_t total = (size_t)start[n];
  std::vector<short2> flat;
  flat.reserve(total);
  for (int i = 0; i < n; ++i) flat.insert(flat.end(), c->h_pat[i].begin(), c->h_pat[i].end());
  cudaFree(c->d_pstart);
  cudaFree(c->d_pat);
  cudaFree(c->d_pat0);
  cudaFree(c->d_w0);
  cudaFree(c->d_order);
  c->d_pstart = nullptr;
  c->d_pat = c->d_pat0 = nullptr;
  c->d_w0 = nullptr;
  c->d_order = nullptr;
  CK(cudaMalloc(&c->d_pstart, sizeof(int) * (n + 1)));
  CK(cudaMalloc(&c->d_pat, sizeof(short2) * (total ? total : 1)));
  CK(cudaMalloc(&c->d_pat0, sizeof(short2) * (total ? total : 1)));
  CK(cudaMalloc(&c->d_w0, sizeof(uint16_t) * (total ? total : 1)));
  CK(cudaMalloc(&c->d_order, sizeof(int) * (n ? n : 1)));
  CK(cudaMemcpyAsync(c->d_pstart, start.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice, c->stream));
  if (total) CK(cudaMemcpyAsync(c->d_pat, flat.data(), sizeof(short2) * total, cudaMemcpyHostToDevice, c->stream));
  // level-0 work order: decreasing pattern size (heavy grains first)
  std::vector<int> order(n);
  for (int i = 0; i < n; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return c->h_pat[a].size() > c->h_pat[b].size(); });
  if (n) CK(cudaMemcpyAsync(c->d_order, order.data(), sizeof(int) * n, cudaMemcpyHostToDevice, c->stream));
  int cnt0 = n;
  CK(cudaMemcpyAsync(c->d_counts, &cnt0, sizeof(int), cudaMemcpyHostToDevice, c->stream));
  c->max_P = maxP;
  c->max_R = (int)std::ceil(maxnorm) + 1;
  int max_dup = 1;
  for (int i = 0; i < n; ++i) {
    std::vector<int> keys;
    keys.reserve(c->h_pat[i].size());
    for (const short2& q : c->h_pat[i]) keys.push_back(((int)q.y << 16) ^ ((int)q.x & 0xffff));
    std::sort(keys.begin(), keys.end());
    for (size_t k = 0; k < keys.size();) {
      size_t e = k;
      while (e < keys.size() && keys[e] == keys[k]) ++e;
      max_dup = std::max(max_dup, (int)(e - k));
      k = e;
    }
  }
  c->max_dup = max_dup;
  c->bf_geom_dirty = true;
  c->patterns_ok = true;
  for (int i = 0; i < n; ++i)
    if (c->h_pat[i].empty()) c->patterns_ok = false;
  bind_grains(c);
  c->need_precompute = true;
  invalidate(c);
  return PTK_OK;
}

int ensure_stage(ptk_ctx* c, size_t bytes) {
  if (bytes <= c->h_stage_bytes) return PTK_OK;
  if (c->h_stage) cudaFreeHost(c->h_stage);
  c->h_stage = nullptr;
  c->h_stage_bytes = 0;
  CK(cudaHostAlloc(&c->h_stage, bytes, cudaHostAllocDefault));
  c->h_stage_bytes = bytes;
  return PTK_OK;
}

int check_ready(ptk_ctx* c, bool need_frames) {
  if (c->n <= 0) return fail(c, PTK_ERR_STATE, "no grains set");
  if (!c->patterns_ok) return fail(c, PTK_ERR_STATE, "some grains have no pattern");
  if (need_frames && !(c->loaded[0] && c->loaded[1])) return fail(c, PTK_ERR_STATE, "both frames must be loaded");
  return PTK_OK;
}

// Enqueue helpers (no synchronisation; usable inside stream capture).
int enqueue_precompute(ptk_ctx* c, cudaStream_t s) {
  launch_precompute(c->g, frame(c, c->ref_slot), s);
  c->launches += 1;
  return PTK_OK;
}

struct SearchGeom {
  int nrot, nu, nv, tiles_u, tiles_v;
  size_t smem;
  int grid;
  size_t items;
  bool tiled;  // register-tiled exact kernel (else the direct one)
  bool bf16;   // BF16 tensor-core candidate search + exact rescoring
};

int search_geometry(ptk_ctx* c, int level, SearchGeom* sg, bool allow_bf16 = true) {
  const ptk_zone& z = c->cfg.zone[level];
  sg->nrot = (int)c->steps[level].size();
  sg->nu = z.left + z.right + 1;
  sg->nv = z.up + z.down + 1;
  sg->tiles_u = (sg->nu + kTileU - 1) / kTileU;
  sg->tiles_v = (sg->nv + kTileV - 1) / kTileV;
  sg->items = (size_t)c->n * sg->nrot * sg->tiles_u * sg->tiles_v;
  if (sg->items > (size_t)INT32_MAX) return fail(c, PTK_ERR_LIMIT, "too many search work items");
  // The BF16 form covers footprints up to 95 px and 32 rotation steps; other
  // geometries take the exact kernels (same results, exact ranking).
  sg->bf16 = allow_bf16 && c->cfg.search_method == PTK_SEARCH_BF16 && bf16_supported(c->max_R, sg->nrot, c->max_dup);
  if (sg->bf16) {
    prepare_search_bf16();
    sg->tiled = false;
    sg->smem = 0;
    sg->grid = c->num_sms;  // one CTA per SM: the whole tensor memory holds both accumulators
    sg->items = (size_t)c->n * sg->tiles_u * sg->tiles_v;
    return PTK_OK;
  }
  // The tiled kernel decodes multiplicities from its map (at most 16 points per
  // pixel): a rotated pattern stacks at most 4 distinct offsets on one pixel,
  // so patterns whose offsets repeat more than 4 times use the direct kernel.
  const size_t tsmem = search_tiled_smem(c->max_R);
  const int span = 2 * c->max_R + kTileU;
  const bool direct_ok = search_smem_bytes(c->max_P, span * span) <= 227 * 1024;
  sg->tiled = c->cfg.search_method != PTK_SEARCH_EXACT_DIRECT && c->max_dup <= 4 && c->max_R <= 112 &&
              tsmem <= 227 * 1024 && !(level == 0 && c->tune_exact == 2 && direct_ok);
  if (sg->tiled) {
    sg->smem = tsmem;
    const int occ = search_tiled_occupancy(sg->smem, c->max_R);
    sg->grid = c->num_sms * (occ > 0 ? occ : 1);
    return PTK_OK;
  }
  sg->smem = search_smem_bytes(c->max_P, span * span);
  if (sg->smem > 227 * 1024) return fail(c, PTK_ERR_LIMIT, "pattern too large for the shared-memory search tile");
  const int occ = search_occupancy(sg->smem);
  sg->grid = c->num_sms * (occ > 0 ? occ : 1);
  return PTK_OK;
}

int ensure_best(ptk_ctx* c, size_t items) {
  if (items <= c->best_cap) return PTK_OK;
  cudaFree(c->d_best);
  c->d_best = nullptr;
  CK(cudaMalloc(&c->d_best, sizeof(SearchBest) * items));
  c->best_cap = items;
  invalidate(c);
  return PTK_OK;
}

// Per-tile buffers of the BF16 search for `items` (list entries x tiles), and
// the per-grain weight slots: footprint half-extent ceil(max |offset|) + 1 of
// each pattern and the slot offsets, laid out once per pattern set.
int ensure_bf16(ptk_ctx* c, size_t items) {
  if (c->bf_geom_dirty) {
    const int n = c->n;
    std::vector<int> half(n > 0 ? n : 1, 1);
    std::vector<size_t> wofs(n > 0 ? n : 1, 0);
    size_t total = 0;
    for (int i = 0; i < n; ++i) {
      long long m2 = 0;
      for (const short2& q : c->h_pat[i]) m2 = std::max(m2, (long long)q.x * q.x + (long long)q.y * q.y);
      half[i] = (int)std::ceil(std::sqrt((double)m2)) + 1;
      wofs[i] = total;
      total += bf16_weight_entries(half[i]);
    }
    cudaFree(c->d_bf_half);
    cudaFree(c->d_bf_wofs);
    c->d_bf_half = nullptr;
    c->d_bf_wofs = nullptr;
    CK(cudaMalloc(&c->d_bf_half, sizeof(int) * half.size()));
    CK(cudaMalloc(&c->d_bf_wofs, sizeof(size_t) * wofs.size()));
    CK(cudaMemcpyAsync(c->d_bf_half, half.data(), sizeof(int) * half.size(), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->d_bf_wofs, wofs.data(), sizeof(size_t) * wofs.size(), cudaMemcpyHostToDevice, c->stream));
    c->h_bf_half = half;
    c->h_bf_wofs = wofs;
    cudaFree(c->d_bf_rot_cs);
    c->d_bf_rot_cs = nullptr;
    CK(cudaMalloc(&c->d_bf_rot_cs, sizeof(double2) * 32 * half.size()));
    for (int l = 0; l < 3; ++l) {  // the slots move (and the grain count may change): encode the maps again
      cudaFree(c->d_bf_tmaps[l]);
      c->d_bf_tmaps[l] = nullptr;
      c->bf_tmaps_nrot[l] = 0;
    }
    const size_t bytes = std::max<size_t>(total, 1) * 16;
    if (bytes > c->bf_wslots_bytes) {
      cudaFree(c->d_bf_wslots);
      c->d_bf_wslots = nullptr;
      c->bf_wslots_bytes = 0;
      CK(cudaMalloc(&c->d_bf_wslots, bytes));
      c->bf_wslots_bytes = bytes;
      // rotation slots beyond a level's steps are copied with their block: defined contents
      CK(cudaMemsetAsync(c->d_bf_wslots, 0, bytes, c->stream));
    }
    c->bf_geom_dirty = false;
    invalidate(c);
  }
  if (items > c->bf_cap) {
    cudaFree(c->d_topk);
    cudaFree(c->d_topk_rot);
    cudaFree(c->d_tile_top);
    cudaFree(c->d_rescored);
    c->d_topk = nullptr;
    c->d_topk_rot = nullptr;
    c->d_tile_top = nullptr;
    c->d_rescored = nullptr;
    c->bf_cap = 0;
    CK(cudaMalloc(&c->d_topk, sizeof(int2) * kBf16KeepMax * items));
    CK(cudaMalloc(&c->d_topk_rot, sizeof(unsigned) * kBf16KeepMax * items));
    CK(cudaMalloc(&c->d_tile_top, sizeof(float) * items));
    CK(cudaMalloc(&c->d_rescored, sizeof(SearchBest) * kBf16KeepMax * items));
    c->bf_cap = items;
    invalidate(c);
  }
  return PTK_OK;
}

// Tensor maps of the grains' operand slots for a BF16 level (its rotation
// step count decides the slots' layout), encoded on the host when the slots
// were laid out anew or the level's step count changed.
int ensure_bf16_tmaps(ptk_ctx* c, int level, int nrot) {
  if (c->bf_tmaps_nrot[level] == nrot && c->d_bf_tmaps[level]) return PTK_OK;
  const int n = c->n > 0 ? c->n : 1;
  std::vector<CUtensorMap> maps((size_t)n);
  std::memset(static_cast<void*>(maps.data()), 0, sizeof(CUtensorMap) * maps.size());
  if (c->n > 0 && !bf16_encode_tmaps(c->h_bf_half.data(), c->h_bf_wofs.data(), c->n, c->d_bf_wslots, nrot,
                                     maps.data()))
    return fail(c, PTK_ERR_CUDA, "cuTensorMapEncodeTiled refused the BF16 operand maps");
  if (!c->d_bf_tmaps[level]) CK(cudaMalloc(&c->d_bf_tmaps[level], sizeof(CUtensorMap) * (size_t)n));
  CK(cudaMemcpyAsync(c->d_bf_tmaps[level], maps.data(), sizeof(CUtensorMap) * (size_t)n, cudaMemcpyHostToDevice, c->stream));
  c->bf_tmaps_nrot[level] = nrot;
  return PTK_OK;
}

// A BF16 level also needs the exact kernels' scratch: the grains it rejects
// are searched again exactly.
int ensure_search_scratch(ptk_ctx* c, int level, const SearchGeom& sg) {
  if (!sg.bf16) return ensure_best(c, sg.items);
  SearchGeom sx;
  int rc = search_geometry(c, level, &sx, false);
  if (rc) return rc;
  if ((rc = ensure_best(c, sx.items))) return rc;
  if ((rc = ensure_bf16(c, sg.items))) return rc;
  return ensure_bf16_tmaps(c, level, sg.nrot);
}

// Kernels one search level launches (finalizes included): BF16 weights,
// search, rescore and finalize, then the exact search and finalize of the
// grains the BF16 pass rejected.
int level_launches(const SearchGeom& sg) { return sg.bf16 ? 6 : 2; }

// frame_ready: inside a frame's graph, the event of the current frame's
// upload, waited for just before the first kernel that reads that frame.
int enqueue_search(ptk_ctx* c, int level, cudaStream_t s, cudaEvent_t* ev = nullptr,
                   cudaEvent_t frame_ready = nullptr) {
  SearchGeom sg;
  int rc = search_geometry(c, level, &sg);
  if (rc) return rc;
  SearchGeom sx = sg;  // the exact kernels' geometry (a BF16 level's re-search)
  if (sg.bf16 && (rc = search_geometry(c, level, &sx, false))) return rc;
  if ((sg.bf16 && (c->bf_cap < sg.items || c->bf_geom_dirty)) || c->best_cap < sx.items)
    return fail(c, PTK_ERR_STATE, "search scratch not prepared");
  if (level == 0) {
    launch_stage_begin(c->g, c->d_counts, s);
    c->launches += 1;
  }
  const int* list = level == 0 ? c->d_order : (level == 1 ? c->d_lists : c->d_lists + c->n);
  const int* count = c->d_counts + level;
  CK(cudaMemsetAsync(c->d_work, 0, 2 * sizeof(int), s));
  const ptk_zone& z = c->cfg.zone[level];
  FinalizeLaunch f;
  f.g = c->g;
  f.steps = c->d_steps[level];
  f.left = z.left;
  f.up = z.up;
  f.nu = sg.nu;
  f.nv = sg.nv;
  f.tiles = sg.tiles_u * sg.tiles_v;
  f.level = level;
  f.NCC_min = c->cfg.NCC_min;
  f.NCC_min_super = c->cfg.NCC_min_super;
  if (sg.bf16) {
    Bf16Launch b;
    b.g = c->g;
    b.cur = frame(c, c->cur_slot);
    b.list = list;
    b.list_count = count;
    b.work_next = c->d_work;
    b.steps = c->d_steps[level];
    b.nrot = sg.nrot;
    b.left = z.left;
    b.right = z.right;
    b.up = z.up;
    b.down = z.down;
    b.tiles_u = sg.tiles_u;
    b.tiles_v = sg.tiles_v;
    b.keep = std::min(std::max(c->cfg.topk, 1), kBf16KeepMax);
    b.max_items = (int)sg.items;
    b.half = c->d_bf_half;
    b.wofs = c->d_bf_wofs;
    b.wslots = c->d_bf_wslots;
    b.tmaps = c->d_bf_tmaps[level];
    b.rot_cs = c->d_bf_rot_cs;
    if (!b.tmaps || c->bf_tmaps_nrot[level] != sg.nrot)  // every caller prepares them first
      return fail(c, PTK_ERR_STATE, "BF16 operand tensor maps missing for this level");
    if (!c->d_frame_tmaps) return fail(c, PTK_ERR_STATE, "BF16 search: the driver's tensor-map encoder is unavailable");
    b.frame_tmaps = c->d_frame_tmaps + c->cur_slot * kBf16FrameMaps;
    b.topk = c->d_topk;
    b.topk_rot = c->d_topk_rot;
    b.tile_top = c->d_tile_top;
    b.ring = c->tune_ring > 0 && bf16_ring_ok(c->max_R, c->tune_ring) ? c->tune_ring : kBf16RingDefault;
    b.rescored = c->d_rescored;
    b.error = c->d_counts + 3;
    b.probe_wait = c->probe_wait;
    launch_search_bf16(b, sg.grid, s, ev, frame_ready);
    frame_ready = nullptr;
    // The ranking finds the exact best wherever it is a match; a grain the
    // level rejects (best below the threshold, among candidates that all
    // match poorly) is searched again exactly, so that its recorded NCC and
    // its acceptance are the exact search's.
    f.list = list;
    f.list_count = count;
    f.nrot = kBf16KeepMax;  // rescored records per tile
    f.best = c->d_rescored;
    f.redo = 1;
    f.out_list = c->d_lists + 2 * (size_t)c->n;
    f.out_count = c->d_counts + 4 + level;
    launch_finalize(f, c->n, s);
    list = f.out_list;
    count = f.out_count;
  }
  SearchLaunch p;
  p.g = c->g;
  p.cur = frame(c, c->cur_slot);
  p.list = list;
  p.list_count = count;
  p.work_next = c->d_work + 1;
  p.steps = c->d_steps[level];
  p.nrot = sx.nrot;
  p.left = z.left;
  p.right = z.right;
  p.up = z.up;
  p.down = z.down;
  p.tiles_u = sx.tiles_u;
  p.tiles_v = sx.tiles_v;
  p.best = c->d_best;
  p.max_items = (int)c->best_cap;
  if (frame_ready) cudaStreamWaitEvent(s, frame_ready, cudaEventWaitExternal);
  if (ev && !sg.bf16) cudaEventRecord(ev[0], s);
  if (sx.tiled) launch_search_tiled(p, c->max_R, sx.grid, sx.smem, s);
  else launch_search(p, sx.grid, sx.smem, s);
  if (ev && !sg.bf16) cudaEventRecord(ev[1], s);
  f.list = list;
  f.list_count = count;
  f.nrot = sx.nrot;
  f.best = c->d_best;
  f.redo = 0;
  f.out_list = level == 0 ? c->d_lists : c->d_lists + c->n;
  f.out_count = c->d_counts + (level == 0 ? 1 : 2);
  launch_finalize(f, c->n, s);
  c->launches += level_launches(sg);
  return PTK_OK;
}

int enqueue_subpixel(ptk_ctx* c, int method, cudaStream_t s) {
  if (method == PTK_SUBPIX_ADJOINT_LM) {
    if (c->cfg.image_interpolator != PTK_INTERP_CUBIC)
      return fail(c, PTK_ERR_ARG, "the adjoint LM refinement is implemented for the cubic interpolator");
    LmParams lp;
    lp.max_iter = c->cfg.lm_max_iter > 0 ? c->cfg.lm_max_iter : 30;
    lp.tol = c->cfg.lm_tol > 0.0 ? c->cfg.lm_tol : 1e-4;
    lp.iters = nullptr;
    lp.order = c->d_order;
    lp.max_r = c->max_R;
    // the cell of the integer optimum: half a pixel, half a level-0 rotation step
    lp.redo_list = c->d_lists + 3 * (size_t)c->n;
    lp.redo_count = c->d_counts + 7;
    lp.cell_px = c->cfg.lm_cell_px;
    const ptk_zone& z0 = c->cfg.zone[0];
    lp.cell_rot = (c->cfg.rotations != 0 && z0.num_rot != 0 && z0.inc_rot > 0.0 && c->cfg.lm_cell_rot > 0.0)
                      ? c->cfg.lm_cell_rot * z0.inc_rot
                      : HUGE_VAL;
    if (!(lp.cell_px > 0.0)) lp.redo_list = nullptr;  // hand-off disabled: every LM result is kept
    CK(cudaMemsetAsync(lp.redo_count, 0, sizeof(int), s));
    launch_subpix_lm(c->g, frame(c, c->cur_slot), lp, s);
    if (lp.redo_list) {  // those grains: the reference's Powell from their pixel-stage state
      launch_subpix_powell(c->g, frame(c, c->cur_slot), frame(c, c->ref_slot), subpix_params(c), c->max_P, c->max_R,
                           lp.redo_list, s, lp.redo_count);
      c->launches += 1;
    }
  } else if (method == PTK_SUBPIX_POWELL) {
    launch_subpix_powell(c->g, frame(c, c->cur_slot), frame(c, c->ref_slot), subpix_params(c), c->max_P, c->max_R,
                         c->d_order, s);
  } else {
    return fail(c, PTK_ERR_ARG, "unknown subpixel method");
  }
  c->launches += 1;
  return PTK_OK;
}

int prepare_searches(ptk_ctx* c) {
  size_t need = 0, need_bf = 0;
  for (int level = 0; level < 3; ++level) {
    if (level > c->cfg.rescue_level) break;
    SearchGeom sg;
    int rc = search_geometry(c, level, &sg);
    if (rc) return rc;
    if (sg.bf16) {
      need_bf = std::max(need_bf, sg.items);
      SearchGeom sx;  // the exact re-search of the grains a BF16 level rejects
      if ((rc = search_geometry(c, level, &sx, false))) return rc;
      need = std::max(need, sx.items);
    } else {
      need = std::max(need, sg.items);
    }
  }
  if (need_bf) {
    int rc = ensure_bf16(c, need_bf);
    if (rc) return rc;
    for (int level = 0; level < 3 && level <= c->cfg.rescue_level; ++level) {
      SearchGeom sg;
      if ((rc = search_geometry(c, level, &sg))) return rc;
      if (sg.bf16 && (rc = ensure_bf16_tmaps(c, level, sg.nrot))) return rc;
    }
  }
  return ensure_best(c, need ? need : 1);
}

// Enqueues one frame body; `swap` decided by the caller.
// Captured into the frame's graph: the reference buffer's last reader is the
// precompute (buf_free recorded after it), the current buffer's the graph's
// end.
int enqueue_frame(ptk_ctx* c, bool precompute, bool swap, cudaStream_t s) {
  int rc;
  const int ref_phys = c->ref_slot, cur_phys = c->cur_slot;
  if (precompute) {
    if ((rc = enqueue_precompute(c, s))) return rc;
    cudaEventRecordWithFlags(c->buf_free[ref_phys], s, cudaEventRecordExternal);
  }
  if (c->cfg.rescue_level >= 0 && (rc = enqueue_search(c, 0, s, nullptr, c->buf_ready[cur_phys]))) return rc;
  if (c->cfg.rescue_level < 0) cudaStreamWaitEvent(s, c->buf_ready[cur_phys], cudaEventWaitExternal);
  if (c->cfg.rescue_level >= 1 && (rc = enqueue_search(c, 1, s))) return rc;
  if (c->cfg.rescue_level >= 2 && (rc = enqueue_search(c, 2, s))) return rc;
  if (c->cfg.subpixel && (rc = enqueue_subpixel(c, c->cfg.subpix_method, s))) return rc;
  launch_end_frame(c->g, swap ? 1 : 0, s);
  c->launches += 1;
  cudaEventRecordWithFlags(c->buf_free[cur_phys], s, cudaEventRecordExternal);
  return PTK_OK;
}

}  // namespace

// ===========================================================================
extern "C" {

int ptk_config_default(ptk_config* cfg) {
  if (!cfg) return fail(nullptr, PTK_ERR_ARG, "null config");
  std::memset(cfg, 0, sizeof(*cfg));
  cfg->rescue_level = 2;
  cfg->NCC_min = 0.7;
  cfg->NCC_min_super = 0.5;
  cfg->subpixel = 1;
  cfg->subpix_tol = 1e-8;
  cfg->initial_direction[0] = cfg->initial_direction[1] = cfg->initial_direction[2] = 0.01;
  cfg->image_interpolator = PTK_INTERP_CUBIC;
  cfg->overflow_stiffness = 0.0;
  cfg->subpix_displacement_max = 3.0;
  cfg->rotations = 1;
  for (int l = 0; l < 3; ++l) {
    cfg->zone[l].inc_rot = 1.0;
    cfg->zone[l].num_rot = 0;
  }
  cfg->iraz = 0;
  cfg->subpix_method = PTK_SUBPIX_POWELL;
  cfg->search_method = PTK_SEARCH_EXACT;
  cfg->topk = 8;
  cfg->lm_max_iter = 30;
  cfg->lm_tol = 1e-4;
  cfg->autotune = 0;
  cfg->lm_cell_px = 0.0;
  cfg->lm_cell_rot = 0.0;
  return PTK_OK;
}

int ptk_create(ptk_ctx** out, const ptk_config* cfg) {
  if (!out || !cfg) return fail(nullptr, PTK_ERR_ARG, "null argument");
  *out = nullptr;
  if (cfg->dimx < 4 || cfg->dimy < 4 || cfg->dimx > 65535 || cfg->dimy > 65535)
    return fail(nullptr, PTK_ERR_ARG, "frame size must be within 4..65535 pixels");
  ptk_ctx* c = new ptk_ctx();
  c->cfg = *cfg;
  auto bail = [&](int rc) {
    g_static_error = c->err;
    ptk_destroy(c);
    return rc;
  };
  cudaError_t e = cudaGetDevice(&c->device);
  if (e != cudaSuccess) return bail(cuda_fail(c, e, "cudaGetDevice"));
  cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, c->device);
  e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) return bail(cuda_fail(c, e, "cudaStreamCreate"));
  e = cudaStreamCreateWithFlags(&c->cap_stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) return bail(cuda_fail(c, e, "cudaStreamCreate"));
  for (int p = 0; p < kFrameBufs && e == cudaSuccess; ++p) {
    e = cudaStreamCreateWithFlags(&c->copy_stream[p], cudaStreamNonBlocking);
    if (e != cudaSuccess) return bail(cuda_fail(c, e, "cudaStreamCreate"));
    e = cudaEventCreateWithFlags(&c->buf_ready[p], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->buf_free[p], cudaEventDisableTiming);
  }
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->main_mark, cudaEventDisableTiming);
  if (e != cudaSuccess) return bail(cuda_fail(c, e, "cudaEventCreate"));
  c->stream = c->own_stream;
  // rows of whole 16-byte units as they are (host rows and device rows then
  // coincide and an upload is one contiguous copy), else padded to 64 pixels
  c->pitch = cfg->dimx % 16 == 0 ? cfg->dimx : (cfg->dimx + 63) & ~63;
  const size_t bytes = (size_t)c->pitch * cfg->dimy * sizeof(uint16_t);
  for (int k = 0; k < kFrameBufs; ++k) {
    e = cudaMalloc(&c->d_img[k], bytes);
    if (e != cudaSuccess) return bail(cuda_fail(c, e, "cudaMalloc(frame)"));
    e = cudaMemsetAsync(c->d_img[k], 0, bytes, c->stream);
    if (e != cudaSuccess) return bail(cuda_fail(c, e, "cudaMemsetAsync(frame)"));
  }
  // no work has read the buffers yet (the zeroing above is finished): an
  // upload into any of them need not wait
  e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return bail(cuda_fail(c, e, "cudaStreamSynchronize"));
  for (int k = 0; k < kFrameBufs; ++k) c->free_valid[k] = true;
  {  // the BF16 search's tensor maps of the frame buffers (left unset without the driver's encoder)
    CUtensorMap h[kFrameBufs * kBf16FrameMaps];
    bool ok = true;
    for (int k = 0; k < kFrameBufs && ok; ++k)
      ok = bf16_encode_frame_tmaps(c->d_img[k], cfg->dimx, cfg->dimy, c->pitch, h + k * kBf16FrameMaps);
    if (ok) {
      e = cudaMalloc(&c->d_frame_tmaps, sizeof(h));
      if (e != cudaSuccess) return bail(cuda_fail(c, e, "cudaMalloc(frame maps)"));
      e = cudaMemcpyAsync(c->d_frame_tmaps, h, sizeof(h), cudaMemcpyHostToDevice, c->stream);
      if (e != cudaSuccess) return bail(cuda_fail(c, e, "cudaMemcpy(frame maps)"));
    }
  }
  // counts: [0] grains, [1] rescue list, [2] super-rescue list, [3] error flag,
  // [4 + level] exact re-search list of a BF16 level
  e = cudaMalloc(&c->d_counts, 8 * sizeof(int));
  if (e != cudaSuccess) return bail(cuda_fail(c, e, "cudaMalloc(counts)"));
  // (on the context stream: the legacy stream does not order with it)
  e = cudaMemsetAsync(c->d_counts, 0, 8 * sizeof(int), c->stream);
  if (e != cudaSuccess) return bail(cuda_fail(c, e, "cudaMemsetAsync(counts)"));
  e = cudaMalloc(&c->d_work, 2 * sizeof(int));  // work-queue heads of the BF16 and exact kernels
  if (e != cudaSuccess) return bail(cuda_fail(c, e, "cudaMalloc(work)"));
  for (int l = 0; l < 3; ++l) {
    int rc = build_steps(c, l);
    if (rc) return bail(rc);
  }
  e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return bail(cuda_fail(c, e, "cudaStreamSynchronize"));
  *out = c;
  return PTK_OK;
}

int ptk_destroy(ptk_ctx* c) {
  if (!c) return PTK_OK;
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (int p = 0; p < kFrameBufs; ++p)
    if (c->copy_stream[p]) cudaStreamSynchronize(c->copy_stream[p]);
  drop_graphs(c);
  for (int k = 0; k < kFrameBufs; ++k) cudaFree(c->d_img[k]);
  cudaFree(c->d_tmp);
  cudaFree(c->d_u8);
  cudaFree(c->d_raw);
  cudaFree(c->d_minmax);
  cudaFree(c->d_block);
  cudaFree(c->d_snap);
  if (c->h_stage) cudaFreeHost(c->h_stage);
  cudaFree(c->d_pstart);
  cudaFree(c->d_pat);
  cudaFree(c->d_pat0);
  cudaFree(c->d_w0);
  cudaFree(c->d_order);
  for (int l = 0; l < 3; ++l) cudaFree(c->d_steps[l]);
  cudaFree(c->d_counts);
  cudaFree(c->d_lists);
  cudaFree(c->d_work);
  cudaFree(c->d_best);
  cudaFree(c->d_bf_half);
  cudaFree(c->d_bf_wofs);
  cudaFree(c->d_bf_wslots);
  for (int l = 0; l < 3; ++l) cudaFree(c->d_bf_tmaps[l]);
  cudaFree(c->d_bf_rot_cs);
  cudaFree(c->d_frame_tmaps);
  cudaFree(c->d_topk);
  cudaFree(c->d_topk_rot);
  cudaFree(c->d_tile_top);
  cudaFree(c->d_rescored);
  cudaFree(c->d_map);
  cudaFree(c->d_X);
  cudaFree(c->d_f);
  cudaFree(c->d_gr);
  if (c->own_stream) cudaStreamDestroy(c->own_stream);
  if (c->cap_stream) cudaStreamDestroy(c->cap_stream);
  for (int p = 0; p < kFrameBufs; ++p) {
    if (c->copy_stream[p]) cudaStreamDestroy(c->copy_stream[p]);
    if (c->buf_ready[p]) cudaEventDestroy(c->buf_ready[p]);
    if (c->buf_free[p]) cudaEventDestroy(c->buf_free[p]);
  }
  if (c->main_mark) cudaEventDestroy(c->main_mark);
  delete c;
  return PTK_OK;
}

int ptk_set_config(ptk_ctx* c, const ptk_config* cfg) {
  if (!c || !cfg) return fail(c, PTK_ERR_ARG, "null argument");
  if (cfg->dimx != c->cfg.dimx || cfg->dimy != c->cfg.dimy)
    return fail(c, PTK_ERR_ARG, "frame size cannot change on a context");
  if (cfg->rescue_level < -1 || cfg->rescue_level > 2) return fail(c, PTK_ERR_ARG, "rescue_level must be -1..2");
  const ptk_zone &z0 = cfg->zone[0], &o0 = c->cfg.zone[0];
  if (cfg->search_method != c->cfg.search_method || z0.left != o0.left || z0.right != o0.right ||
      z0.up != o0.up || z0.down != o0.down || z0.num_rot != o0.num_rot || z0.inc_rot != o0.inc_rot) {
    c->tune_ring = c->tune_exact = 0;  // another form or level-0 zone is tuned afresh
    c->tuned = false;
  }
  c->cfg = *cfg;
  for (int l = 0; l < 3; ++l) {
    int rc = build_steps(c, l);
    if (rc) return rc;
  }
  invalidate(c);
  return PTK_OK;
}

int ptk_set_search_zone(ptk_ctx* c, int level, const ptk_zone* z) {
  if (!c || !z || level < 0 || level > 2) return fail(c, PTK_ERR_ARG, "bad search zone arguments");
  const ptk_zone old = c->cfg.zone[level];
  c->cfg.zone[level] = *z;
  int rc = build_steps(c, level);
  if (rc) c->cfg.zone[level] = old;
  return rc;
}

int ptk_set_grains(ptk_ctx* c, const ptk_grain* grains, int n) {
  if (!c || (n > 0 && !grains) || n < 0) return fail(c, PTK_ERR_ARG, "bad grain arguments");
  CK(cudaStreamSynchronize(c->stream));
  all_released(c);
  const bool resized = n != c->n;
  if (resized) {
    cudaFree(c->d_block);
    cudaFree(c->d_snap);
    cudaFree(c->d_lists);
    c->d_block = nullptr;
    c->d_snap = nullptr;
    c->d_lists = nullptr;
    c->n = n;
    BlockLayout L(n);
    CK(cudaMalloc(&c->d_block, L.total));
    CK(cudaMalloc(&c->d_lists, sizeof(int) * 4 * (n > 0 ? n : 1)));
    c->h_pat.assign(n, std::vector<short2>());
    c->patterns_ok = false;
    cudaFree(c->d_best);
    c->d_best = nullptr;
    c->best_cap = 0;
  }
  BlockLayout L(n);
  int rc = ensure_stage(c, L.total);
  if (rc) return rc;
  char* h = static_cast<char*>(c->h_stage);
  std::memset(h, 0, L.total);
  const size_t nn = (size_t)(n > 0 ? n : 1);
  auto D = [&](int k) { return reinterpret_cast<double*>(h + L.d_off + k * nn * 8); };
  auto I = [&](int k) { return reinterpret_cast<int*>(h + L.i_off + k * nn * 4); };
  auto B = [&](int k) { return reinterpret_cast<uint8_t*>(h + L.b_off + k * nn); };
  c->h_radius.resize(n);
  for (int i = 0; i < n; ++i) {
    const ptk_grain& s = grains[i];
    I(I_REFX)[i] = s.refcoord_xpix;
    I(I_REFY)[i] = s.refcoord_ypix;
    D(D_REFROT)[i] = s.refrot;
    D(D_RADIUS)[i] = s.radius_pix;
    D(D_DX)[i] = s.dx;
    D(D_DY)[i] = s.dy;
    D(D_DROT)[i] = s.drot;
    D(D_DXP)[i] = s.dx;
    D(D_DYP)[i] = s.dy;
    D(D_DROTP)[i] = s.drot;
    D(D_UPIX)[i] = s.upix;
    D(D_VPIX)[i] = s.vpix;
    D(D_ROTINC)[i] = s.rot_inc;
    D(D_NCC)[i] = s.NCC;
    D(D_NCCR)[i] = s.NCC_rescue;
    D(D_NCCS)[i] = s.NCC_subpix;
    B(B_MASKED)[i] = s.masked ? 1 : 0;
    c->h_radius[i] = s.radius_pix;
  }
  // the next call that touches the staging buffer synchronises the stream first
  if (n) CK(cudaMemcpyAsync(c->d_block, h, L.total, cudaMemcpyHostToDevice, c->stream));
  bind_grains(c);
  c->need_precompute = true;
  // the frame graphs hold the grain block's addresses, which change only with
  // the grain count: new values for as many grains keep them
  if (resized) invalidate(c);
  return PTK_OK;
}

int ptk_get_grains(ptk_ctx* c, ptk_grain* out, int n) {
  if (!c || (n > 0 && !out)) return fail(c, PTK_ERR_ARG, "bad arguments");
  if (n != c->n) return fail(c, PTK_ERR_ARG, "grain count mismatch");
  if (n == 0) return PTK_OK;
  BlockLayout L(n);
  CK(cudaStreamSynchronize(c->stream));
  all_released(c);
  int rc = ensure_stage(c, L.total);
  if (rc) return rc;
  const char* h = static_cast<const char*>(c->h_stage);
  CK(cudaMemcpyAsync(c->h_stage, c->d_block, L.total, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  const size_t nn = (size_t)n;
  auto D = [&](int k) { return reinterpret_cast<const double*>(h + L.d_off + k * nn * 8); };
  auto I = [&](int k) { return reinterpret_cast<const int*>(h + L.i_off + k * nn * 4); };
  auto B = [&](int k) { return reinterpret_cast<const uint8_t*>(h + L.b_off + k * nn); };
  for (int i = 0; i < n; ++i) {
    ptk_grain& s = out[i];
    std::memset(&s, 0, sizeof(s));
    s.refcoord_xpix = I(I_REFX)[i];
    s.refcoord_ypix = I(I_REFY)[i];
    s.refrot = D(D_REFROT)[i];
    s.radius_pix = D(D_RADIUS)[i];
    s.dx = D(D_DX)[i];
    s.dy = D(D_DY)[i];
    s.drot = D(D_DROT)[i];
    s.upix = D(D_UPIX)[i];
    s.vpix = D(D_VPIX)[i];
    s.rot_inc = D(D_ROTINC)[i];
    s.NCC = D(D_NCC)[i];
    s.NCC_rescue = D(D_NCCR)[i];
    s.NCC_subpix = D(D_NCCS)[i];
    s.masked = B(B_MASKED)[i];
    s.status = B(B_STATUS)[i];
  }
  return PTK_OK;
}

int ptk_snapshot_grains(ptk_ctx* c) {
  if (!c) return fail(c, PTK_ERR_ARG, "null context");
  if (c->n <= 0) return fail(c, PTK_ERR_STATE, "no grains set");
  BlockLayout L(c->n);
  if (!c->d_snap) CK(cudaMalloc(&c->d_snap, L.total));
  CK(cudaMemcpyAsync(c->d_snap, c->d_block, L.total, cudaMemcpyDeviceToDevice, c->stream));
  return PTK_OK;
}

int ptk_restore_grains(ptk_ctx* c) {
  if (!c) return fail(c, PTK_ERR_ARG, "null context");
  if (!c->d_snap) return fail(c, PTK_ERR_STATE, "no grain snapshot");
  BlockLayout L(c->n);
  CK(cudaMemcpyAsync(c->d_block, c->d_snap, L.total, cudaMemcpyDeviceToDevice, c->stream));
  c->need_precompute = true;
  return PTK_OK;
}

int ptk_set_patterns(ptk_ctx* c, const int32_t* xy, const int64_t* starts, int n) {
  if (!c || n != c->n || (n > 0 && (!xy || !starts))) return fail(c, PTK_ERR_ARG, "bad pattern arguments");
  CK(cudaStreamSynchronize(c->stream));
  for (int i = 0; i < n; ++i) {
    if (starts[i + 1] < starts[i]) return fail(c, PTK_ERR_ARG, "pattern starts must be non-decreasing");
    std::vector<short2>& v = c->h_pat[i];
    v.clear();
    for (int64_t k = starts[i]; k < starts[i + 1]; ++k) {
      const int32_t x = xy[2 * k], y = xy[2 * k + 1];
      if (x < -4096 || x > 4096 || y < -4096 || y > 4096) return fail(c, PTK_ERR_LIMIT, "pattern offset beyond 4096 px");
      v.push_back(make_short2((short)x, (short)y));
    }
  }
  return upload_patterns(c);
}

int ptk_make_patterns(ptk_ctx* c, int kind, double a, double b, double target_radius) {
  if (!c) return fail(c, PTK_ERR_ARG, "null context");
  if (c->n <= 0) return fail(c, PTK_ERR_STATE, "set grains before patterns");
  CK(cudaStreamSynchronize(c->stream));
  for (int i = 0; i < c->n; ++i) {
    if (!(target_radius < 0.0 || c->h_radius[i] == target_radius)) continue;
    std::vector<short2>& v = c->h_pat[i];
    v.clear();
    int r_in = 0, r_out = 0, hw = 0, hh = 0;
    int k = kind;
    if (kind == PTK_PATTERN_GRAIN_DIAMETER) {
      // src/p-tracker.cpp:1656-1666
      int radius = (int)(c->h_radius[i] * a);
      if (radius < b) radius = (int)b;
      r_out = radius;
      k = PTK_PATTERN_CIRC;
    } else if (kind == PTK_PATTERN_CIRC) {
      r_out = (int)a;
    } else if (kind == PTK_PATTERN_RING) {
      r_in = (int)a;
      r_out = (int)b;
    } else if (kind == PTK_PATTERN_RECT) {
      hw = (int)a;
      hh = (int)b;
    } else {
      return fail(c, PTK_ERR_ARG, "unknown pattern kind");
    }
    if (r_out > 64 || hw > 64 || hh > 64) return fail(c, PTK_ERR_LIMIT, "pattern radius above 64 px");
    if (k == PTK_PATTERN_RECT) {  // src/p-tracker.cpp:1369-1384
      for (int dy = -hh; dy <= hh; ++dy)
        for (int dx = -hw; dx <= hw; ++dx) v.push_back(make_short2((short)dx, (short)dy));
    } else {  // circ / ring, src/p-tracker.cpp:1386-1442
      for (int dy = -r_out; dy <= r_out; ++dy)
        for (int dx = -r_out; dx <= r_out; ++dx) {
          const double dst = std::sqrt((double)dx * (double)dx + (double)dy * (double)dy);
          const bool in = k == PTK_PATTERN_CIRC ? dst <= (double)r_out
                                                 : (dst <= (double)r_out && dst >= (double)r_in);
          if (in) v.push_back(make_short2((short)dx, (short)dy));
        }
    }
  }
  return upload_patterns(c);
}

int ptk_pattern_size(ptk_ctx* c, int grain, int* npts) {
  if (!c || !npts || grain < 0 || grain >= c->n) return fail(c, PTK_ERR_ARG, "bad arguments");
  *npts = (int)c->h_pat[grain].size();
  return PTK_OK;
}

int ptk_load_frame(ptk_ctx* c, int slot, const void* pix, int dimx, int dimy, int bpp, size_t pitch_bytes) {
  if (!c || !pix || slot < 0 || slot > 1) return fail(c, PTK_ERR_ARG, "bad frame arguments");
  if (dimx != c->cfg.dimx || dimy != c->cfg.dimy) return fail(c, PTK_ERR_ARG, "frame size differs from the context");
  if (bpp != 1 && bpp != 2) return fail(c, PTK_ERR_ARG, "bytes_per_px must be 1 or 2");
  if (pitch_bytes < (size_t)dimx * bpp) return fail(c, PTK_ERR_ARG, "pitch smaller than a row");
  // The upload waits for the buffer's last reader: a frame graph's record of
  // buf_free while that is valid, else all queued work.  Of the slot's buffer
  // and the spare, the one released first takes it: one the latest graph did
  // not read, then one it released after its precompute, then one it
  // released at its end, then one waiting for all queued work.
  auto release_rank = [&](int b) {
    if (!c->free_valid[b]) return 3;
    if (c->used_by_graph[b] < c->graph_seq) return 0;
    return c->released_early[b] ? 1 : 2;
  };
  int& slot_buf = slot == 0 ? c->ref_slot : c->cur_slot;
  if (release_rank(c->spare_buf) < release_rank(slot_buf)) std::swap(slot_buf, c->spare_buf);
  const int phys = slot_buf;
  const bool after_graph = c->free_valid[phys];
  cudaStream_t cs = c->copy_stream[phys];
  if (after_graph) {
    CK(cudaStreamWaitEvent(cs, c->buf_free[phys], 0));
  } else {
    CK(cudaEventRecord(c->main_mark, c->stream));
    CK(cudaStreamWaitEvent(cs, c->main_mark, 0));
  }
  if (!c->d_u8 && bpp == 1) CK(cudaMalloc(&c->d_u8, (size_t)c->pitch * dimy));
  if (bpp == 2) {
    CK(cudaMemcpy2DAsync(c->d_img[phys], (size_t)c->pitch * 2, pix, pitch_bytes, (size_t)dimx * 2, dimy,
                         cudaMemcpyHostToDevice, cs));
  } else {
    // the 8-bit staging buffer is shared: after the other buffers' last uploads
    for (int b = 0; b < kFrameBufs; ++b)
      if (b != phys) CK(cudaStreamWaitEvent(cs, c->buf_ready[b], 0));
    CK(cudaMemcpy2DAsync(c->d_u8, (size_t)c->pitch, pix, pitch_bytes, (size_t)dimx, dimy, cudaMemcpyHostToDevice,
                         cs));
    launch_widen_u8(c->d_u8, (size_t)c->pitch, c->d_img[phys], c->pitch, dimx, dimy, cs);
    c->launches += 1;
  }
  CK(cudaEventRecord(c->buf_ready[phys], cs));
  c->ready_pending[phys] = true;
  c->loaded[slot] = true;
  if (slot == 0) c->need_precompute = true;
  return PTK_OK;
}

int ptk_host_alloc(void** ptr, size_t bytes) {
  if (!ptr || bytes == 0) return fail(nullptr, PTK_ERR_ARG, "bad host allocation arguments");
  *ptr = nullptr;
  const cudaError_t e = cudaMallocHost(ptr, bytes);
  if (e != cudaSuccess) {
    *ptr = nullptr;
    return fail(nullptr, PTK_ERR_CUDA, std::string("cudaMallocHost: ") + cudaGetErrorString(e));
  }
  return PTK_OK;
}

int ptk_host_free(void* ptr) {
  if (ptr && cudaFreeHost(ptr) != cudaSuccess) return fail(nullptr, PTK_ERR_CUDA, "cudaFreeHost");
  return PTK_OK;
}

int ptk_load_frame_device(ptk_ctx* c, int slot, const void* dev_pix, size_t pitch_bytes) {
  if (!c || !dev_pix || slot < 0 || slot > 1) return fail(c, PTK_ERR_ARG, "bad frame arguments");
  if (pitch_bytes < (size_t)c->cfg.dimx * 2) return fail(c, PTK_ERR_ARG, "pitch smaller than a row");
  sync_cur(c);
  const int phys = slot == 0 ? c->ref_slot : c->cur_slot;
  CK(cudaMemcpy2DAsync(c->d_img[phys], (size_t)c->pitch * 2, dev_pix, pitch_bytes, (size_t)c->cfg.dimx * 2,
                       c->cfg.dimy, cudaMemcpyDeviceToDevice, c->stream));
  c->loaded[slot] = true;
  if (slot == 0) c->need_precompute = true;
  return PTK_OK;
}

static int load_frame_raw(ptk_ctx* c, int slot, const uint16_t* raw, bool raw_on_device, int raw_width,
                          int raw_height, int left, int top, int mode, int rescale, uint16_t* min_max) {
  if (!c || !raw || slot < 0 || slot > 1) return fail(c, PTK_ERR_ARG, "bad frame arguments");
  if (mode != -1 && mode != -2 && mode != -20)
    return fail(c, PTK_ERR_ARG, "DemosaicModel must be -1, -2 or -20 (libraw's own modes need libraw)");
  if (raw_width < 1 || raw_height < 1 || left < 0 || top < 0) return fail(c, PTK_ERR_ARG, "bad mosaic geometry");
  const long long n = (long long)raw_width * raw_height;
  const int lo = raw_stencil_lo(mode), hi = raw_stencil_hi(mode);
  const long long first = (long long)(left + lo) + (long long)raw_width * (top + lo);
  const long long last =
      (long long)(left + c->cfg.dimx - 1 + hi) + (long long)raw_width * (top + c->cfg.dimy - 1 + hi);
  if (first < 0 || last >= n)
    return fail(c, PTK_ERR_ARG, "the demosaic stencil reaches outside the raw mosaic (check margins and sizes)");
  if (!c->d_minmax) CK(cudaMalloc(&c->d_minmax, 2 * sizeof(unsigned)));
  sync_cur(c);
  const uint16_t* src = raw;
  if (!raw_on_device) {
    if ((size_t)n > c->raw_cap) {
      cudaFree(c->d_raw);
      c->d_raw = nullptr;
      c->raw_cap = 0;
      CK(cudaMalloc(&c->d_raw, (size_t)n * 2));
      c->raw_cap = (size_t)n;
    }
    CK(cudaMemcpyAsync(c->d_raw, raw, (size_t)n * 2, cudaMemcpyHostToDevice, c->stream));
    src = c->d_raw;
  }
  const int phys = slot == 0 ? c->ref_slot : c->cur_slot;
  launch_raw_demosaic(src, raw_width, left, top, mode, rescale, c->d_img[phys], c->pitch, c->cfg.dimx, c->cfg.dimy,
                      c->d_minmax, c->num_sms, c->stream);
  CK(cudaGetLastError());
  c->launches += rescale ? 2 : 1;
  if (min_max) {
    unsigned mm[2];
    CK(cudaMemcpyAsync(mm, c->d_minmax, sizeof(mm), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    min_max[0] = (uint16_t)mm[0];
    min_max[1] = (uint16_t)mm[1];
  }
  c->loaded[slot] = true;
  if (slot == 0) c->need_precompute = true;
  return PTK_OK;
}

int ptk_load_frame_raw(ptk_ctx* c, int slot, const uint16_t* raw, int raw_width, int raw_height, int left_margin,
                       int top_margin, int mode, int rescale, uint16_t* min_max) {
  return load_frame_raw(c, slot, raw, false, raw_width, raw_height, left_margin, top_margin, mode, rescale, min_max);
}

int ptk_load_frame_raw_device(ptk_ctx* c, int slot, const uint16_t* dev_raw, int raw_width, int raw_height,
                              int left_margin, int top_margin, int mode, int rescale, uint16_t* min_max) {
  return load_frame_raw(c, slot, dev_raw, true, raw_width, raw_height, left_margin, top_margin, mode, rescale,
                        min_max);
}

int ptk_read_frame(ptk_ctx* c, int slot, uint16_t* out) {
  if (!c || !out || slot < 0 || slot > 1) return fail(c, PTK_ERR_ARG, "bad arguments");
  sync_cur(c);
  const int phys = slot == 0 ? c->ref_slot : c->cur_slot;
  CK(cudaMemcpy2DAsync(out, (size_t)c->cfg.dimx * 2, c->d_img[phys], (size_t)c->pitch * 2, (size_t)c->cfg.dimx * 2,
                       c->cfg.dimy, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return PTK_OK;
}

int ptk_precompute(ptk_ctx* c) {
  if (!c) return fail(c, PTK_ERR_ARG, "null context");
  int rc = check_ready(c, false);
  if (rc) return rc;
  if (!c->loaded[0]) return fail(c, PTK_ERR_STATE, "reference frame not loaded");
  sync_cur(c);  // the reference frame's upload first
  rc = enqueue_precompute(c, c->stream);
  if (rc) return rc;
  c->need_precompute = false;
  CK(cudaGetLastError());
  return PTK_OK;
}

int ptk_search(ptk_ctx* c, int level) {
  if (!c || level < 0 || level > 2) return fail(c, PTK_ERR_ARG, "bad search level");
  int rc = check_ready(c, true);
  if (rc) return rc;
  sync_cur(c);
  if (c->need_precompute && (rc = ptk_precompute(c))) return rc;
  SearchGeom sg;
  if ((rc = search_geometry(c, level, &sg))) return rc;
  if ((rc = ensure_search_scratch(c, level, sg))) return rc;
  if ((rc = enqueue_search(c, level, c->stream))) return rc;
  CK(cudaGetLastError());
  return PTK_OK;
}

int ptk_search_timed(ptk_ctx* c, int level, float* kernel_ms, int max_kernels, int* n_kernels) {
  if (!c || level < 0 || level > 2 || !n_kernels || (max_kernels > 0 && !kernel_ms))
    return fail(c, PTK_ERR_ARG, "bad argument");
  int rc = check_ready(c, true);
  if (rc) return rc;
  sync_cur(c);
  if (c->need_precompute && (rc = ptk_precompute(c))) return rc;
  SearchGeom sg;
  if ((rc = search_geometry(c, level, &sg))) return rc;
  if ((rc = ensure_search_scratch(c, level, sg))) return rc;
  cudaEvent_t ev[5] = {};
  const int nev = sg.bf16 ? 4 : 2;
  for (int k = 0; k < nev; ++k) {
    cudaError_t e = cudaEventCreate(&ev[k]);
    if (e != cudaSuccess) {
      for (int j = 0; j < k; ++j) cudaEventDestroy(ev[j]);
      return cuda_fail(c, e, "cudaEventCreate");
    }
  }
  rc = enqueue_search(c, level, c->stream, ev);
  cudaError_t e = rc ? cudaSuccess : cudaStreamSynchronize(c->stream);
  *n_kernels = nev - 1;
  for (int k = 0; !rc && e == cudaSuccess && k + 1 < nev; ++k) {
    float ms = 0.0f;
    e = cudaEventElapsedTime(&ms, ev[k], ev[k + 1]);
    if (k < max_kernels) kernel_ms[k] = ms;
  }
  for (int k = 0; k < nev; ++k) cudaEventDestroy(ev[k]);
  if (rc) return rc;
  if (e != cudaSuccess) return cuda_fail(c, e, "search timing");
  return PTK_OK;
}

// The autotune cache's key: GPU model, search method and the workload's shape.
static int tune_signature(ptk_ctx* c, const SearchGeom& sg, std::string* out) {
  int dev = 0;
  cudaDeviceProp prop{};
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaGetDeviceProperties(&prop, dev);
  if (e != cudaSuccess) return cuda_fail(c, e, "cudaGetDeviceProperties");
  // grains per 8-px class of pattern extent (ceil of the largest offset norm)
  std::vector<int> hist;
  for (const auto& pat : c->h_pat) {
    double m = 0.0;
    for (const short2& q : pat) m = std::max(m, std::sqrt((double)q.x * q.x + (double)q.y * q.y));
    const size_t k = (size_t)std::ceil(m) / 8;
    if (hist.size() <= k) hist.resize(k + 1, 0);
    ++hist[k];
  }
  std::string name(prop.name);
  for (char& ch : name)
    if ((unsigned char)ch < 0x20 || (unsigned char)ch >= 0x7F || ch == '|') ch = '_';
  const ptk_zone& z = c->cfg.zone[0];
  char b[256];
  snprintf(b, sizeof b, "sm_%d%d %s x%d|%s|frame %dx%d|grains %d|rmax %d|zone %d,%d,%d,%d|nrot %d|topk %d|r8", prop.major,
           prop.minor, name.c_str(), prop.multiProcessorCount, sg.bf16 ? "bf16" : "exact", c->cfg.dimx, c->cfg.dimy,
           c->n, c->max_R, z.left, z.right, z.up, z.down, sg.nrot, c->cfg.topk);
  std::string sig(b);
  for (size_t k = 0; k < hist.size(); ++k) sig += (k ? "," : " ") + std::to_string(hist[k]);
  *out = sig;
  return PTK_OK;
}

int ptk_set_tune_cache(ptk_ctx* c, const char* path) {
  if (!c) return fail(c, PTK_ERR_ARG, "null context");
  c->tune_cache = path ? path : "";
  return PTK_OK;
}

int ptk_tune_signature(ptk_ctx* c, char* buf, int32_t cap) {
  if (!c || !buf || cap < 1) return fail(c, PTK_ERR_ARG, "ptk_tune_signature: null context or buffer");
  int rc = check_ready(c, true);
  if (rc) return rc;
  SearchGeom sg;
  if ((rc = search_geometry(c, 0, &sg))) return rc;
  std::string sig;
  if ((rc = tune_signature(c, sg, &sig))) return rc;
  if ((int64_t)sig.size() + 1 > cap) return fail(c, PTK_ERR_LIMIT, "ptk_tune_signature: buffer too small");
  memcpy(buf, sig.c_str(), sig.size() + 1);
  return PTK_OK;
}

int ptk_autotune(ptk_ctx* c, ptk_tune_report* report) {
  if (!c) return fail(c, PTK_ERR_ARG, "null context");
  int rc = check_ready(c, true);
  if (rc) return rc;
  sync_cur(c);
  if (c->need_precompute && (rc = ptk_precompute(c))) return rc;
  c->tune_ring = c->tune_exact = 0;
  SearchGeom sg;
  if ((rc = search_geometry(c, 0, &sg))) return rc;
  // candidates of the level-0 search: ring depths of the BF16 kernel, or the
  // exact kernels that can hold the patterns (every candidate gives the same
  // results; only the time differs)
  std::vector<int> cand;
  const int method = sg.bf16 ? 1 : 0;
  if (sg.bf16) {
    for (int r : {2, 3, 4, 6})
      if (bf16_ring_ok(c->max_R, r)) cand.push_back(r);
  } else {
    const int span = 2 * c->max_R + kTileU;
    if (sg.tiled) cand.push_back(1);
    if (search_smem_bytes(c->max_P, span * span) <= 227 * 1024) cand.push_back(2);
  }
  if (cand.empty()) return fail(c, PTK_ERR_STATE, "no admissible search shape");
  std::string sig;
  if (!c->tune_cache.empty()) {
    if ((rc = tune_signature(c, sg, &sig))) return rc;
    int32_t found = 0, m = 0, ch = 0;
    if (ptk_tune_cache_lookup(c->tune_cache.c_str(), sig.c_str(), &found, &m, &ch) != PTK_OK)
      return fail(c, PTK_ERR_IO, "autotune cache unreadable or malformed");
    if (found && m == method && std::find(cand.begin(), cand.end(), (int)ch) != cand.end()) {
      if (method) c->tune_ring = ch;
      else c->tune_exact = ch;
      c->tuned = true;
      invalidate(c);
      if (report) {
        report->method = method;
        report->choice = ch;
        report->n = 0;  // taken from the cache, nothing timed
      }
      return PTK_OK;
    }
  }
  BlockLayout L(c->n);
  void* snap = nullptr;
  void* flush = nullptr;  // written before every run: each starts with the L2 state a frame sees
  const size_t flush_bytes = (size_t)256 << 20;
  cudaEvent_t ev[2] = {};
  auto cleanup = [&]() {
    if (snap) cudaFree(snap);
    if (flush) cudaFree(flush);
    for (cudaEvent_t e : ev)
      if (e) cudaEventDestroy(e);
  };
  if (cudaMalloc(&snap, L.total) != cudaSuccess || cudaEventCreate(&ev[0]) != cudaSuccess ||
      cudaEventCreate(&ev[1]) != cudaSuccess) {
    cleanup();
    return fail(c, PTK_ERR_CUDA, "autotune scratch");
  }
  if (cudaMalloc(&flush, flush_bytes) != cudaSuccess) {
    flush = nullptr;  // no room: the runs go without the flush
    cudaGetLastError();
  }
  cudaMemcpyAsync(snap, c->d_block, L.total, cudaMemcpyDeviceToDevice, c->stream);
  std::vector<float> best((size_t)cand.size(), 1e30f);
  cudaError_t e = cudaSuccess;
  for (size_t k = 0; k < cand.size() && !rc && e == cudaSuccess; ++k) {
    if (method) c->tune_ring = cand[k];
    else c->tune_exact = cand[k];
    SearchGeom g;
    if ((rc = search_geometry(c, 0, &g)) || (rc = ensure_search_scratch(c, 0, g))) break;
    for (int rep = 0; rep < 5 && !rc && e == cudaSuccess; ++rep) {  // the first run is a warm-up
      cudaMemcpyAsync(c->d_block, snap, L.total, cudaMemcpyDeviceToDevice, c->stream);
      if (flush) cudaMemsetAsync(flush, rep, flush_bytes, c->stream);
      cudaEventRecord(ev[0], c->stream);
      rc = enqueue_search(c, 0, c->stream);
      cudaEventRecord(ev[1], c->stream);
      e = cudaEventSynchronize(ev[1]);
      float ms = 0.0f;
      if (!rc && e == cudaSuccess) e = cudaEventElapsedTime(&ms, ev[0], ev[1]);
      if (rep > 0 && ms < best[k]) best[k] = ms;
    }
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(c->d_block, snap, L.total, cudaMemcpyDeviceToDevice, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cleanup();
  c->tune_ring = c->tune_exact = 0;
  if (rc) return rc;
  if (e != cudaSuccess) return cuda_fail(c, e, "autotune");
  // the built-in shape stays unless another is more than 2 % faster
  size_t k_best = 0;
  for (size_t k = 1; k < cand.size(); ++k)
    if (best[k] < best[k_best]) k_best = k;
  for (size_t k = 0; k < cand.size(); ++k)
    if (cand[k] == (method ? kBf16RingDefault : 1) && best[k] <= 1.02f * best[k_best]) k_best = k;
  if (method) c->tune_ring = cand[k_best];
  else c->tune_exact = cand[k_best];
  c->tuned = true;
  invalidate(c);
  if (report) {
    report->method = method;
    report->choice = cand[k_best];
    report->n = (int)std::min<size_t>(cand.size(), 8);
    for (int k = 0; k < report->n; ++k) {
      report->values[k] = cand[(size_t)k];
      report->ms[k] = best[(size_t)k];
    }
  }
  if (!c->tune_cache.empty()) {
    std::vector<int32_t> vals(cand.begin(), cand.end());
    if (ptk_tune_cache_store(c->tune_cache.c_str(), sig.c_str(), method, cand[k_best], (int32_t)cand.size(),
                             vals.data(), best.data()) != PTK_OK)
      return fail(c, PTK_ERR_IO, "autotune cache could not be written");
  }
  return PTK_OK;
}

int ptk_subpixel(ptk_ctx* c, int method) {
  if (!c) return fail(c, PTK_ERR_ARG, "null context");
  int rc = check_ready(c, true);
  if (rc) return rc;
  sync_cur(c);
  if (c->need_precompute && (rc = ptk_precompute(c))) return rc;
  if ((rc = enqueue_subpixel(c, method, c->stream))) return rc;
  CK(cudaGetLastError());
  return PTK_OK;
}

int ptk_end_frame(ptk_ctx* c, int num_image) {
  if (!c) return fail(c, PTK_ERR_ARG, "null context");
  if (c->n <= 0) return fail(c, PTK_ERR_STATE, "no grains set");
  sync_cur(c);
  const bool swap = num_image - c->iref >= c->cfg.iraz;
  launch_end_frame(c->g, swap ? 1 : 0, c->stream);
  c->launches += 1;
  CK(cudaGetLastError());
  if (swap) {
    std::swap(c->ref_slot, c->cur_slot);
    c->iref = num_image;
    c->need_precompute = true;
  }
  return PTK_OK;
}

int ptk_swap_reference(ptk_ctx* c, int num_image) {
  if (!c) return fail(c, PTK_ERR_ARG, "null context");
  const int saved = c->cfg.iraz;
  c->cfg.iraz = INT32_MIN / 2;
  int rc = ptk_end_frame(c, num_image);
  c->cfg.iraz = saved;
  return rc;
}

int ptk_set_iref(ptk_ctx* c, int iref) {
  if (!c) return fail(c, PTK_ERR_ARG, "null context");
  c->iref = iref;
  return PTK_OK;
}

int ptk_track_frame(ptk_ctx* c, int num_image) {
  if (!c) return fail(c, PTK_ERR_ARG, "null context");
  int rc = check_ready(c, true);
  if (rc) return rc;
  if (c->cfg.autotune && !c->tuned && ptk_autotune(c, nullptr) != PTK_OK) {
    c->tuned = true;  // tuning failed (e.g. no memory for its scratch): the built-in shapes track the frame
    c->tune_ring = c->tune_exact = 0;
  }
  if ((rc = prepare_searches(c))) return rc;
  if (c->graph_dirty) drop_graphs(c);
  const bool pre = c->need_precompute;
  const bool swap = num_image - c->iref >= c->cfg.iraz;
  const int key = ((c->ref_slot * kFrameBufs + c->cur_slot) * 2 + (pre ? 1 : 0)) * 2 + (swap ? 1 : 0);
  if (!c->graph[key]) {
    // all attribute and occupancy queries happen before capture
    for (int l = 0; l <= c->cfg.rescue_level && l < 3; ++l) {
      SearchGeom sg;
      if ((rc = search_geometry(c, l, &sg))) return rc;
    }
    prepare_subpix(c->max_P, c->max_R);
    const int64_t before = c->launches;
    CK(cudaStreamBeginCapture(c->cap_stream, cudaStreamCaptureModeRelaxed));
    rc = enqueue_frame(c, pre, swap, c->cap_stream);
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(c->cap_stream, &graph);
    if (rc) {
      if (graph) cudaGraphDestroy(graph);
      return rc;
    }
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaStreamEndCapture");
    e = cudaGraphInstantiate(&c->graph[key], graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaGraphInstantiate");
    c->launches = before;  // counted again at each replay below
  }
  const int ref_phys = c->ref_slot, cur_phys = c->cur_slot;
  if (c->ready_pending[ref_phys]) {  // the precompute reads the reference buffer first
    CK(cudaStreamWaitEvent(c->stream, c->buf_ready[ref_phys], 0));
    c->ready_pending[ref_phys] = false;
  }
  CK(cudaGraphLaunch(c->graph[key], c->stream));
  c->ready_pending[cur_phys] = false;  // the graph waits for it before its first kernel reading the frame
  // the graph records each buffer's release: the reference after its
  // precompute (none without one), the current one at its end
  ++c->graph_seq;
  c->used_by_graph[ref_phys] = c->used_by_graph[cur_phys] = c->graph_seq;
  c->free_valid[ref_phys] = pre;
  c->released_early[ref_phys] = pre;
  c->free_valid[cur_phys] = true;
  c->released_early[cur_phys] = false;
  // launches of one frame: precompute, stage_begin, (search, finalize) per level,
  // subpixel, end_frame
  int64_t nk = (pre ? 1 : 0) + 1;
  for (int l = 0; l <= c->cfg.rescue_level && l < 3; ++l) {
    SearchGeom sg;
    if ((rc = search_geometry(c, l, &sg))) return rc;
    nk += (l == 0 ? 1 : 0) + level_launches(sg);
  }
  if (c->cfg.subpixel) nk += 1;
  c->launches += nk;
  if (swap) {
    std::swap(c->ref_slot, c->cur_slot);
    c->iref = num_image;
    c->need_precompute = true;
  } else {
    c->need_precompute = false;
  }
  return PTK_OK;
}

int ptk_get_rescue_counts(ptk_ctx* c, int* n_rescued, int* n_super) {
  if (!c || !n_rescued || !n_super) return fail(c, PTK_ERR_ARG, "null argument");
  int h[3];
  CK(cudaMemcpyAsync(h, c->d_counts, 3 * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  *n_rescued = h[1];
  *n_super = h[2];
  return PTK_OK;
}

static int objective_common(ptk_ctx* c, const double* X3n, double* f, double* g3n) {
  if (!c || !X3n || !f) return fail(c, PTK_ERR_ARG, "null argument");
  int rc = check_ready(c, true);
  if (rc) return rc;
  sync_cur(c);
  if (g3n && c->cfg.image_interpolator != PTK_INTERP_CUBIC)
    return fail(c, PTK_ERR_ARG, "the gradient is implemented for the cubic interpolator");
  if (g3n && (size_t)c->max_P * 24 > 227 * 1024) return fail(c, PTK_ERR_LIMIT, "pattern too large for ptk_grad");
  if (c->need_precompute && (rc = ptk_precompute(c))) return rc;
  const size_t n = (size_t)c->n;
  if (!c->d_X) {
    CK(cudaMalloc(&c->d_X, sizeof(double) * 3 * n));
    CK(cudaMalloc(&c->d_f, sizeof(double) * n));
    CK(cudaMalloc(&c->d_gr, sizeof(double) * 3 * n));
  }
  CK(cudaMemcpyAsync(c->d_X, X3n, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, c->stream));
  if (g3n && c->cfg.subpix_method == PTK_SUBPIX_ADJOINT_LM)
    launch_grad_f32(c->g, frame(c, c->cur_slot), c->d_X, c->d_f, c->d_gr, c->stream);  // the LM's FP32 adjoint
  else
    launch_objective(c->g, frame(c, c->cur_slot), subpix_params(c), c->d_X, c->d_f, g3n ? c->d_gr : nullptr,
                     c->max_P, c->stream);
  c->launches += 1;
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(f, c->d_f, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
  if (g3n) CK(cudaMemcpyAsync(g3n, c->d_gr, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return PTK_OK;
}

int ptk_objective(ptk_ctx* c, const double* X3n, double* f) { return objective_common(c, X3n, f, nullptr); }

int ptk_grad(ptk_ctx* c, const double* X3n, double* f, double* g3n) {
  if (!g3n) return fail(c, PTK_ERR_ARG, "null gradient");
  return objective_common(c, X3n, f, g3n);
}

int ptk_set_distortion(ptk_ctx* c, const double* p14) {
  if (!c || !p14) return fail(c, PTK_ERR_ARG, "null argument");
  std::memcpy(c->disto, p14, sizeof(c->disto));
  c->have_disto = true;
  c->map_valid = false;
  return PTK_OK;
}

int ptk_remap_frame(ptk_ctx* c, int slot) {
  if (!c || slot < 0 || slot > 1) return fail(c, PTK_ERR_ARG, "bad arguments");
  sync_cur(c);
  if (!c->have_disto) return fail(c, PTK_ERR_STATE, "no distortion parameters set");
  if (!c->loaded[slot]) return fail(c, PTK_ERR_STATE, "frame not loaded");
  const int dimx = c->cfg.dimx, dimy = c->cfg.dimy;
  if (!c->d_map) CK(cudaMalloc(&c->d_map, sizeof(double2) * (size_t)dimx * dimy));
  if (!c->d_tmp) CK(cudaMalloc(&c->d_tmp, (size_t)c->pitch * dimy * 2));
  if (!c->map_valid) {
    const double trig[4] = {std::cos(c->disto[10]), -std::sin(c->disto[10]), -std::sin(c->disto[12]),
                            std::cos(c->disto[12])};
    launch_remap_build(c->disto, trig, c->d_map, dimx, dimy, c->stream);
    c->launches += 1;
    c->map_valid = true;
  }
  const int phys = slot == 0 ? c->ref_slot : c->cur_slot;
  launch_remap_apply(c->d_map, c->d_img[phys], c->d_tmp, c->pitch, dimx, dimy, c->stream);
  c->launches += 1;
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(c->d_img[phys], c->d_tmp, (size_t)c->pitch * dimy * 2, cudaMemcpyDeviceToDevice, c->stream));
  if (slot == 0) c->need_precompute = true;
  return PTK_OK;
}

int ptk_set_stream(ptk_ctx* c, void* s) {
  if (!c) return fail(c, PTK_ERR_ARG, "null context");
  sync_cur(c);
  CK(cudaStreamSynchronize(c->stream));
  c->stream = s ? static_cast<cudaStream_t>(s) : c->own_stream;
  return PTK_OK;
}

void* ptk_get_stream(ptk_ctx* c) { return c ? static_cast<void*>(c->stream) : nullptr; }

int ptk_synchronize(ptk_ctx* c) {
  if (!c) return fail(c, PTK_ERR_ARG, "null context");
  sync_cur(c);
  CK(cudaStreamSynchronize(c->stream));
  all_released(c);
  int flag = 0;  // set by a device wait that gave up (BF16 search)
  CK(cudaMemcpy(&flag, c->d_counts + 3, sizeof(int), cudaMemcpyDeviceToHost));
  if (flag) {
    CK(cudaMemsetAsync(c->d_counts + 3, 0, sizeof(int), c->stream));
    return fail(c, PTK_ERR_TIMEOUT, "a tensor-core search wait gave up");
  }
  return PTK_OK;
}

int64_t ptk_kernel_launches(ptk_ctx* c) { return c ? c->launches : 0; }

int ptk_test_bf16_wait_timeout(ptk_ctx* c, int polls) {
  if (!c) return fail(c, PTK_ERR_ARG, "null context");
  if (polls < 0) return fail(c, PTK_ERR_ARG, "polls must be >= 0");
  c->probe_wait = polls;
  invalidate(c);  // captured frame graphs hold the old launch parameters
  return PTK_OK;
}

int ptk_abi_sizes(size_t* config_bytes, size_t* grain_bytes, size_t* zone_bytes) {
  if (!config_bytes || !grain_bytes || !zone_bytes) return fail(nullptr, PTK_ERR_ARG, "null argument");
  *config_bytes = sizeof(ptk_config);
  *grain_bytes = sizeof(ptk_grain);
  *zone_bytes = sizeof(ptk_zone);
  return PTK_OK;
}

const char* ptk_last_error(ptk_ctx* c) { return c ? c->err.c_str() : g_static_error.c_str(); }

}  // extern "C"
