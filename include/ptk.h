/*
 * ptk.h -- C ABI of the B200 (sm_100a) per-grain tracking path.
 *
 * Replaces the call surface of p-tracker's `ptracker` class for particle
 * tracking (reference src/p-tracker.hpp:66-238): the data members it reads
 * (images, grains, search zones, options) become a context, and the per-grain
 * member functions called from OpenMP loops become batched calls over all
 * grains.  Every function returns an int status (PTK_OK = 0); the reference
 * instead calls std::exit on I/O errors (src/p-tracker.cpp:98,216,1217,1317).
 *
 * Ownership: the caller owns every host array passed in or out; the context
 * owns its device memory and one CUDA stream (or borrows a caller stream, see
 * ptk_set_stream).  A context is not thread-safe; distinct contexts are
 * independent.  All device work of a call is enqueued on the context stream
 * (host frame uploads on the context's copy streams, ordered with it, see
 * ptk_load_frame); calls that return host data synchronise that stream.
 */
#ifndef PTK_H
#define PTK_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
enum {
  PTK_OK = 0,
  PTK_ERR_ARG = 1,     /* invalid argument                                  */
  PTK_ERR_STATE = 2,   /* call out of order (e.g. no frame loaded)          */
  PTK_ERR_CUDA = 3,    /* CUDA runtime error (message in ptk_last_error)    */
  PTK_ERR_IO = 4,      /* file could not be read or written                 */
  PTK_ERR_LIMIT = 5,   /* size beyond a documented limit                    */
  PTK_ERR_TIMEOUT = 6  /* a bounded device wait gave up                     */
};

/* ---- per-grain status bits (ptk_grain.status) -------------------------- */
enum {
  PTK_ST_RESCUED = 1,        /* pixel NCC < NCC_min: rescue search ran        */
  PTK_ST_SUPER_RESCUED = 2,  /* rescue NCC < NCC_min_super: super-rescue ran  */
  PTK_ST_FAILED = 4,         /* super-rescue did not exceed NCC_min_super     */
  PTK_ST_OUT_OF_BOUNDS = 8,  /* pattern + zone + interpolation support leaves
                                the frame: grain not searched (the reference
                                reads out of bounds here, src/interpol.cpp:28) */
  PTK_ST_MASKED = 16,        /* grain_type_2D::masked (src/grain_type_2D.hpp:53) */
  PTK_ST_SUBPIX_CLAMPED = 32 /* a subpixel sample was clamped to the frame     */
};

enum { PTK_INTERP_LINEAR = 0, PTK_INTERP_CUBIC = 1, PTK_INTERP_QUINTIC = 2 };
enum { PTK_SUBPIX_POWELL = 0, PTK_SUBPIX_ADJOINT_LM = 1 };
/* PTK_SEARCH_EXACT picks the register-tiled exact kernel when its shared-memory
 * layout fits, else the direct one; PTK_SEARCH_EXACT_DIRECT forces the direct
 * per-point kernel.  Both return identical results. */
enum { PTK_SEARCH_EXACT = 0, PTK_SEARCH_BF16 = 1, PTK_SEARCH_EXACT_DIRECT = 2 };
enum { PTK_LEVEL_PIXEL = 0, PTK_LEVEL_RESCUE = 1, PTK_LEVEL_SUPER_RESCUE = 2 };
enum { PTK_PATTERN_CIRC = 0, PTK_PATTERN_RING = 1, PTK_PATTERN_RECT = 2, PTK_PATTERN_GRAIN_DIAMETER = 3 };

/* search_zone_type, reference src/search_zone_type.hpp:20-27 */
typedef struct ptk_zone {
  int32_t left, right, up, down; /* pixels, >= 0                             */
  int32_t num_rot;               /* rotations tested: the list produced by
                                    for (d = -|inc*num|; d <= |inc*num|; d += inc) */
  double inc_rot;                /* radians                                   */
} ptk_zone;

/* One grain: the 13 columns of a dic_out file (reference
 * src/p-tracker.cpp:1330-1343, grain_type_2D src/grain_type_2D.hpp:23-71). */
typedef struct ptk_grain {
  int32_t refcoord_xpix, refcoord_ypix;
  double refrot, radius_pix;
  double dx, dy, drot;
  double upix, vpix, rot_inc;
  double NCC, NCC_rescue, NCC_subpix;
  uint8_t masked; /* input: grain is skipped (mask_rect)                      */
  uint8_t status; /* output: PTK_ST_* bits of the last tracked frame         */
  uint8_t pad_[6];
} ptk_grain;

/* Options of the command file that drive tracking (reference
 * src/p-tracker.cpp:1487-1784; defaults src/p-tracker.hpp:67-178). */
typedef struct ptk_config {
  int32_t dimx, dimy;            /* frame size in pixels                      */
  int32_t rescue_level;          /* -1..2, default 2                          */
  double NCC_min;                /* default 0.7                               */
  double NCC_min_super;          /* default 0.5                               */
  int32_t subpixel;              /* 0/1, default 1                            */
  double subpix_tol;             /* Powell ftol, default 1e-8                 */
  double initial_direction[3];   /* dx, dy, dr, default 0.01 each             */
  int32_t image_interpolator;    /* PTK_INTERP_*, default cubic               */
  double overflow_stiffness;     /* default 0                                 */
  double subpix_displacement_max;/* default 3                                 */
  int32_t rotations;             /* 0 disables rotation search (init rule
                                    src/p-tracker.cpp:1191-1201)              */
  ptk_zone zone[3];              /* pixel, rescue, super-rescue               */
  int32_t iraz;                  /* reference change period, default 0        */
  int32_t subpix_method;         /* PTK_SUBPIX_*, default POWELL              */
  int32_t search_method;         /* PTK_SEARCH_*, default EXACT               */
  int32_t topk;                  /* BF16 search: candidates per 32x32 tile rescored exactly, those within 3 % of its best score (1..8, default 8) */
  int32_t lm_max_iter;           /* adjoint LM: iteration cap                 */
  double lm_tol;                 /* adjoint LM: step tolerance (pixels, default 1e-4) */
  int32_t autotune;              /* 1: ptk_track_frame runs ptk_autotune once, before its first frame;
                                    if tuning fails the built-in shapes are kept (default 0) */
  double lm_cell_px;             /* adjoint LM: a refinement ending more than this many pixels (x or y)
                                    from its integer optimum ... (default 0: every LM result kept) */
  double lm_cell_rot;            /* ... or more than this many level-0 rotation steps from it (<= 0: no
                                    rotation bound) leaves the grain, untouched, to the reference's Powell */
} ptk_config;

typedef struct ptk_ctx ptk_ctx;

/* Fills *cfg with the reference defaults (src/p-tracker.hpp:67-178); search
 * zones (which have no default in the reference) become 0 px, 0 rotations. */
int ptk_config_default(ptk_config* cfg);

/* Context lifetime.  Replaces ptracker::ptracker / ptracker::init
 * (src/p-tracker.cpp:19-73, 1150-1210). */
int ptk_create(ptk_ctx** out, const ptk_config* cfg);
int ptk_destroy(ptk_ctx* ctx);
int ptk_set_config(ptk_ctx* ctx, const ptk_config* cfg);

/* Replaces ptracker::search_zone / search_zone_rescue / search_zone_super_rescue
 * assignment in read_data (src/p-tracker.cpp:1616-1669). */
int ptk_set_search_zone(ptk_ctx* ctx, int level, const ptk_zone* zone);

/* Grains.  Replaces read_grains' fill of ptracker::grain
 * (src/p-tracker.cpp:1213-1278) and the dic_out write (src/p-tracker.cpp:1313-1360). */
int ptk_set_grains(ptk_ctx* ctx, const ptk_grain* grains, int n);
int ptk_get_grains(ptk_ctx* ctx, ptk_grain* out, int n);
/* Device-side copy of the whole grain state and its restoration (stream
 * ordered, no host transfer).  The per-frame dic_out files are the
 * reference's checkpoint (src/p-tracker.cpp:584, restart_file :1515-1518);
 * these keep one in device memory, e.g. to re-track a frame pair. */
int ptk_snapshot_grains(ptk_ctx* ctx);
int ptk_restore_grains(ptk_ctx* ctx);

/* Patterns as CSR: grain g owns offsets_xy[2*starts[g] .. 2*starts[g+1]).
 * Replaces make_custom_pattern (src/p-tracker.cpp:1444-1476). */
int ptk_set_patterns(ptk_ctx* ctx, const int32_t* offsets_xy, const int64_t* starts, int n);
/* Generators of the `pattern` token (src/p-tracker.cpp:1650-1688):
 * CIRC a, RING a b, RECT a b, GRAIN_DIAMETER (radius_reduction=a, min_radius=b);
 * applied to every grain whose radius equals target_radius, or to all grains
 * when target_radius < 0 (targetRadiusPattern). */
int ptk_make_patterns(ptk_ctx* ctx, int kind, double a, double b, double target_radius);
int ptk_pattern_size(ptk_ctx* ctx, int grain, int* npts);

/* Frames.  slot 0 = reference image, 1 = current image (ptracker::image[
 * im_index_ref / im_index_current], src/p-tracker.hpp:80-83).  `pix` is a
 * row-major host buffer of 1- or 2-byte grey levels with `pitch_bytes` per
 * row; 1-byte values are widened to uint16 unchanged.  Replaces read_image
 * (src/p-tracker.cpp:75-83) after decode.  The copy runs on a copy stream of
 * the frame buffer it fills: after a queued ptk_track_frame it waits only
 * until that frame no longer reads the buffer (the reference buffer after
 * its precompute, the current one at the frame's end), otherwise until all
 * queued work is done; calls that read the frame wait for the copy.  `pix`
 * must stay unchanged until a frame that reads it has been tracked and its
 * records read back, or ptk_synchronize has returned. */
int ptk_load_frame(ptk_ctx* ctx, int slot, const void* pix, int dimx, int dimy, int bytes_per_px,
                   size_t pitch_bytes);
/* Same with a device pointer (uint16, row-major, pitch in bytes). */
int ptk_load_frame_device(ptk_ctx* ctx, int slot, const void* dev_pix, size_t pitch_bytes);
/* Page-locked host memory (no reference counterpart): frames uploaded from
 * it with ptk_load_frame go up asynchronously at full link speed (from
 * ordinary memory the copy is staged and the call returns only when it is
 * done).  ptk_host_free releases it. */
int ptk_host_alloc(void** ptr, size_t bytes);
int ptk_host_free(void* ptr);
/* A frame from an unpacked RAW sensor mosaic, demosaiced on the GPU as
 * read_raw_image does after libraw's unpack (src/p-tracker.cpp:288-383):
 * `raw` is libraw's rawdata.raw_image (raw_width x raw_height uint16,
 * row-major), the frame (the context's dimx x dimy = sizes.width x height)
 * starts at (left_margin, top_margin).  mode = DemosaicModel:
 * PTK_DEMOSAIC_BOX2 (-1) floor of the 2x2 mean, PTK_DEMOSAIC_BINOMIAL3 (-2)
 * floor of the 1-2-1 x 1-2-1 / 16 mean, PTK_DEMOSAIC_GREY (-20) the raw
 * values.  Neighbours are taken in the flat raw array as the reference does;
 * a call whose stencil reaches outside it is rejected (PTK_ERR_ARG), and so
 * are libraw's own modes (>= 0).  rescale != 0 is rescaleGrayLevels:
 * floor((v - MinGray) * 65535 / (MaxGray - MinGray)), skipped when all
 * pixels are equal (the reference divides by zero there).  min_max, when not
 * NULL, receives MinGray and MaxGray (and the call waits for the stream). */
enum { PTK_DEMOSAIC_BOX2 = -1, PTK_DEMOSAIC_BINOMIAL3 = -2, PTK_DEMOSAIC_GREY = -20 };
int ptk_load_frame_raw(ptk_ctx* ctx, int slot, const uint16_t* raw, int raw_width, int raw_height, int left_margin,
                       int top_margin, int mode, int rescale, uint16_t* min_max);
/* Same with the mosaic already in device memory. */
int ptk_load_frame_raw_device(ptk_ctx* ctx, int slot, const uint16_t* dev_raw, int raw_width, int raw_height,
                              int left_margin, int top_margin, int mode, int rescale, uint16_t* min_max);
/* Copies a slot back to the host as uint16 rows of dimx values. */
int ptk_read_frame(ptk_ctx* ctx, int slot, uint16_t* out);

/* Stages.  ptk_precompute replaces do_precomputations (src/p-tracker.cpp:624-656).
 * ptk_search(level) replaces the omp loops of follow_pattern_pixel /
 * follow_pattern_rescue_pixel / follow_pattern_super_rescue_pixel
 * (src/p-tracker.cpp:471-536, 659-1016); level 0 also performs the
 * reset()/backup() of every grain (src/p-tracker.cpp:478-479) and rebuilds
 * the rescue list, levels 1/2 consume the lists left by the previous level.
 * ptk_subpixel replaces follow_pattern_subpixel_xyR (src/p-tracker.cpp:1090-1128). */
int ptk_precompute(ptk_ctx* ctx);
int ptk_search(ptk_ctx* ctx, int level);
/* Profiling aid (no reference counterpart): ptk_search(level) with CUDA events
 * recorded on the context stream between its search kernels; synchronizes and
 * writes each kernel's duration in milliseconds to kernel_ms, in launch order -
 * PTK_SEARCH_BF16: window statistics, weights, tensor-core search, rescoring
 * (4 values); exact forms: the search kernel (1 value).  *n_kernels receives
 * the count; max_kernels bounds what is written. */
int ptk_search_timed(ptk_ctx* ctx, int level, float* kernel_ms, int max_kernels, int* n_kernels);
int ptk_subpixel(ptk_ctx* ctx, int method);
/* Increments upix = dx - dx_prev ... and, when num_image - iref >= iraz, the
 * reference change (src/p-tracker.cpp:577-611). */
int ptk_end_frame(ptk_ctx* ctx, int num_image);
/* The whole per-frame body of particle_tracking after the image read
 * (src/p-tracker.cpp:458-611, file output excluded), captured once as a CUDA
 * graph and replayed. */
int ptk_track_frame(ptk_ctx* ctx, int num_image);
/* Forces the reference change of ptk_end_frame regardless of iraz. */
int ptk_swap_reference(ptk_ctx* ctx, int num_image);
int ptk_set_iref(ptk_ctx* ctx, int iref);

/* Rescue bookkeeping of the last frame: counts of ptracker::to_be_rescued /
 * to_be_super_rescued (src/p-tracker.hpp:108-118). */
int ptk_get_rescue_counts(ptk_ctx* ctx, int* n_rescued, int* n_super_rescued);

/* Subpixel objective NCC_to_minimize_xyR (src/p-tracker.cpp:1018-1088) for
 * every grain at X[3*g .. 3*g+2]; f[g] receives (1 - NCC) * W. */
int ptk_objective(ptk_ctx* ctx, const double* X3n, double* f);
/* Same objective and its gradient with respect to (dx, dy, drot) through the
 * cubic interpolation (adjoint kernel; no reference counterpart). */
int ptk_grad(ptk_ctx* ctx, const double* X3n, double* f, double* g3n);

/* Distortion correction.  params14 in the order of
 * ptracker::disto_parameters (src/p-tracker.hpp:151-165) as used by undistor
 * (src/distortion_correction.cpp:20-61).  ptk_remap_frame resamples a slot so
 * that pixel (x, y) holds the distorted frame at the point whose undistor()
 * image is (x, y) (cubic interpolation, rounded); pixels whose support leaves
 * the frame become 0.  The inverse map is computed once per parameter set and
 * cached on the device. */
int ptk_set_distortion(ptk_ctx* ctx, const double* params14);
int ptk_remap_frame(ptk_ctx* ctx, int slot);

/* Stream control.  A non-null stream is borrowed (not destroyed). */
int ptk_set_stream(ptk_ctx* ctx, void* cuda_stream);
void* ptk_get_stream(ptk_ctx* ctx);
int ptk_synchronize(ptk_ctx* ctx);
/* Number of device kernels this context launched since creation. */
int64_t ptk_kernel_launches(ptk_ctx* ctx);

/* Failure-path test hook (no counterpart in the reference).  Every wait of the
 * BF16 search kernel on its barriers is bounded; one that runs out sets a
 * device flag that ptk_synchronize reports as PTK_ERR_TIMEOUT, and the kernel
 * drains its own copies and MMAs, frees its tensor memory and returns.  With
 * polls > 0, each later BF16 search launch of this context first waits on a
 * barrier that nothing arrives on -- before it issues any copy or MMA -- and
 * gives up after `polls` polls, so that path runs without a real fault.
 * polls = 0 turns it off.  Frame graphs captured before the call are rebuilt. */
int ptk_test_bf16_wait_timeout(ptk_ctx* ctx, int polls);

/* Pixel-stage search that allocates nothing (no counterpart in the reference).
 * For callers that cannot call cudaMalloc -- a plug-in whose host application
 * owns all device memory, or a loop where an allocation and the device
 * synchronisation it may imply are not allowed.  Computes, for every grain,
 * what ptk_search(level 0) computes before its acceptance rule: the first
 * strict NCC maximum above 0 over the zone's rotation steps and offsets.
 * All pointers are device pointers the caller owns (frames: uint16 rows of
 * pitch_bytes; pattern_starts: n_grains + 1 CSR offsets into pattern_xy,
 * int16 x,y pairs); `zone` is a host struct; rotations == 0 searches the
 * single step -0.0 as the reference's `rotations 0`.  max_points must bound
 * every pattern's size (<= 16384) and max_radius every |x| and |y| of a
 * pattern offset after it is rotated by any searched angle (refrot + drot +
 * step) and rounded; a pattern's Euclidean radius, rounded up, plus one
 * always suffices.  Outputs: best NCC, best x/y offset and rotation step
 * per grain (0, 0, 0, 0.0 when no NCC exceeds 0).  A grain gets NaN and
 * best_u = best_v = INT_MIN + 1 when its pattern exceeds max_points or a
 * rotated offset exceeds max_radius (the caller's limits), and NaN with
 * INT_MIN when its footprint leaves the frame.  Each enqueue's own status is
 * returned (PTK_ERR_CUDA when it fails); an error left pending by earlier
 * work of the caller is neither reported nor cleared.  Scratch lives in one fixed 4 MiB device
 * array per GPU, kept for the life of the process: n_grains x rotation steps
 * x ceil(nu/32) x ceil(nv/32) must not exceed 260,080 (PTK_ERR_LIMIT
 * otherwise), with at most 4096 rotation steps.  Calls share that array, so
 * calls that overlap on the GPU race.  The first call on a device looks up
 * the array's device address; make it before any stream capture.
 * Work is enqueued on `stream` (NULL = legacy default stream). */
int ptk_search_pixel_noalloc(const uint16_t* ref_pix, const uint16_t* cur_pix, size_t pitch_bytes, int dimx,
                             int dimy, int n_grains, const int32_t* refx, const int32_t* refy, const double* refrot,
                             const double* drot, const double* dx, const double* dy, const int32_t* pattern_starts,
                             const int16_t* pattern_xy, int max_points, int max_radius, const ptk_zone* zone,
                             int rotations, double* best_ncc, int32_t* best_u, int32_t* best_v, double* best_drot,
                             void* stream);

/* sizeof of the ABI structs as compiled into the library, for FFI binders. */
int ptk_abi_sizes(size_t* config_bytes, size_t* grain_bytes, size_t* zone_bytes);

/* Last error message of the context (static storage if ctx is NULL). */
const char* ptk_last_error(ptk_ctx* ctx);

/* Grain files.  ptk_read_grains_file parses the 13-column dic_out form
 * (format13 != 0, restart_file, src/p-tracker.cpp:1235-1252) or the
 * 4-column start form (format13 == 0, grains_to_follow,
 * src/p-tracker.cpp:1253-1272).  Call once with out == NULL to get the count.
 * ptk_save_grains_file writes the dic_out form byte for byte as
 * save_grains (src/p-tracker.cpp:1313-1360). */
int ptk_read_grains_file(const char* path, int format13, ptk_grain* out, int capacity, int* n);
int ptk_save_grains_file(const char* path, const ptk_grain* grains, int n, const char* from_image,
                         const char* from_datetime, const char* to_image, const char* to_datetime);

/* Autotuner (no reference counterpart): times the admissible shapes of the
 * level-0 search on the loaded frame pair - the BF16 kernel's operand-row
 * ring depth (2, 3, 4 or 6 buffers; the strip height follows from the
 * shared-memory budget) or, in the exact form, the register-tiled against
 * the direct kernel - with CUDA events, five runs each (the first a
 * warm-up), each after a 256 MiB write that evicts L2 (when that much memory
 * is free), from the same grain state (restored after every run and at the
 * end), and keeps the fastest for this context until its search method or
 * level-0 zone changes; the built-in shape (4 buffers, the tiled kernel)
 * stays unless another is more than 2 % faster.  Every candidate gives the same results.  With
 * ptk_config.autotune = 1, ptk_track_frame calls it once before building its
 * first graph.  report (may be NULL): method 1 = BF16 (values = ring depths),
 * 0 = exact (1 tiled, 2 direct); the candidates' best times in ms. */
typedef struct ptk_tune_report {
  int32_t method, choice, n;
  int32_t values[8];
  float ms[8];
} ptk_tune_report;
int ptk_autotune(ptk_ctx* ctx, ptk_tune_report* report);

/* Autotune cache (no reference counterpart).  ptk_set_tune_cache(ctx, path)
 * (path NULL: off) makes ptk_autotune look up the context's workload
 * signature in the JSON file at path first: an entry for the same search
 * method whose choice is admissible is taken without timing (report->n = 0);
 * otherwise ptk_autotune times the candidates as above and writes its result
 * into the file (created if missing).  The signature names the GPU (compute
 * capability, name, SM count), the search method, the frame size, the grain
 * count, the largest pattern radius and the grains per 8-px radius class,
 * the level-0 zone, rotation steps and topk: ptk_tune_signature writes it to
 * buf (capacity cap, PTK_ERR_LIMIT when too small).  ptk_tune_cache_lookup /
 * ptk_tune_cache_store read and update one entry of such a file on the host
 * (no GPU): lookup sets *found = 0 when the file or the entry is missing;
 * both return PTK_ERR_IO for a malformed or unwritable file (which they
 * leave unchanged). */
int ptk_set_tune_cache(ptk_ctx* ctx, const char* path);
int ptk_tune_signature(ptk_ctx* ctx, char* buf, int32_t cap);
int ptk_tune_cache_lookup(const char* path, const char* signature, int32_t* found, int32_t* method,
                          int32_t* choice);
int ptk_tune_cache_store(const char* path, const char* signature, int32_t method, int32_t choice, int32_t n,
                         const int32_t* values, const float* ms);

/* Image files (host only, no GPU).  ptk_read_image_file decodes a strip
 * TIFF (uncompressed, LZW, Deflate or PackBits, optional horizontal
 * predictor; 8/16-bit grey or RGB) into the grey levels that read_tiff_image
 * computes through libtiff's RGBA reader (src/p-tracker.cpp:86-187): 8-bit
 * channels r, g, b scaled by 1/255, grey = (uint16)(65535 (0.299 r + 0.587 g
 * + 0.114 b)), rows top-down (16-bit grey keeps its high byte, as that reader
 * does).  Binary PGM (P5, no reference counterpart) is returned as stored.
 * With out == NULL only dimx / dimy are filled; datetime (may be NULL)
 * receives the TIFF DateTime tag or "dateTime unknown".  ptk_image_error
 * describes the calling thread's last failure. */
int ptk_read_image_file(const char* path, uint16_t* out, size_t capacity, int* dimx, int* dimy, char* datetime,
                        int datetime_len);
const char* ptk_image_error(void);

/* Distortion-parameter fit: the minimisation of the correction_distortion
 * procedure (src/distortion_correction.cpp:135-479) over grains tracked from
 * a reference image into n_tracked images.
 * ptk_disto_pairs: precompute_paires (src/distortion_correction.cpp:63-81),
 *   the pairs (i < j, i-major) whose reference positions lie dmin .. dmax
 *   apart; host only.  Writes at most `capacity` pairs (2 ints each) and the
 *   count to *npairs (PTK_ERR_LIMIT when it exceeds capacity).
 * ptk_disto_create: uploads the grains' reference positions, their tracked
 *   displacements and subpixel NCC per image ([image][grain], images after the
 *   reference) and the pairs.
 * ptk_disto_objective: the equiprojectivity criterion (the POWELL functor,
 *   :249-290) for the 14 undistor parameters, evaluated on the GPU in FP64;
 *   ptk_disto_residuals also returns the residual of every (image, pair),
 *   image-major, 0 where a pair is skipped (NCC below NCC_min).
 * ptk_disto_fit: default centres (negative xc/yc entries -> the frame centre),
 *   then POWELL (one minimisation, ftol 1e-12, initial directions the
 *   perturbations) or POWELL_ITER (num_iter minimisations, each followed by
 *   re-anchoring on the undistorted reference positions, :300-386); params14
 *   in/out, index_ini / index_end = criterion / n_tracked before and after,
 *   history (may be NULL) = num_iter x 15 (index, 14 parameters) for
 *   POWELL_ITER.  LEVMAR (src/distortion_correction.cpp:400-479): all 14
 *   parameters by Levenberg-Marquardt over the residual vector, the
 *   published MINPACK lmdif1 algorithm with tol = DBL_EPSILON (the reference
 *   calls it from the absent toofus library; perturb14 is not used); history
 *   (may be NULL) = 1 x 15, the final index and parameters.
 * ptk_disto_levmar_info (no reference counterpart): exit state of the last
 *   LEVMAR fit (lmdif's info code 0-8, or -2 when none ran), its residual
 *   evaluations, and the text the reference prints for the code.
 * ptk_disto_tracked: the displacements after POWELL_ITER's re-anchoring.
 * ptk_disto_objective_timed (no reference counterpart): `reps` evaluations of
 *   the objective's kernels between two CUDA events, without read-back;
 *   *ms_per_eval = their average device time. */
typedef struct ptk_disto ptk_disto;
enum { PTK_DISTO_POWELL = 0, PTK_DISTO_POWELL_ITER = 1, PTK_DISTO_LEVMAR = 2 };
int ptk_disto_pairs(const int32_t* refx, const int32_t* refy, int n, double dmin, double dmax, int32_t* pairs_ij,
                    int64_t capacity, int64_t* npairs);
int ptk_disto_create(ptk_disto** out, int dimx, int dimy, const int32_t* refx, const int32_t* refy, int n,
                     int n_tracked, const double* dx, const double* dy, const double* ncc_subpix, double NCC_min,
                     const int32_t* pairs_ij, int64_t npairs);
int ptk_disto_destroy(ptk_disto* d);
const char* ptk_disto_last_error(ptk_disto* d);
int ptk_disto_objective(ptk_disto* d, const double* params14, double* value);
int ptk_disto_residuals(ptk_disto* d, const double* params14, double* value, double* fvec);
int ptk_disto_fit(ptk_disto* d, double* params14, const double* perturb14, int algo, int num_iter,
                  double* index_ini, double* index_end, double* history);
int ptk_disto_tracked(ptk_disto* d, double* dx, double* dy);
int ptk_disto_levmar_info(ptk_disto* d, int* info, int* nfev, const char** text);
int ptk_disto_objective_timed(ptk_disto* d, const double* params14, int reps, double* ms_per_eval);

#ifdef __cplusplus
}
#endif

#endif /* PTK_H */
