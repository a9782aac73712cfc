// ORACLE / TEST INFRASTRUCTURE ONLY -- never linked into the product library.
//
// C harness around the reference's own tracking code, compiled unmodified from
// the reference sources (src/p-tracker.cpp, src/interpol.cpp,
// src/grain_type_2D.cpp, src/NCC_optimizer_functor.cpp,
// src/distortion_correction.cpp) against the stub headers in oracle/stubs.
// Image decode is bypassed: pixel values are written straight into
// ptracker::image (x-major, src/p-tracker.hpp:80).  The per-frame orchestration
// of ptracker::particle_tracking (src/p-tracker.cpp:442-611) is restated here
// without its file I/O and console output, calling the reference's member
// functions for every computation.
#include <omp.h>

#include <cstdlib>
#include <cstring>

#include "p-tracker.hpp"

namespace {

struct Handle {
  ptracker trk;
  int nthreads{1};
};

void fill_slot(ptracker& t, int idx, const uint16_t* rowmajor, int dimx, int dimy) {
  for (int x = 0; x < dimx; ++x)
    for (int y = 0; y < dimy; ++y) t.image[idx][x][y] = rowmajor[(size_t)y * dimx + x];
}

void set_threads(Handle* h) {
  int n = h->nthreads;
  if (n < 1) n = 1;
  if (n > MAX_NUMBER_THREADS) n = MAX_NUMBER_THREADS;  // src/p-tracker.hpp:35,141
  omp_set_num_threads(n);
}

}  // namespace

extern "C" {

void* ref_create(int dimx, int dimy) {
  Handle* h = new Handle();
  ptracker& t = h->trk;
  t.dimx = dimx;
  t.dimy = dimy;
  t.image.assign(2, std::vector<std::vector<uint16_t>>(dimx, std::vector<uint16_t>(dimy, 0)));
  t.imageData.resize(2);
  t.imageData[0].dateTime = "dateTime unknown";
  t.imageData[1].dateTime = "dateTime unknown";
  std::strcpy(t.image_name, "image%d.tiff");
  // search zones have no defaults in the reference (src/search_zone_type.hpp:20-27)
  search_zone_type z{0, 0, 0, 0, 0, 1.0};
  t.search_zone = t.search_zone_rescue = t.search_zone_super_rescue = z;
  return h;
}

void ref_destroy(void* p) { delete static_cast<Handle*>(p); }

void ref_set_threads(void* p, int n) { static_cast<Handle*>(p)->nthreads = n; }

// Writes the reference frame (first_time semantics of read_tiff_image,
// src/p-tracker.cpp:191-198: both slots receive the image).
void ref_load_first(void* p, const uint16_t* img) {
  ptracker& t = static_cast<Handle*>(p)->trk;
  fill_slot(t, t.im_index_ref, img, t.dimx, t.dimy);
  fill_slot(t, t.im_index_current, img, t.dimx, t.dimy);
}

void ref_load_reference(void* p, const uint16_t* img) {
  ptracker& t = static_cast<Handle*>(p)->trk;
  fill_slot(t, t.im_index_ref, img, t.dimx, t.dimy);
}

void ref_load_current(void* p, const uint16_t* img) {
  ptracker& t = static_cast<Handle*>(p)->trk;
  fill_slot(t, t.im_index_current, img, t.dimx, t.dimy);
}

void ref_get_indices(void* p, int* iref_idx, int* icur_idx, int* iref) {
  ptracker& t = static_cast<Handle*>(p)->trk;
  *iref_idx = t.im_index_ref;
  *icur_idx = t.im_index_current;
  *iref = t.iref;
}

// rec13: n x 13 doubles in dic_out column order (src/p-tracker.cpp:1330-1343).
void ref_set_grains(void* p, int n, const double* rec13, const uint8_t* masked) {
  ptracker& t = static_cast<Handle*>(p)->trk;
  t.num_grains = n;
  t.grain.clear();
  t.grain.resize(n);
  t.to_be_rescued.assign(n, 0);
  t.to_be_super_rescued.assign(n, 0);
  for (int i = 0; i < n; ++i) {
    const double* r = rec13 + 13 * (size_t)i;
    grain_type_2D& g = t.grain[i];
    g.refcoord_xpix = (int)r[0];
    g.refcoord_ypix = (int)r[1];
    g.refrot = r[2];
    g.radius_pix = r[3];
    g.dx = r[4];
    g.dy = r[5];
    g.drot = r[6];
    g.upix = r[7];
    g.vpix = r[8];
    g.rot_inc = r[9];
    g.NCC = r[10];
    g.NCC_rescue = r[11];
    g.NCC_subpix = r[12];
    g.masked = masked ? masked[i] != 0 : false;
  }
  t.require_precomputations = true;
}

void ref_get_grains(void* p, double* rec13) {
  ptracker& t = static_cast<Handle*>(p)->trk;
  for (int i = 0; i < t.num_grains; ++i) {
    double* r = rec13 + 13 * (size_t)i;
    const grain_type_2D& g = t.grain[i];
    r[0] = g.refcoord_xpix;
    r[1] = g.refcoord_ypix;
    r[2] = g.refrot;
    r[3] = g.radius_pix;
    r[4] = g.dx;
    r[5] = g.dy;
    r[6] = g.drot;
    r[7] = g.upix;
    r[8] = g.vpix;
    r[9] = g.rot_inc;
    r[10] = g.NCC;
    r[11] = g.NCC_rescue;
    r[12] = g.NCC_subpix;
  }
}

void ref_get_precomp(void* p, double* mean0, double* C0C0) {
  ptracker& t = static_cast<Handle*>(p)->trk;
  for (int i = 0; i < t.num_grains; ++i) {
    mean0[i] = t.grain[i].mean0;
    C0C0[i] = t.grain[i].C0C0;
  }
}

// Custom pattern (the "pattern file" form, src/p-tracker.cpp:1444-1476).
void ref_set_pattern(void* p, int ig, int npts, const int32_t* xy) {
  ptracker& t = static_cast<Handle*>(p)->trk;
  grain_type_2D& g = t.grain[ig];
  g.pattern.resize(npts);
  g.pattern0_rotated.resize(npts);
  g.pattern1_rotated.resize(npts);
  for (int i = 0; i < npts; ++i) {
    g.pattern[i].dx = xy[2 * i];
    g.pattern[i].dy = xy[2 * i + 1];
  }
  t.require_precomputations = true;
}

// kind: 0 circ(a), 1 ring(a, b), 2 rect(a, b)  (src/p-tracker.cpp:1369-1442)
void ref_make_pattern(void* p, int ig, int kind, int a, int b) {
  ptracker& t = static_cast<Handle*>(p)->trk;
  if (kind == 0) t.make_circ_pattern(ig, a);
  else if (kind == 1) t.make_ring_pattern(ig, a, b);
  else t.make_rect_pattern(ig, a, b);
  t.require_precomputations = true;
}

int ref_pattern_size(void* p, int ig) {
  return (int)static_cast<Handle*>(p)->trk.grain[ig].pattern.size();
}

void ref_get_pattern(void* p, int ig, int which, int32_t* xy) {
  const grain_type_2D& g = static_cast<Handle*>(p)->trk.grain[ig];
  const std::vector<relative_coord_type>& v = which == 0 ? g.pattern : g.pattern0_rotated;
  for (size_t i = 0; i < v.size(); ++i) {
    xy[2 * i] = v[i].dx;
    xy[2 * i + 1] = v[i].dy;
  }
}

void ref_set_zone(void* p, int level, int left, int right, int up, int down, int num_rot, double inc_rot) {
  ptracker& t = static_cast<Handle*>(p)->trk;
  search_zone_type z{left, right, up, down, num_rot, inc_rot};
  if (level == 0) t.search_zone = z;
  else if (level == 1) t.search_zone_rescue = z;
  else t.search_zone_super_rescue = z;
}

// Scalar options of the command file (src/p-tracker.cpp:1487-1784).
int ref_set_param(void* p, const char* key, double v) {
  ptracker& t = static_cast<Handle*>(p)->trk;
  std::string k(key);
  if (k == "NCC_min") t.NCC_min = v;
  else if (k == "NCC_min_super") t.NCC_min_super = v;
  else if (k == "rescue_level") t.rescue_level = (int)v;
  else if (k == "subpixel") t.subpixel = (int)v;
  else if (k == "subpix_tol") t.subpix_tol = v;
  else if (k == "initial_direction_dx") t.initial_direction_dx = v;
  else if (k == "initial_direction_dy") t.initial_direction_dy = v;
  else if (k == "initial_direction_dr") t.initial_direction_dr = v;
  else if (k == "overflow_stiffness") t.overflow_stiffness = v;
  else if (k == "subpix_displacement_max") t.subpix_displacement_max = v;
  else if (k == "use_neighbour_list") t.use_neighbour_list = (int)v;
  else if (k == "neighbour_dist_pix") t.neighbour_dist_pix = v;
  else if (k == "period_rebuild_neighbour_list") t.period_rebuild_neighbour_list = (int)v;
  else if (k == "iref") t.iref = (int)v;
  else if (k == "iraz") t.iraz = (int)v;
  else if (k == "image_interpolator") {
    int kind = (int)v;
    t.IMAGE_INTERPOLATOR = kind == 0 ? (image_interpolator*)&t.IMAGE_INTERPOLATOR_LINEAR
                           : kind == 2 ? (image_interpolator*)&t.IMAGE_INTERPOLATOR_QUINTIC
                                       : (image_interpolator*)&t.IMAGE_INTERPOLATOR_CUBIC;
  } else return -1;
  return 0;
}

void ref_precompute(void* p) { static_cast<Handle*>(p)->trk.do_precomputations(); }

void ref_build_neighbours(void* p) {
  ptracker& t = static_cast<Handle*>(p)->trk;
  for (int i = 0; i < t.num_grains; ++i) {
    t.grain[i].neighbour.clear();
    t.find_neighbours(i);
  }
}

// Pixel stage (src/p-tracker.cpp:471-484).  Returns num_to_be_rescued.
int ref_pixel_all(void* p) {
  Handle* h = static_cast<Handle*>(p);
  ptracker& t = h->trk;
  set_threads(h);
  t.num_to_be_rescued = t.num_to_be_super_rescued = 0;
  int ig;
#pragma omp parallel for schedule(dynamic)
  for (ig = 0; ig < t.num_grains; ig++) {
    t.grain[ig].reset();
    t.grain[ig].backup();
    if (t.grain[ig].masked) continue;
    t.follow_pattern_pixel(ig);
  }
  return t.num_to_be_rescued;
}

// Pixel search of one grain only, without the reset/backup of the stage loop.
void ref_pixel_one(void* p, int ig) { static_cast<Handle*>(p)->trk.follow_pattern_pixel(ig); }

// Rescue stage (src/p-tracker.cpp:491-504).  Returns num_to_be_super_rescued.
int ref_rescue_all(void* p) {
  Handle* h = static_cast<Handle*>(p);
  ptracker& t = h->trk;
  set_threads(h);
  int ir, ig;
#pragma omp parallel for private(ig) schedule(dynamic)
  for (ir = 0; ir < t.num_to_be_rescued; ir++) {
    ig = t.to_be_rescued[ir];
    t.follow_pattern_rescue_pixel(ig);
  }
  return t.num_to_be_super_rescued;
}

// Super-rescue stage (src/p-tracker.cpp:524-536).
void ref_super_rescue_all(void* p) {
  Handle* h = static_cast<Handle*>(p);
  ptracker& t = h->trk;
  set_threads(h);
  int ir, ig;
#pragma omp parallel for private(ig) schedule(dynamic)
  for (ir = 0; ir < t.num_to_be_super_rescued; ir++) {
    ig = t.to_be_super_rescued[ir];
    t.follow_pattern_super_rescue_pixel(ig);
  }
}

int ref_get_lists(void* p, int* rescued, int* super_rescued, int* n_super) {
  ptracker& t = static_cast<Handle*>(p)->trk;
  for (int i = 0; i < t.num_to_be_rescued; ++i) rescued[i] = t.to_be_rescued[i];
  for (int i = 0; i < t.num_to_be_super_rescued; ++i) super_rescued[i] = t.to_be_super_rescued[i];
  *n_super = t.num_to_be_super_rescued;
  return t.num_to_be_rescued;
}

// Subpixel stage (src/p-tracker.cpp:558-572).
void ref_subpixel_all(void* p) {
  Handle* h = static_cast<Handle*>(p);
  ptracker& t = h->trk;
  set_threads(h);
  int ig;
#pragma omp parallel for schedule(dynamic)
  for (ig = 0; ig < t.num_grains; ig++) {
    if (t.grain[ig].masked) continue;
    t.follow_pattern_subpixel_xyR(ig);
  }
}

// Increments and reference change (src/p-tracker.cpp:577-611).
void ref_end_frame(void* p, int num_image) {
  ptracker& t = static_cast<Handle*>(p)->trk;
  for (int ig = 0; ig < t.num_grains; ig++) {
    t.grain[ig].upix = t.grain[ig].dx - t.grain[ig].dx_prev;
    t.grain[ig].vpix = t.grain[ig].dy - t.grain[ig].dy_prev;
    t.grain[ig].rot_inc = t.grain[ig].drot - t.grain[ig].drot_prev;
  }
  if (num_image - t.iref >= t.iraz) {
    int tmp = t.im_index_current;
    t.im_index_current = t.im_index_ref;
    t.im_index_ref = tmp;
    double actual_pos;
    for (int ig = 0; ig < t.num_grains; ig++) {
      actual_pos = (double)(t.grain[ig].refcoord_xpix) + t.grain[ig].dx;
      t.grain[ig].refcoord_xpix = std::round(actual_pos);
      t.grain[ig].dx = actual_pos - t.grain[ig].refcoord_xpix;
      actual_pos = (double)(t.grain[ig].refcoord_ypix) + t.grain[ig].dy;
      t.grain[ig].refcoord_ypix = std::round(actual_pos);
      t.grain[ig].dy = actual_pos - t.grain[ig].refcoord_ypix;
      t.grain[ig].refrot += t.grain[ig].drot;
      t.grain[ig].drot = 0.0;
    }
    t.iref = num_image;
    t.require_precomputations = true;
  }
}

// One frame of the particle_tracking loop body after the image read
// (src/p-tracker.cpp:458-611), file output excluded.
void ref_track_frame(void* p, int num_image) {
  Handle* h = static_cast<Handle*>(p);
  ptracker& t = h->trk;
  if (t.require_precomputations) t.do_precomputations();
  t.num_to_be_rescued = t.num_to_be_super_rescued = 0;
  if (t.rescue_level >= 0) ref_pixel_all(p);
  if (t.rescue_level >= 1) ref_rescue_all(p);
  if (t.rescue_level >= 2) ref_super_rescue_all(p);
  if (t.subpixel) ref_subpixel_all(p);
  ref_end_frame(p, num_image);
}

double ref_objective(void* p, int ig, const double* X3) {
  ptracker& t = static_cast<Handle*>(p)->trk;
  std::vector<double> X(X3, X3 + 3);
  t.igrain_of_thread[omp_get_thread_num()] = ig;
  return t.NCC_to_minimize_xyR(X);
}

// kind: 0 linear, 1 cubic, 2 quintic; slot indexes ptracker::image directly.
double ref_interp(void* p, int kind, int slot, double x, double y) {
  ptracker& t = static_cast<Handle*>(p)->trk;
  image_interpolator* ip = kind == 0 ? (image_interpolator*)&t.IMAGE_INTERPOLATOR_LINEAR
                           : kind == 2 ? (image_interpolator*)&t.IMAGE_INTERPOLATOR_QUINTIC
                                       : (image_interpolator*)&t.IMAGE_INTERPOLATOR_CUBIC;
  return ip->getValue(t.image[slot], x, y);
}

void ref_undistor(void* p, const double* params14, double xd, double yd, double* xu, double* yu) {
  ptracker& t = static_cast<Handle*>(p)->trk;
  std::vector<double> X(params14, params14 + 14);
  t.undistor(X, xd, yd, *xu, *yu);
}

// ptracker::precompute_paires (src/distortion_correction.cpp:63-81) on grains
// placed at the given reference positions; writes at most cap pairs.
int64_t ref_disto_pairs(void* p, const int32_t* refx, const int32_t* refy, int n, double dmin, double dmax,
                        int32_t* out, int64_t cap) {
  ptracker& t = static_cast<Handle*>(p)->trk;
  t.grain.assign(n, grain_type_2D());
  for (int g = 0; g < n; ++g) {
    t.grain[g].refcoord_xpix = refx[g];
    t.grain[g].refcoord_ypix = refy[g];
  }
  t.num_grains = n;
  t.equiProj_dist_min = dmin;
  t.equiProj_dist_max = dmax;
  t.precompute_paires();
  const int64_t np = (int64_t)t.grain_pairs.size();
  for (int64_t k = 0; k < np && k < cap; ++k) {
    out[2 * k] = t.grain_pairs[k].i;
    out[2 * k + 1] = t.grain_pairs[k].j;
  }
  return np;
}

// The POWELL functor of correction_distortion (src/distortion_correction.cpp:
// 249-290) restated around the reference's ptracker::undistor; use_orig selects
// the POWELL_ITER functor (:318-351, A1 and B1 from origx/origy).
double ref_disto_objective(void* p, const double* X14, const int32_t* refx, const int32_t* refy, const double* origx,
                           const double* origy, int n, int nimg1, const double* dx, const double* dy,
                           const double* ncc, double NCC_min, const int32_t* pairs, int64_t npairs, int use_orig) {
  ptracker& t = static_cast<Handle*>(p)->trk;
  std::vector<double> X(X14, X14 + 14);
  double valret = 0.0;
  for (int im = 0; im < nimg1; ++im)
    for (int64_t il = 0; il < npairs; ++il) {
      const int i = pairs[2 * il], j = pairs[2 * il + 1];
      if (ncc[(size_t)im * n + i] < NCC_min || ncc[(size_t)im * n + j] < NCC_min) continue;
      double A1x, A1y, A2x, A2y, B1x, B1y, B2x, B2y;
      if (use_orig) {
        A1x = origx[i];
        A1y = origy[i];
        B1x = origx[j];
        B1y = origy[j];
      } else {
        t.undistor(X, (double)(refx[i]), (double)(refy[i]), A1x, A1y);
        t.undistor(X, (double)(refx[j]), (double)(refy[j]), B1x, B1y);
      }
      t.undistor(X, (double)(refx[i] + dx[(size_t)im * n + i]), (double)(refy[i] + dy[(size_t)im * n + i]), A2x, A2y);
      t.undistor(X, (double)(refx[j] + dx[(size_t)im * n + j]), (double)(refy[j] + dy[(size_t)im * n + j]), B2x, B2y);
      double ABx = B1x - A1x, ABy = B1y - A1y;
      const double AB = sqrt(ABx * ABx + ABy * ABy);
      ABx /= AB;
      ABy /= AB;
      const double BBx = B2x - B1x, BBy = B2y - B1y, AAx = A2x - A1x, AAy = A2y - A1y;
      const double err = (ABx * (BBx - AAx)) + (ABy * (BBy - AAy));
      valret += err * err;
    }
  return valret;
}

int ref_save_grains(void* p, const char* path, int num) {
  return static_cast<Handle*>(p)->trk.save_grains(path, num);
}

int ref_read_grains(void* p, const char* path, int ptracker_format) {
  ptracker& t = static_cast<Handle*>(p)->trk;
  t.read_grains(path, ptracker_format != 0);
  t.require_precomputations = true;
  return t.num_grains;
}

int ref_num_grains(void* p) { return static_cast<Handle*>(p)->trk.num_grains; }

// ptracker::make_grid (src/p-tracker.cpp:1280-1311) from the C library's
// first random numbers (srand(1), the sequence a fresh process starts with);
// returns the grain count, positions in xy (2 ints per grain).
int ref_make_grid(void* p, double xmin, double xmax, double ymin, double ymax, int nx, int ny, int alea_max,
                  int32_t* xy) {
  ptracker& t = static_cast<Handle*>(p)->trk;
  std::srand(1);
  t.make_grid(xmin, xmax, ymin, ymax, nx, ny, alea_max);
  for (int g = 0; g < t.num_grains; ++g) {
    xy[2 * g] = t.grain[g].refcoord_xpix;
    xy[2 * g + 1] = t.grain[g].refcoord_ypix;
  }
  return t.num_grains;
}

// ptracker::check_distortion (src/check_distortion.cpp:25-100) in the current
// directory: reads the dic files dic_name % iref and % ibeg..iend (step iinc)
// and writes len_variation.txt.
void ref_check_distortion(void* p, const char* dic_name, int iref, int ibeg, int iend, int iinc,
                          const double* params14) {
  ptracker& t = static_cast<Handle*>(p)->trk;
  std::strncpy(t.dic_name, dic_name, sizeof(t.dic_name) - 1);
  t.dic_name[sizeof(t.dic_name) - 1] = '\0';
  t.iref = iref;
  t.ibeg = ibeg;
  t.iend = iend;
  t.iinc = iinc;
  t.disto_parameters.assign(params14, params14 + 14);
  t.check_distortion();
}

// ptracker::read_raw_image (src/p-tracker.cpp:214-387) run on an unpacked
// sensor mosaic (raw_width x raw_height, row-major) registered with the
// libraw stub; the visible width x height frame is read back row-major into
// out (slot 0; first_time, so the reference also sizes dimx/dimy from it).
void ref_raw_demosaic(void* p, const uint16_t* raw, int raw_width, int raw_height, int width, int height,
                      int left_margin, int top_margin, int mode, int rescale, uint16_t* out) {
  ptracker& t = static_cast<Handle*>(p)->trk;
  std::vector<uint16_t> copy(raw, raw + (size_t)raw_width * raw_height);
  libraw_stub_data& src = libraw_stub_source();
  src = libraw_stub_data{};
  src.sizes.width = width;
  src.sizes.height = height;
  src.sizes.raw_width = raw_width;
  src.sizes.left_margin = left_margin;
  src.sizes.top_margin = top_margin;
  src.color.maximum = 65535;
  src.rawdata.raw_image = copy.data();
  t.DemosaicModel = mode;
  t.rescaleGrayLevels = rescale;
  t.read_raw_image(0, "mosaic", true);
  src.rawdata.raw_image = nullptr;
  for (int y = 0; y < height; ++y)
    for (int x = 0; x < width; ++x) out[(size_t)y * width + x] = t.image[0][x][y];
}

}  // extern "C"
