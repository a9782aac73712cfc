// ptracker_b200: the particle_tracking and correction_distortion procedures
// of `ptracker <command_file>` (src/p-tracker.cpp:422-612,
// src/distortion_correction.cpp:135-607, run.cpp) driven through the C ABI of
// this library, for one GPU.
//
// Command file: the reference's token stream (read_data,
// src/p-tracker.cpp:1487-1784): whitespace-separated tokens, '#' or '!' starts
// a comment to the end of the line, unknown tokens are reported and skipped.
// Grain files, `make_grid`, `pattern`, `targetRadiusPattern` and `mask_rect`
// act on the grains loaded so far, in file order, as they do in the reference.  Tokens of
// other features (RAW decoding, neighbour lists, thread counts) are accepted
// and have no effect.  Added tokens select the forms of this library:
//     search_method  exact | bf16          integer search (default exact)
//     subpix_method  powell | adjoint_lm   subpixel refinement (default powell)
//     topk K, lm_max_iter N, lm_tol T      their parameters
//     lm_cell PX STEPS                    LM results beyond this cell go to Powell (0 0: none)
//     autotune 0 | 1                       time the level-0 search shapes
//                                          before the first frame (ptk_autotune)
//     autotune_cache FILE                  JSON file of autotune choices per GPU
//                                          and workload (ptk_set_tune_cache)
//     undistort_images 0 | 1               resample every frame with the
//                                          *_corrDistor / *_corrParallax
//                                          parameters before tracking
//
// Frames: image_name is a printf pattern of the frame number (read_image,
// src/p-tracker.cpp:75-83); frames are strip TIFF (uncompressed, LZW,
// Deflate or PackBits; converted as the reference's libtiff RGBA path) or
// binary PGM.  The next frame is decoded on
// a host thread while the GPU tracks the current one.  After every frame the
// grains go to dic_out_<num>.txt in the working directory, byte for byte as
// save_grains (src/p-tracker.cpp:1313-1367).
//
// `procedure correction_distortion` tracks image_numbers_corrDisto[1..]
// against image_numbers_corrDisto[0] (pixel search from the imposed
// approximate displacements, no rescue, then subpixel; dic_out_<num>.txt per
// image), then fits the 14 undistor parameters with ptk_disto_fit (POWELL,
// POWELL_ITER or LEVMAR) and writes
// corrDisto_log.txt, errors.txt, distobox.txt and, for POWELL_ITER,
// convergence.txt as the reference does.
//
// `procedure check_distortion` (src/check_distortion.cpp:25-100; declared by
// the reference but neither dispatched by its run() nor built by its
// Makefile) reads dic_name % iref and % ibeg..iend and writes the mean length
// drift of the segments joining grains 0-1, 2-3, ..., raw and undistorted, to
// len_variation.txt.  It needs no GPU.
//
//   ptracker_b200 [command_file]     (default: commands.txt)
//   ptracker_b200 --check file       parse only; print the settings as JSON
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <fstream>
#include <future>
#include <iomanip>
#include <iostream>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/ptk.h"

namespace {

struct PatternOp {
  int kind;  // PTK_PATTERN_*, or -1 for a pattern file
  double a, b, target;
  std::string file;
};

struct Settings {
  std::string image_name = "%d.tif", dic_name, procedure = "particle_tracking", tune_cache;
  int iref = 0, ibeg = 0, iend = 0, iinc = 0;
  int raw_images = 0, undistort = 0;
  ptk_config cfg;
  double target_radius = -1.0;
  // undistor parameters (defaults of ptracker::ptracker, src/p-tracker.cpp:
  // 22-52: negative centres stand for the frame centre) and the fit's
  // perturbations
  double disto[14] = {-1.0, -1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, -1.0, -1.0, 0.0, 0.0, 0.0, 0.0};
  double disto_perturb[14] = {1e-6, 1e-6, 1e-6, 1e-6, 1e-6, 1e-6, 1e-6, 1e-6, 1e-6, 1e-6, 1e-6, 1e-6, 1e-6, 1e-6};
  std::vector<int> corr_images;
  std::vector<double> imposed_x, imposed_y;
  double equiproj_min = 0.0, equiproj_max = 1000.0;
  int optim_algo = PTK_DISTO_POWELL, powell_num_iter = 5;
  std::vector<ptk_grain> grains;
  std::vector<PatternOp> patterns;  // acting on the grains loaded last
  std::vector<std::string> warnings;
  int unknown_tokens = 0;
};

// Frame buffers in page-locked memory, reused across frames (the decode
// thread takes one while the GPU still uploads from another), so uploads are
// asynchronous and run at full link speed; ordinary heap memory when pinned
// memory cannot be had.
class BufferPool {
 public:
  ~BufferPool() {
    for (Buf& b : free_) release(b);
  }
  std::shared_ptr<uint16_t> get(size_t elems) {
    Buf b{nullptr, 0, false};
    {
      std::lock_guard<std::mutex> lock(m_);
      for (size_t i = 0; i < free_.size(); ++i)
        if (free_[i].elems >= elems) {
          b = free_[i];
          free_.erase(free_.begin() + (long)i);
          break;
        }
    }
    if (!b.p) {
      void* p = nullptr;
      if (ptk_host_alloc(&p, elems * sizeof(uint16_t)) == PTK_OK) {
        b = Buf{static_cast<uint16_t*>(p), elems, true};
      } else {
        b = Buf{new uint16_t[elems], elems, false};
      }
    }
    return std::shared_ptr<uint16_t>(b.p, [this, b](uint16_t*) {
      std::lock_guard<std::mutex> lock(m_);
      free_.push_back(b);
    });
  }

 private:
  struct Buf {
    uint16_t* p;
    size_t elems;
    bool pinned;
  };
  static void release(const Buf& b) {
    if (b.pinned) ptk_host_free(b.p);
    else delete[] b.p;
  }
  std::mutex m_;
  std::vector<Buf> free_;
};

struct Frame {
  std::shared_ptr<uint16_t> pix;  // dimx x dimy grey levels, from the pool
  int dimx = 0, dimy = 0;
  std::string datetime, name;
  int rc = PTK_OK;
  std::string error;
};

std::string frame_name(const std::string& pattern, int num) {
  char buf[4096];
  std::snprintf(buf, sizeof(buf), pattern.c_str(), num);
  return buf;
}

// expect: the size of the frames read so far (0: unknown); a frame of that
// size is read from disk once, any other after a size query.
Frame read_frame(BufferPool* pool, const std::string& pattern, int num, size_t expect) {
  Frame f;
  f.name = frame_name(pattern, num);
  char when[256];
  if (expect > 0) {
    f.pix = pool->get(expect);
    f.rc = ptk_read_image_file(f.name.c_str(), f.pix.get(), expect, &f.dimx, &f.dimy, when, sizeof(when));
    if (f.rc == PTK_OK) {
      f.datetime = when;
      return f;
    }
    f.pix.reset();
  }
  f.rc = ptk_read_image_file(f.name.c_str(), nullptr, 0, &f.dimx, &f.dimy, nullptr, 0);
  if (f.rc == PTK_OK) {
    const size_t elems = (size_t)f.dimx * f.dimy;
    f.pix = pool->get(elems);
    f.rc = ptk_read_image_file(f.name.c_str(), f.pix.get(), elems, &f.dimx, &f.dimy, when, sizeof(when));
    f.datetime = when;
  }
  if (f.rc) f.error = ptk_image_error();
  return f;
}

[[noreturn]] void die(const std::string& msg) {
  std::fprintf(stderr, "ptracker_b200: %s\n", msg.c_str());
  std::exit(EXIT_FAILURE);
}

void load_grains(Settings& s, const std::string& path, bool format13) {
  int n = 0;
  if (ptk_read_grains_file(path.c_str(), format13 ? 1 : 0, nullptr, 0, &n)) die("cannot read grain file " + path);
  s.grains.assign((size_t)n, ptk_grain{});
  if (n && ptk_read_grains_file(path.c_str(), format13 ? 1 : 0, s.grains.data(), n, &n))
    die("cannot read grain file " + path);
  s.patterns.clear();  // the reference rebuilds its grain vector: earlier patterns are gone
}

// make_grid (src/p-tracker.cpp:1280-1311): nx x ny grains on a grid of
// integer steps floor((max - min) / (n - 1)) from (xmin, ymin), each moved
// by round(alea (cos a, sin a)) with a and alea drawn from the C library's
// rand() in the reference's order (an angle, then a distance up to aleaMax),
// refcoord truncated to int as its assignment does; refrot 0, radius 2 px.
// The grains replace the ones loaded so far (and their patterns).
void make_grid(Settings& s, double xmin, double xmax, double ymin, double ymax, int nx, int ny, int alea_max) {
  if (nx < 2 || ny < 2) die("make_grid needs at least 2 points in each direction");
  const int dx = (int)std::floor((xmax - xmin) / (double)(nx - 1));
  const int dy = (int)std::floor((ymax - ymin) / (double)(ny - 1));
  s.grains.assign((size_t)nx * ny, ptk_grain{});
  size_t i = 0;
  for (int iy = 0; iy < ny; ++iy)
    for (int ix = 0; ix < nx; ++ix) {
      const double angle = (double)std::rand() / (double)RAND_MAX * (2.0 * M_PI);
      const double alea = (double)std::rand() / (double)RAND_MAX * alea_max;
      ptk_grain& g = s.grains[i++];
      g.refcoord_xpix = (int32_t)(xmin + ix * dx + (int)std::round(alea * std::cos(angle)));
      g.refcoord_ypix = (int32_t)(ymin + iy * dy + (int)std::round(alea * std::sin(angle)));
      g.refrot = 0.0;
      g.radius_pix = 2.0;
    }
  s.patterns.clear();
  std::printf("Create grid with %d points\n", nx * ny);
}

// The reference's token loop (read_data); values are read with operator>> as
// there.
Settings read_commands(const char* path) {
  Settings s;
  ptk_config_default(&s.cfg);
  std::ifstream in(path);
  if (!in) die(std::string("cannot open command file ") + path);
  std::string tok;
  auto skip = [&](int n) {
    std::string t;
    for (int i = 0; i < n; ++i) in >> t;
  };
  while (in >> tok) {
    if (tok[0] == '!' || tok[0] == '#') {
      std::getline(in, tok);
    } else if (tok == "image_name") {
      in >> s.image_name;
    } else if (tok == "dic_name") {
      in >> s.dic_name;
    } else if (tok == "RawImages") {
      in >> s.raw_images;
    } else if (tok == "DemosaicModel" || tok == "rescaleGrayLevels" || tok == "idelta" ||
               tok == "wanted_num_threads" || tok == "verbose_level" || tok == "num_neighbour_max" ||
               tok == "neighbour_dist_pix" || tok == "period_rebuild_neighbour_list" || tok == "use_neighbour_list") {
      skip(1);
    } else if (tok == "powell_num_iter") {
      in >> s.powell_num_iter;
    } else if (tok == "optim_algo") {  // src/p-tracker.cpp:1553-1564
      std::string k;
      in >> k;
      if (k == "POWELL") s.optim_algo = PTK_DISTO_POWELL;
      else if (k == "POWELL_ITER") s.optim_algo = PTK_DISTO_POWELL_ITER;
      else if (k == "LEVMAR") s.optim_algo = PTK_DISTO_LEVMAR;
      else std::printf("WARNING, keyword %s is unknown for optim_algo\n", k.c_str());
    } else if (tok == "grains_to_follow" || tok == "start_file") {
      std::string f;
      in >> f;
      load_grains(s, f, false);
    } else if (tok == "restart_file") {
      std::string f;
      in >> f;
      load_grains(s, f, true);
    } else if (tok == "make_grid") {  // src/p-tracker.cpp:1519-1525
      double xmin, xmax, ymin, ymax;
      int nx, ny, alea_max;
      in >> xmin >> xmax >> ymin >> ymax >> nx >> ny >> alea_max;
      make_grid(s, xmin, xmax, ymin, ymax, nx, ny, alea_max);
    } else if (tok == "iref") {
      in >> s.iref;
    } else if (tok == "ibeg") {
      in >> s.ibeg;
    } else if (tok == "iend") {
      in >> s.iend;
    } else if (tok == "iinc") {
      in >> s.iinc;
    } else if (tok == "iraz") {
      in >> s.cfg.iraz;
    } else if (tok == "procedure") {
      in >> s.procedure;
    } else if (tok == "rescue_level") {
      in >> s.cfg.rescue_level;
    } else if (tok == "subpixel") {
      in >> s.cfg.subpixel;
    } else if (tok == "rotations") {
      in >> s.cfg.rotations;
    } else if (tok == "image_interpolator") {
      std::string k;
      in >> k;
      if (k == "linear") s.cfg.image_interpolator = PTK_INTERP_LINEAR;
      else if (k == "cubic") s.cfg.image_interpolator = PTK_INTERP_CUBIC;
      else if (k == "quintic") s.cfg.image_interpolator = PTK_INTERP_QUINTIC;
    } else if (tok == "subpix_tol") {
      in >> s.cfg.subpix_tol;
    } else if (tok == "initial_direction_dx") {
      in >> s.cfg.initial_direction[0];
    } else if (tok == "initial_direction_dy") {
      in >> s.cfg.initial_direction[1];
    } else if (tok == "initial_direction_dr") {
      in >> s.cfg.initial_direction[2];
    } else if (tok == "overflow_stiffness") {
      in >> s.cfg.overflow_stiffness;
    } else if (tok == "subpix_displacement_max") {
      in >> s.cfg.subpix_displacement_max;
    } else if (tok == "NCC_min") {
      in >> s.cfg.NCC_min;
    } else if (tok == "NCC_min_super") {
      in >> s.cfg.NCC_min_super;
    } else if (tok.rfind("search_zone", 0) == 0 && tok.find('.') != std::string::npos) {
      const std::string zone = tok.substr(0, tok.find('.')), field = tok.substr(tok.find('.') + 1);
      const int lvl = zone == "search_zone" ? 0 : zone == "search_zone_rescue" ? 1
                    : zone == "search_zone_super_rescue" ? 2 : -1;
      ptk_zone* z = lvl >= 0 ? &s.cfg.zone[lvl] : nullptr;
      if (z && field == "left") in >> z->left;
      else if (z && field == "right") in >> z->right;
      else if (z && field == "up") in >> z->up;
      else if (z && field == "down") in >> z->down;
      else if (z && field == "inc_rot") in >> z->inc_rot;
      else if (z && field == "num_rot") in >> z->num_rot;
      else {
        std::printf("Unknown token: %s\n", tok.c_str());
        ++s.unknown_tokens;
      }
    } else if (tok == "targetRadiusPattern") {
      in >> s.target_radius;
    } else if (tok == "pattern") {
      std::string k;
      in >> k;
      PatternOp op{PTK_PATTERN_CIRC, 0.0, 0.0, s.target_radius, ""};
      if (k == "circ") {
        int r;
        in >> r;
        op.a = r;
      } else if (k == "grain_diameter") {
        op.kind = PTK_PATTERN_GRAIN_DIAMETER;
        in >> op.a >> op.b;
      } else if (k == "ring") {
        int r0, r1;
        in >> r0 >> r1;
        op.kind = PTK_PATTERN_RING;
        op.a = r0;
        op.b = r1;
      } else if (k == "rect") {
        int hw, hh;
        in >> hw >> hh;
        op.kind = PTK_PATTERN_RECT;
        op.a = hw;
        op.b = hh;
      } else if (k == "file") {
        op.kind = -1;
        in >> op.file;
      } else {
        s.warnings.push_back("unknown pattern kind " + k);
        continue;
      }
      s.patterns.push_back(op);
    } else if (tok == "mask_rect") {
      int x0, x1, y0, y1;
      in >> x0 >> x1 >> y0 >> y1;
      for (ptk_grain& g : s.grains)
        if (g.refcoord_xpix >= x0 && g.refcoord_xpix <= x1 && g.refcoord_ypix >= y0 && g.refcoord_ypix <= y1)
          g.masked = 1;
    } else if (tok == "image_numbers_corrDisto") {  // src/p-tracker.cpp:1696-1702
      size_t nb = 0;
      in >> nb;
      s.corr_images.assign(nb, 0);
      for (size_t i = 0; i < nb; ++i) in >> s.corr_images[i];
    } else if (tok == "imposedDisplApprox_corrDisto") {  // :1703-1710, one pair per image after the first
      s.imposed_x.assign(s.corr_images.size(), 0.0);
      s.imposed_y.assign(s.corr_images.size(), 0.0);
      for (size_t i = 1; i < s.corr_images.size(); ++i) in >> s.imposed_x[i] >> s.imposed_y[i];
    } else if (tok == "equiProj_dist_range") {
      in >> s.equiproj_min >> s.equiproj_max;
    } else if (tok.size() > 11 && (tok.find("_corrDistor") != std::string::npos ||
                                   tok.find("_corrParallax") != std::string::npos)) {
      static const char* names[14] = {"xc_corrDistor", "yc_corrDistor", "K1_corrDistor", "K2_corrDistor",
                                      "K3_corrDistor", "P1_corrDistor", "P2_corrDistor", "P3_corrDistor",
                                      "xc_corrParallax", "yc_corrParallax", "angle1_corrParallax",
                                      "A1_corrParallax", "angle2_corrParallax", "A2_corrParallax"};
      int k = -1, kd = -1;
      for (int i = 0; i < 14; ++i) {
        if (tok == names[i]) k = i;
        if (tok == std::string("d") + names[i]) kd = i;
      }
      double v;
      in >> v;
      if (k >= 0) s.disto[k] = v;
      else if (kd >= 0) s.disto_perturb[kd] = v;
      else {
        std::printf("Unknown token: %s\n", tok.c_str());
        ++s.unknown_tokens;
      }
    } else if (tok == "search_method") {
      std::string k;
      in >> k;
      if (k == "bf16") s.cfg.search_method = PTK_SEARCH_BF16;
      else if (k == "exact") s.cfg.search_method = PTK_SEARCH_EXACT;
      else s.warnings.push_back("unknown search_method " + k);
    } else if (tok == "subpix_method") {
      std::string k;
      in >> k;
      if (k == "adjoint_lm") s.cfg.subpix_method = PTK_SUBPIX_ADJOINT_LM;
      else if (k == "powell") s.cfg.subpix_method = PTK_SUBPIX_POWELL;
      else s.warnings.push_back("unknown subpix_method " + k);
    } else if (tok == "topk") {
      in >> s.cfg.topk;
    } else if (tok == "lm_max_iter") {
      in >> s.cfg.lm_max_iter;
    } else if (tok == "lm_tol") {
      in >> s.cfg.lm_tol;
    } else if (tok == "lm_cell") {  // pixels, rotation steps (0 0: keep every LM result)
      in >> s.cfg.lm_cell_px >> s.cfg.lm_cell_rot;
    } else if (tok == "autotune") {
      in >> s.cfg.autotune;
    } else if (tok == "autotune_cache") {
      in >> s.tune_cache;
    } else if (tok == "undistort_images") {
      in >> s.undistort;
    } else {
      std::printf("Unknown token: %s\n", tok.c_str());
      ++s.unknown_tokens;
    }
  }
  return s;
}

// `pattern file` (make_custom_pattern, src/p-tracker.cpp:1443-1476): the
// count of patterns (must equal the grain count), then per grain its count of
// offsets and the dx dy pairs.
void read_pattern_file(const std::string& path, int n_grains, std::vector<int32_t>* xy, std::vector<int64_t>* starts) {
  std::ifstream f(path);
  if (!f) die("cannot open pattern file " + path);
  int n = 0;
  f >> n;
  if (n != n_grains) die("the number of patterns is not equal to the number of grains");
  starts->assign(1, 0);
  for (int g = 0; g < n; ++g) {
    int k = 0;
    f >> k;
    for (int i = 0; i < k; ++i) {
      int dx, dy;
      f >> dx >> dy;
      xy->push_back(dx);
      xy->push_back(dy);
    }
    starts->push_back((int64_t)(xy->size() / 2));
  }
  if (!f) die("truncated pattern file " + path);
}

void print_json(const Settings& s) {
  const ptk_config& c = s.cfg;
  std::ostringstream o;
  o.precision(17);
  o << "{\"image_name\": \"" << s.image_name << "\", \"iref\": " << s.iref << ", \"ibeg\": " << s.ibeg
    << ", \"iend\": " << s.iend << ", \"iinc\": " << s.iinc << ", \"iraz\": " << c.iraz
    << ", \"procedure\": \"" << s.procedure << "\", \"grains\": " << s.grains.size();
  int masked = 0;
  for (const ptk_grain& g : s.grains) masked += g.masked ? 1 : 0;
  o << ", \"grain_xy\": [";
  for (size_t i = 0; i < s.grains.size(); ++i)
    o << (i ? ", " : "") << "[" << s.grains[i].refcoord_xpix << ", " << s.grains[i].refcoord_ypix << "]";
  o << "], \"masked\": " << masked << ", \"rescue_level\": " << c.rescue_level << ", \"NCC_min\": " << c.NCC_min
    << ", \"NCC_min_super\": " << c.NCC_min_super << ", \"subpixel\": " << c.subpixel
    << ", \"subpix_tol\": " << c.subpix_tol << ", \"initial_direction\": [" << c.initial_direction[0] << ", "
    << c.initial_direction[1] << ", " << c.initial_direction[2] << "], \"image_interpolator\": "
    << c.image_interpolator << ", \"overflow_stiffness\": " << c.overflow_stiffness
    << ", \"subpix_displacement_max\": " << c.subpix_displacement_max << ", \"rotations\": " << c.rotations
    << ", \"zones\": [";
  for (int l = 0; l < 3; ++l)
    o << (l ? ", " : "") << "[" << c.zone[l].left << ", " << c.zone[l].right << ", " << c.zone[l].up << ", "
      << c.zone[l].down << ", " << c.zone[l].num_rot << ", " << c.zone[l].inc_rot << "]";
  o << "], \"patterns\": [";
  for (size_t i = 0; i < s.patterns.size(); ++i)
    o << (i ? ", " : "") << "[" << s.patterns[i].kind << ", " << s.patterns[i].a << ", " << s.patterns[i].b << ", "
      << s.patterns[i].target << ", \"" << s.patterns[i].file << "\"]";
  o << "], \"search_method\": " << c.search_method << ", \"autotune\": " << c.autotune
    << ", \"autotune_cache\": \"" << s.tune_cache << "\""
    << ", \"subpix_method\": " << c.subpix_method
    << ", \"undistort_images\": " << s.undistort << ", \"disto\": [";
  for (int k = 0; k < 14; ++k) o << (k ? ", " : "") << s.disto[k];
  o << "], \"disto_perturb\": [";
  for (int k = 0; k < 14; ++k) o << (k ? ", " : "") << s.disto_perturb[k];
  o << "], \"corr_images\": [";
  for (size_t i = 0; i < s.corr_images.size(); ++i) o << (i ? ", " : "") << s.corr_images[i];
  o << "], \"imposed\": [";
  for (size_t i = 0; i < s.imposed_x.size(); ++i)
    o << (i ? ", " : "") << "[" << s.imposed_x[i] << ", " << s.imposed_y[i] << "]";
  o << "], \"equiproj_range\": [" << s.equiproj_min << ", " << s.equiproj_max << "], \"optim_algo\": "
    << s.optim_algo << ", \"powell_num_iter\": " << s.powell_num_iter;
  o << ", \"unknown_tokens\": " << s.unknown_tokens << ", \"warnings\": " << s.warnings.size() << "}";
  std::printf("%s\n", o.str().c_str());
}

double now() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// undistor (src/distortion_correction.cpp:20-61) on the host, for the
// procedure's output files.
void undistor_host(const double* X, double xd, double yd, double* xo, double* yo) {
  const double dx = xd - X[0], dy = yd - X[1];
  const double r2 = dx * dx + dy * dy, r4 = r2 * r2, r6 = r4 * r2;
  const double xu = xd + dx * (X[2] * r2 + X[3] * r4 + X[4] * r6) +
                    (X[5] * (r2 + 2.0 * dx * dx) + 2.0 * X[6] * dx * dy) * (1.0 + X[7] * r2);
  const double yu = yd + dy * (X[2] * r2 + X[3] * r4 + X[4] * r6) +
                    (2.0 * X[5] * dx * dy + X[6] * (r2 + 2.0 * dy * dy)) * (1.0 + X[7] * r2);
  const double nx1 = std::cos(X[10]), ny1 = -std::sin(X[10]), nx2 = -std::sin(X[12]), ny2 = std::cos(X[12]);
  const double dX = xu - X[8], dY = yu - X[9];
  const double S1 = (1.0 + X[11]) * (dX * nx1 + dY * ny1);
  const double S2 = (1.0 + X[13]) * (dX * nx2 + dY * ny2);
  *xo = X[8] + S1 * nx1 + S2 * nx2;
  *yo = X[9] + S1 * ny1 + S2 * ny2;
}

// Negative centres stand for the frame centre (src/distortion_correction.cpp:222-226).
void default_centres(double* X, int dimx, int dimy) {
  if (X[0] < 0.0) X[0] = 0.5 * (double)dimx;
  if (X[1] < 0.0) X[1] = 0.5 * (double)dimy;
  if (X[8] < 0.0) X[8] = 0.5 * (double)dimx;
  if (X[9] < 0.0) X[9] = 0.5 * (double)dimy;
}

// The output files and console lines after the minimisation
// (src/distortion_correction.cpp:480-607).
void write_disto_outputs(const double* X, double index_ini, double index_end, int dimx, int dimy) {
  static const char* labels[14] = {"xc_corrDistor ",       "yc_corrDistor ",       "K1_corrDistor ",
                                   "K2_corrDistor ",       "K3_corrDistor ",       "P1_corrDistor ",
                                   "P2_corrDistor ",       "P3_corrDistor ",       "xc_corrParallax     ",
                                   "yc_corrParallax     ", "angle1_corrParallax ", "A1_corrParallax     ",
                                   "angle2_corrParallax ", "A2_corrParallax     "};
  const double gain = index_ini / index_end;
  std::ofstream log("corrDisto_log.txt");
  log << std::scientific << std::setprecision(15);
  log << "Initial distorsion index " << index_ini << '\n';
  log << "Final distorsion index " << index_end << '\n';
  log << "Index gain (>1 is good) " << gain << '\n';
  for (int k = 0; k < 14; ++k) log << labels[k] << X[k] << (k == 13 ? "" : "\n");
  log << std::endl;
  std::cout << std::scientific << std::setprecision(15);
  std::cout << "    Initial distorsion index " << index_ini << '\n';
  std::cout << "      Final distorsion index " << index_end << '\n';
  std::cout << "gain (index_ini / index_end) " << gain << " (>1 is good)" << '\n';
  for (int k = 0; k < 14; ++k) std::cout << labels[k] << X[k] << (k == 13 ? "" : "\n");
  std::cout << std::endl;

  std::ofstream ef("errors.txt");
  double xerrmax = -1e20, yerrmax = -1e20, errmax = -1e20, xd, yd, xu, yu;
  double dxd = (double)dimx / 50.0, dyd = (double)dimy / 50.0;
  if (dxd < 1.0) dxd = 1.0;
  if (dyd < 1.0) dyd = 1.0;
  for (xd = 0.0; xd < dimx; xd += dxd) {
    for (yd = 0.0; yd < dimy; yd += dyd) {
      undistor_host(X, xd, yd, &xu, &yu);
      const double xerr = xu - xd, yerr = yu - yd, err = std::sqrt(xerr * xerr + yerr * yerr);
      if (std::fabs(xerr) > xerrmax) xerrmax = std::fabs(xerr);
      if (std::fabs(yerr) > yerrmax) yerrmax = std::fabs(yerr);
      if (err > errmax) errmax = err;
      ef << xd << ' ' << yd << ' ' << xerr << ' ' << yerr << std::endl;
    }
    ef << std::endl;
  }
  log << "max |xu - xd| " << xerrmax << '\n';
  log << "max |yu - yd| " << yerrmax << '\n';
  log << "errormax " << errmax << std::endl;
  std::cout << "max |xu - xd| " << xerrmax << '\n';
  std::cout << "max |yu - yd| " << yerrmax << '\n';
  std::cout << "errormax      " << errmax << std::endl;

  std::ofstream bf("distobox.txt");
  auto box = [&](double x, double y) {
    undistor_host(X, x, y, &xu, &yu);
    bf << x << " " << y << " " << xu - x << " " << yu - y << std::endl;
  };
  yd = 0;
  for (xd = 0; xd < dimx; xd += dxd) box(xd, yd);
  xd = dimx - 1;
  for (yd = 0; yd < dimy; yd += dyd) box(xd, yd);
  yd = dimy - 1;
  for (xd = dimx - 1; xd >= 0; xd -= dxd) box(xd, yd);
  xd = 0;
  for (yd = dimy - 1; yd >= 0; yd -= dyd) box(xd, yd);
  box(0.0, 0.0);
}

// check_distortion (src/check_distortion.cpp:25-100): per dic file, the
// mean over segments (grains 2k, 2k + 1) of (L - L0) / L0, with L0 the
// segment's length in the file of image iref, for the positions as tracked
// and through undistor with the *_corrDistor / *_corrParallax parameters as
// given; one line "idic mean mean_undistorted" per file.  A last grain
// without a partner is left out (the reference reads past its grain array).
int check_distortion(const Settings& s) {
  const std::string pat = s.dic_name.empty() ? std::string("dic_out_%d.txt") : s.dic_name;
  auto lengths = [&](int num, std::vector<double>& raw, std::vector<double>& und) {
    char name[512];
    std::snprintf(name, sizeof(name), pat.c_str(), num);
    int n = 0;
    if (ptk_read_grains_file(name, 1, nullptr, 0, &n)) die(std::string("cannot read ") + name);
    std::vector<ptk_grain> g((size_t)n);
    if (n > 0 && ptk_read_grains_file(name, 1, g.data(), n, &n)) die(std::string("cannot read ") + name);
    raw.clear();
    und.clear();
    for (int k = 0; k + 1 < n; k += 2) {
      double xb = (double)g[k].refcoord_xpix + g[k].dx, yb = (double)g[k].refcoord_ypix + g[k].dy;
      double xe = (double)g[k + 1].refcoord_xpix + g[k + 1].dx, ye = (double)g[k + 1].refcoord_ypix + g[k + 1].dy;
      double sx = xe - xb, sy = ye - yb;
      raw.push_back(std::sqrt(sx * sx + sy * sy));
      undistor_host(s.disto, (double)g[k].refcoord_xpix + g[k].dx, (double)g[k].refcoord_ypix + g[k].dy, &xb, &yb);
      undistor_host(s.disto, (double)g[k + 1].refcoord_xpix + g[k + 1].dx,
                    (double)g[k + 1].refcoord_ypix + g[k + 1].dy, &xe, &ye);
      sx = xe - xb;
      sy = ye - yb;
      und.push_back(std::sqrt(sx * sx + sy * sy));
    }
  };
  std::printf("*** PROCEDURE CHECK DISTORTION ***\n");
  std::ofstream file("len_variation.txt");
  std::vector<double> L0, L0u, L, Lu;
  lengths(s.iref, L0, L0u);
  for (int idic = s.ibeg; idic <= s.iend; idic += s.iinc) {
    lengths(idic, L, Lu);
    if (L.size() != L0.size()) die("dic files with different grain counts");
    double m = 0.0, mu = 0.0;
    for (size_t k = 0; k < L0.size(); ++k) {
      m += (L[k] - L0[k]) / L0[k];
      mu += (Lu[k] - L0u[k]) / L0u[k];
    }
    m /= (double)L0.size();
    mu /= (double)L0.size();
    file << idic << ' ' << m << ' ' << mu << std::endl;
  }
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  bool check = false;
  const char* path = "commands.txt";
  for (int i = 1; i < argc; ++i) {
    if (!std::strcmp(argv[i], "-h") || !std::strcmp(argv[i], "--help")) {
      std::printf("usage: %s [--check] [command_file]\n", argv[0]);
      return 0;
    } else if (!std::strcmp(argv[i], "--check")) {
      check = true;
    } else {
      path = argv[i];
    }
  }
  Settings s = read_commands(path);
  for (const std::string& w : s.warnings) std::fprintf(stderr, "warning: %s\n", w.c_str());
  if (check) {
    print_json(s);
    return 0;
  }
  if (s.procedure == "check_distortion") {
    if (s.iinc <= 0 && s.ibeg <= s.iend) die("iinc must be > 0 (the reference loops forever otherwise)");
    return check_distortion(s);
  }
  const bool corr = s.procedure == "correction_distortion";
  if (!corr && s.procedure != "particle_tracking") die("procedure " + s.procedure + " is not part of this build");
  if (s.raw_images)
    die("RAW camera files need libraw, which this build does not have: convert the frames to TIFF or PGM, or "
        "pass libraw's unpacked mosaic to ptk_load_frame_raw");
  if (s.grains.empty()) die("no grains (grains_to_follow / start_file / restart_file)");
  if (corr) {
    if (s.corr_images.size() < 2) die("image_numbers_corrDisto needs the reference image and at least one more");
    if (s.imposed_x.size() != s.corr_images.size()) {
      s.imposed_x.assign(s.corr_images.size(), 0.0);
      s.imposed_y.assign(s.corr_images.size(), 0.0);
    }
    s.iref = s.corr_images[0];
  } else if (s.iinc <= 0 && s.ibeg <= s.iend) {
    die("iinc must be > 0 (the reference loops forever otherwise)");
  }

  std::printf(corr ? "\n*** PROCEDURE CORRECTION OF DISTORTION (B200) ***\n\n"
                   : "*** PROCEDURE PARTICLE IMAGE TRACKING (B200) ***\n");
  BufferPool pool;  // outlives every frame (declared before them)
  Frame ref = read_frame(&pool, s.image_name, s.iref, 0);
  if (ref.rc) die(ref.error);
  s.cfg.dimx = ref.dimx;
  s.cfg.dimy = ref.dimy;
  ptk_ctx* ctx = nullptr;
  auto ck = [&](int rc, const char* what) {
    if (rc) die(std::string(what) + ": " + ptk_last_error(ctx));
  };
  ck(ptk_create(&ctx, &s.cfg), "ptk_create");
  if (!s.tune_cache.empty()) ck(ptk_set_tune_cache(ctx, s.tune_cache.c_str()), "ptk_set_tune_cache");
  const int n = (int)s.grains.size();
  ck(ptk_set_grains(ctx, s.grains.data(), n), "ptk_set_grains");
  for (const PatternOp& op : s.patterns) {
    if (op.kind < 0) {
      std::vector<int32_t> xy;
      std::vector<int64_t> starts;
      read_pattern_file(op.file, n, &xy, &starts);
      ck(ptk_set_patterns(ctx, xy.data(), starts.data(), n), "ptk_set_patterns");
    } else {
      ck(ptk_make_patterns(ctx, op.kind, op.a, op.b, op.target), "ptk_make_patterns");
    }
  }
  bool disto = false;  // a non-identity undistor
  for (int k : {2, 3, 4, 5, 6, 7, 10, 11, 12, 13}) disto = disto || s.disto[k] != 0.0;
  if (corr) disto = false;  // the fit works on the frames as recorded
  if (s.undistort && disto) {
    double X[14];
    std::memcpy(X, s.disto, sizeof(X));
    default_centres(X, ref.dimx, ref.dimy);
    ck(ptk_set_distortion(ctx, X), "ptk_set_distortion");
  }
  auto load = [&](int slot, const Frame& f) {
    if (f.dimx != s.cfg.dimx || f.dimy != s.cfg.dimy) die(f.name + ": frame size differs from the reference frame");
    ck(ptk_load_frame(ctx, slot, f.pix.get(), f.dimx, f.dimy, 2, (size_t)f.dimx * 2), "ptk_load_frame");
    if (s.undistort && disto) ck(ptk_remap_frame(ctx, slot), "ptk_remap_frame");
  };
  load(0, ref);
  load(1, ref);  // as read_image(..., first_time) copies the first frame to both slots
  ck(ptk_set_iref(ctx, s.iref), "ptk_set_iref");
  int iref = s.iref;
  std::string ref_name = ref.name, ref_time = ref.datetime;

  if (corr) {
    // ---- correction_distortion: tracking from the reference image into
    // each other image (src/distortion_correction.cpp:157-220)
    std::vector<int32_t> refx((size_t)n), refy((size_t)n);
    for (int g = 0; g < n; ++g) {
      refx[g] = s.grains[g].refcoord_xpix;
      refy[g] = s.grains[g].refcoord_ypix;
    }
    int64_t np = 0;
    ptk_disto_pairs(refx.data(), refy.data(), n, s.equiproj_min, s.equiproj_max, nullptr, 0, &np);
    std::vector<int32_t> pairs((size_t)(2 * np + 2));
    if (ptk_disto_pairs(refx.data(), refy.data(), n, s.equiproj_min, s.equiproj_max, pairs.data(), np, &np))
      die("ptk_disto_pairs");
    std::printf("Number of points for equiprojectivity computations: %lld\n", (long long)np);
    std::printf("Tracking displacements... \n");
    const int nimg1 = (int)s.corr_images.size() - 1;
    std::vector<double> dx((size_t)nimg1 * n), dy((size_t)nimg1 * n), ncc((size_t)nimg1 * n);
    std::vector<ptk_grain> cur_g((size_t)n);
    for (int im = 1; im <= nimg1; ++im) {
      const int num = s.corr_images[im];
      Frame cur = read_frame(&pool, s.image_name, num, (size_t)ref.dimx * ref.dimy);
      if (cur.rc) die(cur.error);
      load(1, cur);
      // the estimated displacement starts every grain's search (:173-178)
      ck(ptk_get_grains(ctx, cur_g.data(), n), "ptk_get_grains");
      for (ptk_grain& g : cur_g) {
        g.dx = s.imposed_x[im];
        g.dy = s.imposed_y[im];
      }
      ck(ptk_set_grains(ctx, cur_g.data(), n), "ptk_set_grains");
      std::printf("> Follow %d grains... (from image number %d to number %d)\n", n, iref, num);
      const double t0 = now();
      ck(ptk_search(ctx, 0), "ptk_search");  // no rescue is attempted
      ck(ptk_subpixel(ctx, s.cfg.subpix_method), "ptk_subpixel");
      ck(ptk_get_grains(ctx, cur_g.data(), n), "ptk_get_grains");
      int failed = 0;
      for (int g = 0; g < n; ++g) {
        dx[(size_t)(im - 1) * n + g] = cur_g[g].dx;
        dy[(size_t)(im - 1) * n + g] = cur_g[g].dy;
        ncc[(size_t)(im - 1) * n + g] = cur_g[g].NCC_subpix;
        if (cur_g[g].NCC_subpix < s.cfg.NCC_min) ++failed;
      }
      std::printf("< [DONE in %f seconds]\nFailure rate = %g%%\n", now() - t0, 100.0 * (double)failed / (double)n);
      char fname[64];
      std::snprintf(fname, sizeof(fname), "dic_out_%d.txt", num);
      if (ptk_save_grains_file(fname, cur_g.data(), n, ref_name.c_str(), ref_time.c_str(), cur.name.c_str(),
                               cur.datetime.c_str()))
        die(std::string("cannot write ") + fname);
    }
    std::printf("Tracking of points done\n");
    ptk_destroy(ctx);

    // ---- minimisation (:222-478)
    double X[14];
    std::memcpy(X, s.disto, sizeof(X));
    std::printf("Numbers of position pairs used to undistor: %lld\nNumbers of image pairs: %d\n", (long long)np,
                nimg1);
    ptk_disto* dfit = nullptr;
    if (ptk_disto_create(&dfit, s.cfg.dimx, s.cfg.dimy, refx.data(), refy.data(), n, nimg1, dx.data(), dy.data(),
                         ncc.data(), s.cfg.NCC_min, pairs.data(), np))
      die("ptk_disto_create failed");
    const int iters = s.optim_algo == PTK_DISTO_POWELL_ITER ? s.powell_num_iter : 0;
    std::vector<double> hist((size_t)(iters > 0 ? iters : 1) * 15);
    double ini = 0.0, end = 0.0;
    const char* algo_name = s.optim_algo == PTK_DISTO_POWELL        ? "POWELL"
                            : s.optim_algo == PTK_DISTO_POWELL_ITER ? "POWELL_ITER"
                                                                    : "LEVMAR";
    std::printf("START minimizing equiprojectivity criterion (with %s)\n", algo_name);
    if (ptk_disto_fit(dfit, X, s.disto_perturb, s.optim_algo, iters, &ini, &end, hist.data()))
      die(std::string("ptk_disto_fit: ") + ptk_disto_last_error(dfit));
    std::printf("END minimizing equiprojectivity criterion (with %s)\n\n", algo_name);
    if (s.optim_algo == PTK_DISTO_LEVMAR) {  // src/distortion_correction.cpp:474
      int info = 0, nfev = 0;
      const char* text = "";
      ptk_disto_levmar_info(dfit, &info, &nfev, &text);
      std::printf("exit state: %s\n", text);
    }
    ptk_disto_destroy(dfit);
    if (s.optim_algo == PTK_DISTO_POWELL_ITER) {
      std::ofstream cf("convergence.txt");
      cf << std::scientific << std::setprecision(15);
      for (int it = 0; it < iters; ++it) {
        cf << it + 1;
        for (int k = 0; k < 15; ++k) cf << ' ' << hist[(size_t)it * 15 + k];
        cf << ' ' << std::endl;
      }
    }
    write_disto_outputs(X, ini, end, s.cfg.dimx, s.cfg.dimy);
    return 0;
  }

  // the next two frames are read and decoded on host threads while the GPU
  // tracks the current one (one frame's file read overlaps the other's decode)
  const size_t frame_elems = (size_t)ref.dimx * ref.dimy;
  std::deque<std::future<Frame>> ahead;
  int queued = s.ibeg;
  auto refill = [&]() {
    while (ahead.size() < 2 && queued <= s.iend) {
      ahead.push_back(std::async(std::launch::async, read_frame, &pool, s.image_name, queued, frame_elems));
      queued += s.iinc;
    }
  };
  refill();
  std::vector<ptk_grain> out((size_t)n);
  // The next frame is handed to the library right after the current one is
  // queued, before its records are read back, so that its upload overlaps the
  // tracking; it stays alive (its pinned buffer unchanged) until it is tracked.
  Frame next;
  bool have_next = false;
  auto take = [&]() {
    Frame f = ahead.front().get();
    ahead.pop_front();
    if (f.rc) die(f.error);
    refill();
    return f;
  };
  for (int num = s.ibeg; num <= s.iend; num += s.iinc) {
    const double t0 = now();
    Frame cur;
    if (have_next) {
      cur = std::move(next);
      have_next = false;
    } else {
      cur = take();
      load(1, cur);
    }
    std::printf("\n____ Correlations from image %d towards image %d (%d/%d)\n", iref, num, num - s.ibeg + 1,
                s.iend - s.ibeg + 1);
    ck(ptk_track_frame(ctx, num), "ptk_track_frame");
    if (num + s.iinc <= s.iend) {
      next = take();
      load(1, next);  // into the buffer the queued frame reads last (the old reference after a change)
      have_next = true;
    }
    ck(ptk_get_grains(ctx, out.data(), n), "ptk_get_grains");  // waits for the frame
    int nres = 0, nsup = 0;
    ck(ptk_get_rescue_counts(ctx, &nres, &nsup), "ptk_get_rescue_counts");
    char fname[64];
    std::snprintf(fname, sizeof(fname), "dic_out_%d.txt", num);
    if (ptk_save_grains_file(fname, out.data(), n, ref_name.c_str(), ref_time.c_str(), cur.name.c_str(),
                             cur.datetime.c_str()))
      die(std::string("cannot write ") + fname);
    std::printf("%d grains, %d rescued, %d super-rescued; %s written [%.3f s]\n", n, nres, nsup, fname, now() - t0);
    if (num - iref >= s.cfg.iraz) {  // the context changed its reference frame (src/p-tracker.cpp:587-611)
      iref = num;
      ref_name = cur.name;
      ref_time = cur.datetime;
    }
  }
  ptk_destroy(ctx);
  return 0;
}
