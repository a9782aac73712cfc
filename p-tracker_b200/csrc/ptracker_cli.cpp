// ptracker_b200: the particle_tracking procedure of `ptracker <command_file>`
// (src/p-tracker.cpp:422-612, run.cpp) driven through the C ABI of this
// library, for one GPU.
//
// Command file: the reference's token stream (read_data,
// src/p-tracker.cpp:1487-1784): whitespace-separated tokens, '#' or '!' starts
// a comment to the end of the line, unknown tokens are reported and skipped.
// Grain files, `pattern`, `targetRadiusPattern` and `mask_rect` act on the
// grains loaded so far, in file order, as they do in the reference.  Tokens of
// procedures other than particle tracking (distortion fitting, RAW decoding,
// neighbour lists, thread counts) are accepted and have no effect.  Added
// tokens select the forms of this library:
//     search_method  exact | bf16          integer search (default exact)
//     subpix_method  powell | adjoint_lm   subpixel refinement (default powell)
//     topk K, lm_max_iter N, lm_tol T      their parameters
//     undistort_images 0 | 1               resample every frame with the
//                                          *_corrDistor / *_corrParallax
//                                          parameters before tracking
//
// Frames: image_name is a printf pattern of the frame number (read_image,
// src/p-tracker.cpp:75-83); frames are uncompressed TIFF (converted as the
// reference's libtiff RGBA path) or binary PGM.  The next frame is decoded on
// a host thread while the GPU tracks the current one.  After every frame the
// grains go to dic_out_<num>.txt in the working directory, byte for byte as
// save_grains (src/p-tracker.cpp:1313-1367).
//
//   ptracker_b200 [command_file]     (default: commands.txt)
//   ptracker_b200 --check file       parse only; print the settings as JSON
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <future>
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
  std::string image_name = "%d.tif", dic_name, procedure = "particle_tracking";
  int iref = 0, ibeg = 0, iend = 0, iinc = 0;
  int raw_images = 0, undistort = 0;
  ptk_config cfg;
  double target_radius = -1.0;
  double disto[14] = {};
  std::vector<ptk_grain> grains;
  std::vector<PatternOp> patterns;  // acting on the grains loaded last
  std::vector<std::string> warnings;
  int unknown_tokens = 0;
};

struct Frame {
  std::vector<uint16_t> pix;
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

Frame read_frame(const std::string& pattern, int num) {
  Frame f;
  f.name = frame_name(pattern, num);
  char when[256];
  f.rc = ptk_read_image_file(f.name.c_str(), nullptr, 0, &f.dimx, &f.dimy, nullptr, 0);
  if (f.rc == PTK_OK) {
    f.pix.resize((size_t)f.dimx * f.dimy);
    f.rc = ptk_read_image_file(f.name.c_str(), f.pix.data(), f.pix.size(), &f.dimx, &f.dimy, when, sizeof(when));
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
               tok == "wanted_num_threads" || tok == "verbose_level" || tok == "powell_num_iter" ||
               tok == "num_neighbour_max" || tok == "neighbour_dist_pix" || tok == "period_rebuild_neighbour_list" ||
               tok == "use_neighbour_list" || tok == "optim_algo") {
      skip(1);
    } else if (tok == "grains_to_follow" || tok == "start_file") {
      std::string f;
      in >> f;
      load_grains(s, f, false);
    } else if (tok == "restart_file") {
      std::string f;
      in >> f;
      load_grains(s, f, true);
    } else if (tok == "make_grid") {
      skip(7);
      s.warnings.push_back("make_grid (grain seeding) is not part of this build: ignored");
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
    } else if (tok == "image_numbers_corrDisto") {
      size_t nb;
      in >> nb;
      skip((int)nb);
    } else if (tok == "imposedDisplApprox_corrDisto") {
      s.warnings.push_back("imposedDisplApprox_corrDisto belongs to the distortion fit: ignored");
    } else if (tok == "equiProj_dist_range") {
      skip(2);
    } else if (tok.size() > 11 && (tok.find("_corrDistor") != std::string::npos ||
                                   tok.find("_corrParallax") != std::string::npos)) {
      static const char* names[14] = {"xc_corrDistor", "yc_corrDistor", "K1_corrDistor", "K2_corrDistor",
                                      "K3_corrDistor", "P1_corrDistor", "P2_corrDistor", "P3_corrDistor",
                                      "xc_corrParallax", "yc_corrParallax", "angle1_corrParallax",
                                      "A1_corrParallax", "angle2_corrParallax", "A2_corrParallax"};
      int k = -1;
      for (int i = 0; i < 14; ++i)
        if (tok == names[i]) k = i;
      double v;
      in >> v;
      if (k >= 0) s.disto[k] = v;  // the d*_ perturbations belong to the fit
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
  o << ", \"masked\": " << masked << ", \"rescue_level\": " << c.rescue_level << ", \"NCC_min\": " << c.NCC_min
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
  o << "], \"search_method\": " << c.search_method << ", \"subpix_method\": " << c.subpix_method
    << ", \"undistort_images\": " << s.undistort << ", \"disto\": [";
  for (int k = 0; k < 14; ++k) o << (k ? ", " : "") << s.disto[k];
  o << "], \"unknown_tokens\": " << s.unknown_tokens << ", \"warnings\": " << s.warnings.size() << "}";
  std::printf("%s\n", o.str().c_str());
}

double now() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
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
  if (s.procedure != "particle_tracking") die("procedure " + s.procedure + " is not part of this build");
  if (s.raw_images) die("RAW images (libraw) are not supported: convert the frames to TIFF or PGM");
  if (s.grains.empty()) die("no grains (grains_to_follow / start_file / restart_file)");
  if (s.iinc <= 0 && s.ibeg <= s.iend) die("iinc must be > 0 (the reference loops forever otherwise)");

  std::printf("*** PROCEDURE PARTICLE IMAGE TRACKING (B200) ***\n");
  Frame ref = read_frame(s.image_name, s.iref);
  if (ref.rc) die(ref.error);
  s.cfg.dimx = ref.dimx;
  s.cfg.dimy = ref.dimy;
  ptk_ctx* ctx = nullptr;
  auto ck = [&](int rc, const char* what) {
    if (rc) die(std::string(what) + ": " + ptk_last_error(ctx));
  };
  ck(ptk_create(&ctx, &s.cfg), "ptk_create");
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
  bool disto = false;
  for (double v : s.disto) disto = disto || v != 0.0;
  if (s.undistort && disto) ck(ptk_set_distortion(ctx, s.disto), "ptk_set_distortion");
  auto load = [&](int slot, const Frame& f) {
    if (f.dimx != s.cfg.dimx || f.dimy != s.cfg.dimy) die(f.name + ": frame size differs from the reference frame");
    ck(ptk_load_frame(ctx, slot, f.pix.data(), f.dimx, f.dimy, 2, (size_t)f.dimx * 2), "ptk_load_frame");
    if (s.undistort && disto) ck(ptk_remap_frame(ctx, slot), "ptk_remap_frame");
  };
  load(0, ref);
  load(1, ref);  // as read_image(..., first_time) copies the first frame to both slots
  ck(ptk_set_iref(ctx, s.iref), "ptk_set_iref");
  int iref = s.iref;
  std::string ref_name = ref.name, ref_time = ref.datetime;

  std::future<Frame> next;
  if (s.ibeg <= s.iend) next = std::async(std::launch::async, read_frame, s.image_name, s.ibeg);
  std::vector<ptk_grain> out((size_t)n);
  for (int num = s.ibeg; num <= s.iend; num += s.iinc) {
    const double t0 = now();
    Frame cur = next.get();
    if (cur.rc) die(cur.error);
    if (num + s.iinc <= s.iend) next = std::async(std::launch::async, read_frame, s.image_name, num + s.iinc);
    std::printf("\n____ Correlations from image %d towards image %d (%d/%d)\n", iref, num, num - s.ibeg + 1,
                s.iend - s.ibeg + 1);
    load(1, cur);
    ck(ptk_track_frame(ctx, num), "ptk_track_frame");
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
