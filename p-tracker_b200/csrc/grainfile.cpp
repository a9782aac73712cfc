// Grain-file I/O of the C ABI (include/ptk.h).
//
// The 13-column "dic_out" form is written exactly as ptracker::save_grains
// does (src/p-tracker.cpp:1313-1360): count line, then per grain
// std::scientific, precision 15, refcoord x/y left-aligned in width 6, the
// eleven reals right-aligned in width 23, single spaces, then a blank line and
// the four '#' trailer lines.  Reading follows read_grains
// (src/p-tracker.cpp:1213-1278): the 13-column form fills every field, the
// 4-column form (x y refrot radius) puts floor(x), floor(y) into refcoord and
// the fractional parts into dx/upix and dy/vpix.
#include <cmath>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <string>

#include "../../include/ptk.h"

extern "C" {

int ptk_read_grains_file(const char* path, int format13, ptk_grain* out, int capacity, int* n) {
  if (!path || !n) return PTK_ERR_ARG;
  std::ifstream f(path);
  if (!f) return PTK_ERR_IO;
  int num = 0;
  f >> num;
  if (!f || num < 0) return PTK_ERR_IO;
  *n = num;
  if (!out) return PTK_OK;
  if (capacity < num) return PTK_ERR_ARG;
  for (int i = 0; i < num; ++i) {
    ptk_grain& g = out[i];
    std::memset(&g, 0, sizeof(g));
    if (format13) {
      f >> g.refcoord_xpix >> g.refcoord_ypix >> g.refrot >> g.radius_pix >> g.dx >> g.dy >> g.drot >> g.upix >>
          g.vpix >> g.rot_inc >> g.NCC >> g.NCC_rescue >> g.NCC_subpix;
    } else {
      double x, y, radius;
      f >> x >> y >> g.refrot >> radius;
      g.radius_pix = radius;
      g.refcoord_xpix = (int)std::floor(x);
      g.dx = g.upix = x - std::floor(x);
      g.refcoord_ypix = (int)std::floor(y);
      g.dy = g.vpix = y - std::floor(y);
    }
    if (!f) return PTK_ERR_IO;
  }
  return PTK_OK;
}

int ptk_save_grains_file(const char* path, const ptk_grain* grains, int n, const char* from_image,
                         const char* from_datetime, const char* to_image, const char* to_datetime) {
  if (!path || (n > 0 && !grains) || n < 0) return PTK_ERR_ARG;
  std::ofstream f(path);
  if (!f) return PTK_ERR_IO;
  f << n << std::endl;
  for (int i = 0; i < n; ++i) {
    const ptk_grain& g = grains[i];
    f << std::scientific << std::setprecision(15)
      << std::setw(6) << std::left << g.refcoord_xpix << ' '
      << std::setw(6) << std::left << g.refcoord_ypix << ' '
      << std::setw(23) << std::right << g.refrot << ' '
      << std::setw(23) << std::right << g.radius_pix << ' '
      << std::setw(23) << std::right << g.dx << ' '
      << std::setw(23) << std::right << g.dy << ' '
      << std::setw(23) << std::right << g.drot << ' '
      << std::setw(23) << std::right << g.upix << ' '
      << std::setw(23) << std::right << g.vpix << ' '
      << std::setw(23) << std::right << g.rot_inc << ' '
      << std::setw(23) << std::right << g.NCC << ' '
      << std::setw(23) << std::right << g.NCC_rescue << ' '
      << std::setw(23) << std::right << g.NCC_subpix << '\n';
  }
  f << std::endl;
  f << "#_FROM_image: " << (from_image ? from_image : "") << '\n';
  f << "#___dateTime: " << (from_datetime ? from_datetime : "dateTime unknown") << '\n';
  f << "#___TO_image: " << (to_image ? to_image : "") << '\n';
  f << "#___dateTime: " << (to_datetime ? to_datetime : "dateTime unknown") << '\n';
  f << std::flush;
  return f ? PTK_OK : PTK_ERR_IO;
}

}  // extern "C"
