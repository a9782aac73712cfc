// ORACLE / TEST INFRASTRUCTURE ONLY.
// Minimal stand-in for <libraw.h> so the reference's sources compile
// (src/p-tracker.hpp:46).  Camera files are never decoded: open_file succeeds
// only after the oracle harness has registered an unpacked sensor mosaic with
// libraw_stub_source() (raw_image, raw_width, margins, visible size), which
// the next open_file copies into imgdata; that is what libraw's open_file +
// unpack leave behind, so read_raw_image's own demosaic code (modes -1, -2,
// -20) runs on it.  dcraw_process (libraw's demosaic, modes >= 0) fails.
#pragma once
#include <cstdint>
#include <ctime>
struct libraw_stub_other { float iso_speed, shutter, aperture, focal_len; unsigned shot_order; time_t timestamp; };
struct libraw_stub_idata { char make[64]; char model[64]; };
struct libraw_stub_sizes { int width, height, raw_width, top_margin, left_margin; };
struct libraw_stub_color { unsigned maximum; };
struct libraw_stub_params { int user_qual; };
struct libraw_stub_rawdata { uint16_t* raw_image; };
struct libraw_stub_data {
  libraw_stub_other other; libraw_stub_idata idata; libraw_stub_sizes sizes;
  libraw_stub_color color; libraw_stub_params params; libraw_stub_rawdata rawdata;
  uint16_t (*image)[4];
};
inline libraw_stub_data& libraw_stub_source() {
  static libraw_stub_data d{};
  return d;
}
class LibRaw {
 public:
  libraw_stub_data imgdata{};
  int open_file(const char*) {
    if (!libraw_stub_source().rawdata.raw_image) return -1;
    imgdata = libraw_stub_source();
    return 0;
  }
  int unpack() { return 0; }
  int dcraw_process() { return -1; }
  void recycle() {}
};
