// ORACLE / TEST INFRASTRUCTURE ONLY.
// Minimal stand-in for <libraw.h> so the reference's sources compile
// (src/p-tracker.hpp:46).  RAW decode is bypassed by the oracle harness;
// open_file always fails.
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
class LibRaw {
 public:
  libraw_stub_data imgdata{};
  int open_file(const char*) { return -1; }
  int unpack() { return -1; }
  int dcraw_process() { return -1; }
  void recycle() {}
};
