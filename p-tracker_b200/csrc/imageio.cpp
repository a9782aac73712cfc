// Image files of the C ABI (include/ptk.h): the grey levels the tracking path
// works on, read from disk on the host.
//
// The reference reads frames with libtiff's RGBA reader and converts every
// pixel to one uint16 grey level (src/p-tracker.cpp:86-187):
//     r, g, b = 8-bit channel * (1 / 255)          (double)
//     grey    = (uint16)(65535 * (0.299 r + 0.587 g + 0.114 b))
// with the rows restored to top-down order.  libtiff is not part of this
// build, so strip TIFFs are decoded here - uncompressed, LZW (compression 5,
// as the TIFF 6.0 specification describes it: MSB-first codes of 9 to 12
// bits, Clear 256, EndOfInformation 257, the width growing when the next code
// to assign reaches 511 / 1023 / 2047), PackBits (32773) and Deflate (8 and
// 32946, through zlib), with horizontal-differencing prediction (Predictor 2)
// undone per row - and their samples go through the same 8-bit channels the
// RGBA reader produces: 8-bit grey v -> (v, v, v) (MinIsWhite: 255 - v),
// 16-bit grey -> its high byte, 16-bit colour channels -> (v + 128) / 257,
// 8-bit RGB / RGBA as stored.  Binary PGM (P5) frames are an addition of this
// build and are returned as stored.
#include <cctype>
#include <cstdint>
#include <cstdio>
#include <algorithm>
#include <cstring>
#include <fstream>
#include <string>
#include <thread>
#include <vector>

#include <zlib.h>

#include "../../include/ptk.h"

namespace {

struct Reader {
  std::vector<unsigned char> d;
  bool le = true;
  bool ok(size_t off, size_t n) const { return off <= d.size() && n <= d.size() - off; }
  uint16_t u16(size_t o) const {
    return le ? (uint16_t)(d[o] | (d[o + 1] << 8)) : (uint16_t)((d[o] << 8) | d[o + 1]);
  }
  uint32_t u32(size_t o) const {
    return le ? (uint32_t)d[o] | ((uint32_t)d[o + 1] << 8) | ((uint32_t)d[o + 2] << 16) | ((uint32_t)d[o + 3] << 24)
              : ((uint32_t)d[o] << 24) | ((uint32_t)d[o + 1] << 16) | ((uint32_t)d[o + 2] << 8) | (uint32_t)d[o + 3];
  }
};

struct Entry {
  uint16_t type = 0;
  uint32_t count = 0;
  size_t at = 0;  // file offset of the first value
};

size_t type_size(uint16_t t) {
  switch (t) {
    case 1: case 2: case 6: case 7: return 1;
    case 3: case 8: return 2;
    case 4: case 9: case 11: return 4;
    case 5: case 10: case 12: return 8;
    default: return 0;
  }
}

// k-th value of an integer entry (BYTE / SHORT / LONG)
bool value(const Reader& r, const Entry& e, uint32_t k, uint32_t* v) {
  const size_t s = type_size(e.type);
  if (k >= e.count || (e.type != 1 && e.type != 3 && e.type != 4)) return false;
  const size_t o = e.at + (size_t)k * s;
  if (!r.ok(o, s)) return false;
  *v = e.type == 1 ? r.d[o] : (e.type == 3 ? r.u16(o) : r.u32(o));
  return true;
}

// TIFF LZW: decodes src into dst (at most cap bytes); *out = bytes written.
bool lzw_decode(const unsigned char* src, size_t n, unsigned char* dst, size_t cap, size_t* out) {
  uint16_t prefix[4096], length[4096];  // the code table, on this thread's stack (24 KB)
  unsigned char suffix[4096], first[4096];
  for (int c = 0; c < 256; ++c) {
    prefix[c] = 0xffff;
    suffix[c] = first[c] = (unsigned char)c;
    length[c] = 1;
  }
  size_t o = 0, pos = 0;  // output bytes, input bytes consumed into acc
  uint64_t acc = 0;       // the next nbits input bits, most significant first
  int nbits = 0;
  int width = 9, next = 258, prev = -1;
  auto read = [&](int* code) -> bool {
    while (nbits < width && pos < n) {
      acc = (acc << 8) | src[pos++];
      nbits += 8;
    }
    if (nbits < width) return false;
    nbits -= width;
    *code = (int)((acc >> nbits) & ((1u << width) - 1u));
    return true;
  };
  auto emit = [&](int code) -> bool {  // the string of `code`, written back to front
    const size_t len = length[code];
    if (o + len > cap) return false;
    for (size_t k = len; k-- > 0;) {
      dst[o + k] = suffix[code];
      code = prefix[code];
    }
    o += len;
    return true;
  };
  int code;
  while (read(&code)) {
    if (code == 257) break;
    if (code == 256) {
      width = 9;
      next = 258;
      prev = -1;
      continue;
    }
    if (prev < 0) {
      if (code > 255 || !emit(code)) return false;
      prev = code;
      continue;
    }
    if (next >= 4096) return false;
    if (code < next) {
      if (code >= 256 && code < 258) return false;
      if (!emit(code)) return false;
      prefix[next] = (uint16_t)prev;
      suffix[next] = first[code];
    } else if (code == next) {
      prefix[next] = (uint16_t)prev;
      suffix[next] = first[prev];
      first[next] = first[prev];
      length[next] = (uint16_t)(length[prev] + 1);
      if (!emit(next)) return false;
    } else {
      return false;
    }
    first[next] = first[prev];
    length[next] = (uint16_t)(length[prev] + 1);
    ++next;
    if (next == 511) width = 10;
    else if (next == 1023) width = 11;
    else if (next == 2047) width = 12;
    prev = code;
  }
  *out = o;
  return true;
}

// PackBits: a header byte h, then h + 1 literal bytes (h >= 0) or one byte
// repeated 1 - h times (-127 <= h <= -1); -128 is skipped.
bool packbits_decode(const unsigned char* src, size_t n, unsigned char* dst, size_t cap, size_t* out) {
  size_t i = 0, o = 0;
  while (i < n && o < cap) {
    const int h = (signed char)src[i++];
    if (h >= 0) {
      if (i + (size_t)h + 1 > n || o + (size_t)h + 1 > cap) return false;
      std::memcpy(dst + o, src + i, (size_t)h + 1);
      i += (size_t)h + 1;
      o += (size_t)h + 1;
    } else if (h != -128) {
      if (i >= n || o + (size_t)(1 - h) > cap) return false;
      std::memset(dst + o, src[i++], (size_t)(1 - h));
      o += (size_t)(1 - h);
    }
  }
  *out = o;
  return true;
}

// items [0, n) of a per-item function (rows, strips), split over a few host
// threads when there is enough work (`work` bytes or pixels); the items are
// independent
template <class F>
void for_items(size_t n, size_t work, F&& f) {
  unsigned nt = std::thread::hardware_concurrency();
  nt = nt > 8 ? 8 : (nt < 1 ? 1 : nt);
  if (work < ((size_t)1 << 20) || nt == 1 || n < 2) {
    for (size_t i = 0; i < n; ++i) f(i);
    return;
  }
  if ((size_t)nt > n) nt = (unsigned)n;
  std::vector<std::thread> pool;
  for (unsigned t = 0; t < nt; ++t)
    pool.emplace_back([&, t]() {
      for (size_t i = t; i < n; i += nt) f(i);
    });
  for (std::thread& th : pool) th.join();
}

template <class F>
void for_rows(uint32_t h, size_t pixels, F&& f) {
  for_items(h, pixels, [&](size_t y) { f((uint32_t)y); });
}

uint16_t grey_of(double R, double G, double B) {
  const double fact = 1.0 / 255.0;
  const double rr = R * fact, gg = G * fact, bb = B * fact;
  return (uint16_t)(65535.0 * (0.299 * rr + 0.587 * gg + 0.114 * bb));
}

int read_tiff(Reader& r, uint16_t* out, size_t capacity, int* dimx, int* dimy, std::string* when,
              std::string* err) {
  r.le = r.d[0] == 'I';
  if (r.u16(2) != 42) return (*err = "not a TIFF file", PTK_ERR_IO);
  const size_t ifd = r.u32(4);
  if (!r.ok(ifd, 2)) return (*err = "truncated TIFF header", PTK_ERR_IO);
  const int n = r.u16(ifd);
  if (!r.ok(ifd + 2, (size_t)n * 12)) return (*err = "truncated TIFF directory", PTK_ERR_IO);
  bool have[400] = {};  // baseline tags only (all below 400)
  Entry ent[400];
  for (int i = 0; i < n; ++i) {
    const size_t o = ifd + 2 + (size_t)i * 12;
    const uint16_t t = r.u16(o);
    if (t >= 400) continue;
    Entry e;
    e.type = r.u16(o + 2);
    e.count = r.u32(o + 4);
    const size_t bytes = type_size(e.type) * (size_t)e.count;
    e.at = bytes <= 4 ? o + 8 : r.u32(o + 8);
    ent[t] = e;
    have[t] = true;
  }
  auto get = [&](int t, uint32_t dflt) -> uint32_t {
    uint32_t v = dflt;
    if (have[t] && !value(r, ent[t], 0, &v)) v = dflt;
    return v;
  };
  const uint32_t w = get(256, 0), h = get(257, 0);
  const uint32_t spp = get(277, 1), comp = get(259, 1), photo = get(262, 1), planar = get(284, 1);
  const uint32_t orient = get(274, 1), fmt = get(339, 1), pred = get(317, 1);
  uint32_t bps = 8;
  if (have[258] && !value(r, ent[258], 0, &bps)) bps = 8;
  if (w == 0 || h == 0 || w > 65535 || h > 65535) return (*err = "bad TIFF image size", PTK_ERR_IO);
  if (comp != 1 && comp != 5 && comp != 8 && comp != 32946 && comp != 32773)
    return (*err = "TIFF compression not supported (none, LZW, Deflate or PackBits)", PTK_ERR_IO);
  if (pred != 1 && pred != 2) return (*err = "TIFF predictor not supported (none or horizontal)", PTK_ERR_IO);
  if (planar != 1 || orient != 1 || fmt != 1)
    return (*err = "TIFF layout not supported (chunky, top-left, unsigned samples only)", PTK_ERR_IO);
  if (bps != 8 && bps != 16) return (*err = "TIFF sample depth must be 8 or 16 bits", PTK_ERR_IO);
  const bool grey = photo == 0 || photo == 1;
  if (!(grey && spp >= 1) && !(photo == 2 && spp >= 3))
    return (*err = "TIFF photometric interpretation not supported (grey or RGB)", PTK_ERR_IO);
  if (!have[273] || !have[279]) return (*err = "TIFF without strips (tiled TIFF is not supported)", PTK_ERR_IO);
  *dimx = (int)w;
  *dimy = (int)h;
  if (have[306]) {
    const Entry& e = ent[306];
    if (r.ok(e.at, e.count)) {
      std::string s(reinterpret_cast<const char*>(&r.d[e.at]), e.count);
      const size_t z = s.find('\0');
      *when = z == std::string::npos ? s : s.substr(0, z);
    }
  }
  if (!out) return PTK_OK;
  if (capacity < (size_t)w * h) return (*err = "output buffer too small", PTK_ERR_ARG);
  // the strips, decoded and concatenated, hold the rows top-down
  const size_t bpp = (size_t)spp * (bps / 8), row_bytes = bpp * w;
  uint32_t rps = get(278, h);
  if (rps == 0 || rps > h) rps = h;
  std::vector<unsigned char> pix(row_bytes * h);
  const size_t strip_bytes = (size_t)rps * row_bytes;
  const size_t nstrips = (pix.size() + strip_bytes - 1) / strip_bytes;  // strips the image needs
  if (ent[273].count < nstrips || ent[279].count < nstrips)
    return (*err = "TIFF strips shorter than the image", PTK_ERR_IO);
  // strip k fills bytes [k strip_bytes, ...) of the image: strips decode independently
  std::vector<unsigned char> bad(nstrips, 0);  // 1 truncated, 2 corrupt or short
  auto strip = [&](size_t k) {
    uint32_t off = 0, len = 0;
    if (!value(r, ent[273], (uint32_t)k, &off) || !value(r, ent[279], (uint32_t)k, &len) || !r.ok(off, len)) {
      bad[k] = 1;
      return;
    }
    const size_t at = k * strip_bytes, want = std::min(pix.size() - at, strip_bytes);
    const unsigned char* src = r.d.data() + off;
    unsigned char* dst = pix.data() + at;
    size_t got = 0;
    bool good = true;
    if (comp == 1) {
      got = std::min((size_t)len, want);
      std::memcpy(dst, src, got);
    } else if (comp == 5) {
      good = lzw_decode(src, len, dst, want, &got);
    } else if (comp == 32773) {
      good = packbits_decode(src, len, dst, want, &got);
    } else {
      uLongf dl = (uLongf)want;
      uLong sl = (uLong)len;
      const int zr = uncompress2(dst, &dl, src, &sl);
      // Z_BUF_ERROR with the output full: the strip holds more than the image
      // needs; short output (truncated or corrupt input) fails the check below
      good = zr == Z_OK || zr == Z_BUF_ERROR;
      got = (size_t)dl;
    }
    if (!good || got < want) bad[k] = 2;
  };
  for_items(nstrips, comp == 1 ? pix.size() : pix.size() * 4, strip);
  for (size_t k = 0; k < nstrips; ++k) {
    if (bad[k] == 1) return (*err = "truncated TIFF strip", PTK_ERR_IO);
    if (bad[k] == 2) return (*err = "corrupt or short TIFF strip", PTK_ERR_IO);
  }
  auto sample = [&](size_t o) -> uint32_t {
    return bps == 8 ? pix[o] : (r.le ? (uint32_t)(pix[o] | (pix[o + 1] << 8)) : (uint32_t)((pix[o] << 8) | pix[o + 1]));
  };
  if (pred == 2) {  // horizontal differencing: each sample adds the same channel's sample to its left
    for_rows(h, (size_t)w * h, [&](uint32_t y) {
      unsigned char* row = pix.data() + (size_t)y * row_bytes;
      for (uint32_t x = 1; x < w; ++x)
        for (uint32_t c = 0; c < spp; ++c) {
          const size_t o = ((size_t)x * spp + c) * (bps / 8), q = o - bpp;
          if (bps == 8) {
            row[o] = (unsigned char)(row[o] + row[q]);
          } else {
            const size_t ro = (size_t)y * row_bytes;
            const uint32_t v = (sample(ro + o) + sample(ro + q)) & 0xffffu;
            row[o] = (unsigned char)(r.le ? v & 0xff : v >> 8);
            row[o + 1] = (unsigned char)(r.le ? v >> 8 : v & 0xff);
          }
        }
    });
  }
  // every grey level comes from 8-bit channels: a grey image maps through a
  // 256-entry table of grey_of(v, v, v); a colour one adds the channels'
  // weighted terms, each precomputed per 8-bit value, in grey_of's order
  uint16_t lut[256];
  double tr[256], tg[256], tb[256];
  for (int v = 0; v < 256; ++v) {
    const double f = (double)v * (1.0 / 255.0);
    lut[v] = grey_of(v, v, v);
    tr[v] = 0.299 * f;
    tg[v] = 0.587 * f;
    tb[v] = 0.114 * f;
  }
  for_rows(h, (size_t)w * h, [&](uint32_t y) {
    for (uint32_t x = 0; x < w; ++x) {
      const size_t o = (size_t)y * row_bytes + (size_t)x * bpp;
      if (grey) {
        uint32_t v = sample(o);
        if (bps == 16) v >>= 8;  // the RGBA reader keeps the high byte of 16-bit grey
        if (photo == 0) v = 255 - v;
        out[(size_t)y * w + x] = lut[v];
      } else {
        uint32_t c[3];
        for (int k = 0; k < 3; ++k) {
          c[k] = sample(o + k * (bps / 8));
          if (bps == 16) c[k] = (c[k] + 128) / 257;
        }
        out[(size_t)y * w + x] = (uint16_t)(65535.0 * (tr[c[0]] + tg[c[1]] + tb[c[2]]));
      }
    }
  });
  return PTK_OK;
}

int read_pgm(Reader& r, uint16_t* out, size_t capacity, int* dimx, int* dimy, std::string* err) {
  size_t p = 2;
  auto next = [&](long* v) -> bool {
    while (p < r.d.size()) {
      if (r.d[p] == '#') {
        while (p < r.d.size() && r.d[p] != '\n') ++p;
      } else if (std::isspace(r.d[p])) {
        ++p;
      } else {
        break;
      }
    }
    long x = 0;
    bool any = false;
    while (p < r.d.size() && r.d[p] >= '0' && r.d[p] <= '9') {
      x = x * 10 + (r.d[p++] - '0');
      any = true;
      if (x > 1000000) return false;
    }
    *v = x;
    return any;
  };
  long w, h, maxv;
  if (!next(&w) || !next(&h) || !next(&maxv) || w <= 0 || h <= 0 || w > 65535 || h > 65535 || maxv <= 0 ||
      maxv > 65535)
    return (*err = "bad PGM header", PTK_ERR_IO);
  ++p;  // the single whitespace after maxval
  *dimx = (int)w;
  *dimy = (int)h;
  if (!out) return PTK_OK;
  if (capacity < (size_t)w * h) return (*err = "output buffer too small", PTK_ERR_ARG);
  const size_t bpp = maxv < 256 ? 1 : 2;
  if (!r.ok(p, (size_t)w * h * bpp)) return (*err = "truncated PGM data", PTK_ERR_IO);
  const unsigned char* src = r.d.data() + p;
  for_rows((uint32_t)h, (size_t)w * h, [&](uint32_t y) {
    const size_t i0 = (size_t)y * w, i1 = i0 + w;
    for (size_t i = i0; i < i1; ++i) out[i] = bpp == 1 ? src[i] : (uint16_t)((src[2 * i] << 8) | src[2 * i + 1]);
  });
  return PTK_OK;
}

thread_local std::string g_image_error;

}  // namespace

extern "C" {

int ptk_read_image_file(const char* path, uint16_t* out, size_t capacity, int* dimx, int* dimy, char* datetime,
                        int datetime_len) {
  if (!path || !dimx || !dimy) return PTK_ERR_ARG;
  Reader r;
  {
    std::ifstream f(path, std::ios::binary | std::ios::ate);  // one sized read: frames are tens of MB
    if (!f) {
      g_image_error = std::string("cannot open ") + path;
      return PTK_ERR_IO;
    }
    const std::streamoff size = f.tellg();
    if (size < 0) {
      g_image_error = std::string("cannot read ") + path;
      return PTK_ERR_IO;
    }
    r.d.resize((size_t)size);
    f.seekg(0);
    if (size > 0 && !f.read(reinterpret_cast<char*>(r.d.data()), size)) {
      g_image_error = std::string("cannot read ") + path;
      return PTK_ERR_IO;
    }
  }
  std::string when = "dateTime unknown", err;
  int rc;
  if (r.d.size() >= 8 && ((r.d[0] == 'I' && r.d[1] == 'I') || (r.d[0] == 'M' && r.d[1] == 'M'))) {
    rc = read_tiff(r, out, capacity, dimx, dimy, &when, &err);
  } else if (r.d.size() >= 2 && r.d[0] == 'P' && r.d[1] == '5') {
    rc = read_pgm(r, out, capacity, dimx, dimy, &err);
  } else {
    rc = PTK_ERR_IO;
    err = "unknown image format (TIFF or binary PGM)";
  }
  if (rc) {
    g_image_error = std::string(path) + ": " + err;
    return rc;
  }
  if (datetime && datetime_len > 0) {
    std::strncpy(datetime, when.c_str(), (size_t)datetime_len - 1);
    datetime[datetime_len - 1] = '\0';
  }
  return PTK_OK;
}

const char* ptk_image_error(void) { return g_image_error.c_str(); }

}  // extern "C"
