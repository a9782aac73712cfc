// ORACLE / TEST INFRASTRUCTURE ONLY.
// Minimal stand-in for libtiff's <tiffio.h> so the reference's sources compile
// (src/p-tracker.hpp:47).  Image decode is bypassed by the oracle harness, which
// writes pixel values straight into ptracker::image; every call here fails.
#pragma once
#include <cstddef>
#include <cstdint>
typedef struct tiff TIFF;
#define TIFFTAG_IMAGEWIDTH 256
#define TIFFTAG_IMAGELENGTH 257
#define TIFFTAG_DATETIME 306
#define TIFFGetR(abgr) ((abgr) & 0xff)
#define TIFFGetG(abgr) (((abgr) >> 8) & 0xff)
#define TIFFGetB(abgr) (((abgr) >> 16) & 0xff)
inline TIFF* TIFFOpen(const char*, const char*) { return nullptr; }
inline int TIFFGetField(TIFF*, uint32_t, ...) { return 0; }
inline void* _TIFFmalloc(size_t) { return nullptr; }
inline void _TIFFfree(void*) {}
inline int TIFFReadRGBAImage(TIFF*, uint32_t, uint32_t, uint32_t*, int) { return 0; }
inline void TIFFClose(TIFF*) {}
