/* Compile-only stand-in for libtiff's <tiffio.h> (oracle/_ref build only;
 * libtiff is not installed here).  ST_Tomography.h defines cimg_use_tiff, so
 * CImg.h compiles its libtiff paths.  The checkers never read TIFF files (the
 * projection stack is handed over as a .cimg file, which CImg reads itself)
 * and discard what the reference writes: TIFFOpen succeeds for writing and
 * every write is accepted and dropped, so CImg::save_tiff
 * (ST_Tomography.cpp:464, 805) returns normally without touching the disk;
 * opening for reading fails, and CImg reports that as an I/O error. */
#ifndef STT_ORACLE_SHIM_TIFFIO_H
#define STT_ORACLE_SHIM_TIFFIO_H
#include <cstdarg>
#include <cstdint>
#include <cstdlib>

typedef uint8_t uint8;
typedef int8_t int8;
typedef uint16_t uint16;
typedef int16_t int16;
typedef uint32_t uint32;
typedef int32_t int32;
typedef long tsize_t;
typedef void *tdata_t;
typedef uint32 tstrip_t;
typedef uint32 ttile_t;
typedef void (*TIFFErrorHandler)(const char *, const char *, va_list);

struct stt_shim_tiff {
    const char *name;
    uint32 width, length, spp, bps, rows_per_strip;
};
typedef struct stt_shim_tiff TIFF;

#define TIFFTAG_IMAGEWIDTH 256
#define TIFFTAG_IMAGELENGTH 257
#define TIFFTAG_BITSPERSAMPLE 258
#define TIFFTAG_COMPRESSION 259
#define TIFFTAG_PHOTOMETRIC 262
#define TIFFTAG_FILLORDER 266
#define TIFFTAG_IMAGEDESCRIPTION 270
#define TIFFTAG_ORIENTATION 274
#define TIFFTAG_SAMPLESPERPIXEL 277
#define TIFFTAG_ROWSPERSTRIP 278
#define TIFFTAG_XRESOLUTION 282
#define TIFFTAG_YRESOLUTION 283
#define TIFFTAG_PLANARCONFIG 284
#define TIFFTAG_RESOLUTIONUNIT 296
#define TIFFTAG_SOFTWARE 305
#define TIFFTAG_TILEWIDTH 322
#define TIFFTAG_TILELENGTH 323
#define TIFFTAG_SAMPLEFORMAT 339
#define COMPRESSION_NONE 1
#define COMPRESSION_LZW 5
#define COMPRESSION_JPEG 7
#define PHOTOMETRIC_MINISBLACK 1
#define PHOTOMETRIC_RGB 2
#define FILLORDER_MSB2LSB 1
#define ORIENTATION_TOPLEFT 1
#define PLANARCONFIG_CONTIG 1
#define PLANARCONFIG_SEPARATE 2
#define RESUNIT_NONE 1
#define SAMPLEFORMAT_UINT 1
#define SAMPLEFORMAT_INT 2
#define SAMPLEFORMAT_IEEEFP 3
#define TIFFGetR(abgr) ((abgr) & 0xff)
#define TIFFGetG(abgr) (((abgr) >> 8) & 0xff)
#define TIFFGetB(abgr) (((abgr) >> 16) & 0xff)
#define TIFFGetA(abgr) (((abgr) >> 24) & 0xff)

static inline TIFF *TIFFOpen(const char *name, const char *mode) {
    static thread_local TIFF sink;
    if (!mode || mode[0] != 'w') return 0;
    sink = TIFF{name, 0, 0, 1, 8, 1};
    return &sink;
}
static inline void TIFFClose(TIFF *) {}
static inline const char *TIFFFileName(TIFF *t) { return t && t->name ? t->name : ""; }
// Records the page layout CImg sets, so that the strip size it asks for is
// large enough for the strips it then fills (and drops).
static inline int TIFFSetField(TIFF *t, uint32 tag, ...) {
    va_list ap;
    va_start(ap, tag);
    switch (tag) {
    case TIFFTAG_IMAGEWIDTH: t->width = va_arg(ap, unsigned); break;
    case TIFFTAG_IMAGELENGTH: t->length = va_arg(ap, unsigned); break;
    case TIFFTAG_SAMPLESPERPIXEL: t->spp = va_arg(ap, unsigned); break;
    case TIFFTAG_BITSPERSAMPLE: t->bps = va_arg(ap, unsigned); break;
    case TIFFTAG_ROWSPERSTRIP: t->rows_per_strip = va_arg(ap, unsigned); break;
    default: break;
    }
    va_end(ap);
    return 1;
}
static inline int TIFFGetField(TIFF *, uint32, ...) { return 0; }
static inline int TIFFGetFieldDefaulted(TIFF *, uint32, ...) { return 0; }
static inline tsize_t TIFFWriteEncodedStrip(TIFF *, tstrip_t, tdata_t, tsize_t n) { return n; }
static inline int TIFFWriteDirectory(TIFF *) { return 1; }
static inline uint32 TIFFDefaultStripSize(TIFF *t, uint32 r) {
    // libtiff's rule for a request below 1 (CImg passes (uint32)-1): strips of about 8 KiB
    if ((int32)r >= 1) return r;
    const uint32 line = t->width * t->spp * (t->bps / 8);
    return line && line < 8192 ? 8192 / line : 1;
}
static inline tsize_t TIFFStripSize(TIFF *t) {
    const uint32 rows = t->rows_per_strip < t->length ? t->rows_per_strip : t->length;
    return (tsize_t)rows * t->width * t->spp * (t->bps / 8);
}
static inline tsize_t TIFFTileSize(TIFF *) { return 0; }
static inline tstrip_t TIFFComputeStrip(TIFF *, uint32, uint16) { return 0; }
static inline int TIFFIsTiled(TIFF *) { return 0; }
static inline int TIFFReadDirectory(TIFF *) { return 0; }
static inline int TIFFSetDirectory(TIFF *, uint16) { return 0; }
static inline tsize_t TIFFReadEncodedStrip(TIFF *, tstrip_t, tdata_t, tsize_t) { return -1; }
static inline tsize_t TIFFReadTile(TIFF *, tdata_t, uint32, uint32, uint32, uint16) { return -1; }
static inline int TIFFReadRGBAImage(TIFF *, uint32, uint32, uint32 *, int) { return 0; }
static inline TIFFErrorHandler TIFFSetErrorHandler(TIFFErrorHandler) { return 0; }
static inline TIFFErrorHandler TIFFSetWarningHandler(TIFFErrorHandler) { return 0; }
static inline tdata_t _TIFFmalloc(tsize_t n) { return std::malloc((size_t)n); }
static inline void _TIFFfree(tdata_t p) { std::free(p); }
#endif
