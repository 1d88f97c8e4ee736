/* Test-infrastructure stand-in for libtiff's header (libtiff is not
 * installed here).  It declares the names the reference's mrct.h/mrct.cpp
 * use; oracle/ref_tiff_stub.cpp defines them so that the reference's
 * program links, with TIFFOpen always failing (TIFF input is not used by
 * the reference runs; MRC stacks are). */
#pragma once
#include <stdint.h>
typedef struct tiff TIFF;
typedef uint16_t uint16;
typedef uint32_t uint32;
typedef int64_t tsize_t;
typedef uint32_t tstrip_t;
typedef void* tdata_t;
#define TIFFTAG_IMAGEWIDTH 256
#define TIFFTAG_IMAGELENGTH 257
#define TIFFTAG_BITSPERSAMPLE 258
#ifdef __cplusplus
extern "C" {
#endif
TIFF* TIFFOpen(const char* name, const char* mode);
void TIFFClose(TIFF* t);
int TIFFGetField(TIFF* t, uint32 tag, ...);
int TIFFReadDirectory(TIFF* t);
int TIFFSetDirectory(TIFF* t, uint16 dir);
tsize_t TIFFStripSize(TIFF* t);
tstrip_t TIFFNumberOfStrips(TIFF* t);
tsize_t TIFFReadEncodedStrip(TIFF* t, tstrip_t s, tdata_t buf, tsize_t size);
void TIFFPrintDirectory(TIFF* t, void* fd, long flags);
tdata_t _TIFFmalloc(tsize_t s);
void _TIFFfree(tdata_t p);
#ifdef __cplusplus
}
#endif
