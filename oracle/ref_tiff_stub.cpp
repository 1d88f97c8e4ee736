// Test infrastructure: definitions behind oracle/stubs/tiffio.h so that the
// reference's program links without libtiff.  Opening a TIFF always fails,
// so a TIFF input is rejected the way an unreadable file is.
#include <cstdarg>
#include <cstdlib>

#include "tiffio.h"

extern "C" {
TIFF* TIFFOpen(const char*, const char*) { return nullptr; }
void TIFFClose(TIFF*) {}
int TIFFGetField(TIFF*, uint32, ...) { return 0; }
int TIFFReadDirectory(TIFF*) { return 0; }
int TIFFSetDirectory(TIFF*, uint16) { return 0; }
tsize_t TIFFStripSize(TIFF*) { return 0; }
tstrip_t TIFFNumberOfStrips(TIFF*) { return 0; }
tsize_t TIFFReadEncodedStrip(TIFF*, tstrip_t, tdata_t, tsize_t) { return -1; }
void TIFFPrintDirectory(TIFF*, void*, long) {}
tdata_t _TIFFmalloc(tsize_t s) { return std::malloc((size_t)s); }
void _TIFFfree(tdata_t p) { std::free(p); }
}
