/* Compile-only stand-in for libtiff's <tiff.h> (oracle/_ref build only); the
 * declarations CImg needs are in the tiffio.h stand-in. */
#include "tiffio.h"
