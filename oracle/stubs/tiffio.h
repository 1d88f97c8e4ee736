/* Test-infrastructure stand-in for libtiff's header: the reference's mrct.h
 * only needs the TIFF handle type to declare its class. */
#pragma once
#include <stdint.h>
typedef struct tiff TIFF;
typedef uint16_t uint16;
typedef int64_t tsize_t;
