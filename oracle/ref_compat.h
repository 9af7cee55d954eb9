/*
 * ref_compat.h -- force-included when the reference (frsykzk/MPS_CUDA, an MSVC project) is
 * compiled with nvcc + g++ by ref_build.sh. Maps the MSVC "_s" stdio functions used in
 * kernel.cu onto their C equivalents. Test infrastructure only.
 */
#pragma once
#include <stdio.h>
#include <string.h>

#define printf_s printf
#define fprintf_s fprintf
#define fscanf_s fscanf
#define sprintf_s sprintf

static inline int fopen_s(FILE** f, const char* name, const char* mode) {
    *f = fopen(name, mode);
    return *f ? 0 : 1;
}
