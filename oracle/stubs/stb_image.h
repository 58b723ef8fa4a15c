/* stb_image.h -- stand-in for the reference's un-vendored image loader (TEST ORACLE ONLY).
 *
 * The reference's main.cpp (src/main.cpp:26-27, 95-104) includes this header with
 * STB_IMAGE_IMPLEMENTATION defined and calls stbi_loadf / stbi_image_free for its IBL map.
 * The oracle never loads a map through it: the harness hands the reference's IBL struct a
 * float array it allocated with malloc, which stbi_image_free releases. stbi_loadf reports
 * failure, as the reference's loader does for a missing file. */
#ifndef RT_ORACLE_STUB_STB_IMAGE_H
#define RT_ORACLE_STUB_STB_IMAGE_H
#include <stdlib.h>

static inline float* stbi_loadf(const char* path, int* w, int* h, int* channels, int desired)
{
    (void)path; (void)desired;
    *w = 0; *h = 0; *channels = 0;
    return NULL;
}

static inline void stbi_image_free(void* p) { free(p); }

#endif
