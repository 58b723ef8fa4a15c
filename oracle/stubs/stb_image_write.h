/* stb_image_write.h -- stand-in for the reference's un-vendored image writer (TEST ORACLE
 * ONLY). The reference's main.cpp (src/main.cpp:23-24, 378) writes its result with
 * stbi_write_hdr; the oracle harness never runs that main and reads the image from memory,
 * so this stand-in only has to compile. It reports failure. */
#ifndef RT_ORACLE_STUB_STB_IMAGE_WRITE_H
#define RT_ORACLE_STUB_STB_IMAGE_WRITE_H

static inline int stbi_write_hdr(const char* path, int w, int h, int comp, const float* data)
{
    (void)path; (void)w; (void)h; (void)comp; (void)data;
    return 0;
}

#endif
