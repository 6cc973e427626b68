/* ref_image.c -- ORACLE harness (test infrastructure only): the reference's vendored
 * stb_image / stb_image_write (external/stb, compiled where they lie) behind a plain
 * C interface, so the tests can compare the library's texture decoder with the
 * decoder the reference uses (src/main.cpp:407-470, stbi_load(..., 4)) and write
 * JPEG fixtures with the reference's own encoder.  Built into oracle/_ref only. */
#define STB_IMAGE_IMPLEMENTATION
#define STB_IMAGE_WRITE_IMPLEMENTATION
#include "stb_image.h"
#include "stb_image_write.h"

#include <string.h>

/* stbi_load_from_memory(..., 4): returns 0 and fills w/h/comp (and out when cap is enough), -1 on failure */
int ref_stbi_decode_rgba(const unsigned char* bytes, int n, unsigned char* out, long long cap, int* w, int* h, int* comp)
{
    int x = 0, y = 0, c = 0;
    unsigned char* px = stbi_load_from_memory(bytes, n, &x, &y, &c, 4);
    if (!px) return -1;
    *w = x; *h = y; *comp = c;
    if (out && cap >= (long long)x * y * 4) memcpy(out, px, (size_t)x * y * 4);
    stbi_image_free(px);
    return 0;
}

const char* ref_stbi_failure(void) { return stbi_failure_reason(); }

int ref_stbi_write_jpg(const char* path, int w, int h, int comp, const unsigned char* data, int quality)
{
    return stbi_write_jpg(path, w, h, comp, data, quality);
}
