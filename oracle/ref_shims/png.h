/*
 * No-op stand-in for <png.h>, used ONLY to compile the reference solver's
 * sources into the CPU oracle binary (oracle/_ref). Image output is not part
 * of the time step; every call here does nothing.
 */
#ifndef MC3D_ORACLE_PNG_SHIM_H
#define MC3D_ORACLE_PNG_SHIM_H

#include <cstdio>

typedef unsigned char png_byte;
typedef png_byte *png_bytep;
typedef png_byte **png_bytepp;
typedef void *png_voidp;
typedef struct mc3d_png_s { int unused; } *png_structp;
typedef struct mc3d_png_info_s { int unused; } *png_infop;
typedef png_structp *png_structpp;
typedef png_infop *png_infopp;

#define PNG_LIBPNG_VER_STRING "shim"
#define PNG_COLOR_TYPE_RGB 2
#define PNG_COLOR_TYPE_GRAY 0
#define PNG_INTERLACE_NONE 0
#define PNG_COMPRESSION_TYPE_DEFAULT 0
#define PNG_FILTER_TYPE_DEFAULT 0

inline png_structp png_create_write_struct(const char *, png_voidp, void *, void *) {
    static mc3d_png_s s; return &s;
}
inline png_infop png_create_info_struct(png_structp) { static mc3d_png_info_s i; return &i; }
inline void png_destroy_write_struct(png_structpp, png_infopp) {}
inline void png_init_io(png_structp, FILE *) {}
inline void png_set_IHDR(png_structp, png_infop, unsigned, unsigned, int, int, int, int, int) {}
inline void png_write_info(png_structp, png_infop) {}
inline void png_write_image(png_structp, png_bytepp) {}
inline void png_write_end(png_structp, png_infop) {}

#endif
