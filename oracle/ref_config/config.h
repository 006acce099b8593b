/*
 * Hand-written configuration header for compiling the reference (GLU)
 * sources directly with gcc, as its autotools configure step would for a
 * default x86-64 build with FFTW and OpenMP:
 *   NC=3, ND=4, FP64, SSE/AVX intrinsic paths on, FACG (not SD) selected,
 *   MWC_4096 RNG (configure.ac:470-483 default), CONDOR mode (no wisdom).
 * The FFTW it sees is our own API stand-in (oracle/fftw_shim).
 * Test infrastructure only: used by oracle/Makefile, never by the product.
 */
#ifndef GLU_B200_REF_CONFIG_H
#define GLU_B200_REF_CONFIG_H

#define HAVE_COMPLEX_H 1
#define HAVE_FFTW3_H /**/
#define HAVE_IMMINTRIN_H 1
#define HAVE_INTTYPES_H 1
#define HAVE_LIMITS_H 1
#define HAVE_MATH_H 1
#define HAVE_OMP_H 1
#define HAVE_PREFIX "/usr/local"
#define HAVE_STDINT_H 1
#define HAVE_STDIO_H 1
#define HAVE_STDLIB_H 1
#define HAVE_STRINGS_H 1
#define HAVE_STRING_H 1
#define HAVE_SYS_STAT_H 1
#define HAVE_SYS_TIME_H 1
#define HAVE_SYS_TYPES_H 1
#define HAVE_TIME_H 1
#define HAVE_UNISTD_H 1
#define STDC_HEADERS 1

#define PROJ_GRACEY 0
#define TOP_VALUE 1
#define MWC_4096_RNG /**/

#define PACKAGE "glu"
#define PACKAGE_NAME "GLU"
#define PACKAGE_STRING "GLU (oracle build)"
#define PACKAGE_TARNAME "glu"
#define PACKAGE_VERSION "oracle"
#define PACKAGE_BUGREPORT ""
#define PACKAGE_URL ""
#define VERSION "oracle"

#endif
