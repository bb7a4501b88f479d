/* Minimal configuration header for compiling a handful of PHIST's own C
 * kernel files (builtin SpMMV non-temporal kernels, double-double dot and
 * Gram kernels) straight from the PHIST sources into oracle/_ref/.  They are
 * used only as a second, independent CPU oracle in the test suite. */
#ifndef PHIST_CONFIG_H
#define PHIST_CONFIG_H
#define PHIST_OUTLEV 1
#define PHIST_HAVE_OPENMP
#define PHIST_HAVE_SSE
#define PHIST_HAVE_AVX
#define PHIST_HAVE_AVX2
#define PHIST_KERNEL_LIB_BUILTIN
#define PHIST_MVECS_ROW_MAJOR
#endif
