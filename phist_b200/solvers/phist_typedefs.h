/* Index and handle types of the b200 kernel library, in the form PHIST's
 * phist_kernels.h expects from a kernel library directory (the builtin
 * library's src/kernels/builtin/phist_typedefs.h has the same content:
 * 32-bit local and 64-bit global indices, void-pointer handle aliases). */
#ifndef PHIST_TYPEDEFS_H
#define PHIST_TYPEDEFS_H
#include "phist_config.h"
#include <inttypes.h>
#ifdef __cplusplus
#include <complex>
typedef std::complex<float> phist_s_complex;
typedef std::complex<double> phist_d_complex;
#else
#include <complex.h>
typedef complex float phist_s_complex;
typedef complex double phist_d_complex;
#endif
typedef int32_t phist_lidx;
typedef int64_t phist_gidx;
#define PRlidx "d"
#define PRgidx "ld"
#include "phist_void_aliases.h"
#endif
