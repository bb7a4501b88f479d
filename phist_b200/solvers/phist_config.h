/* Configuration header for compiling PHIST's unchanged solver layers
 * (src/tools, src/core, src/krylov, src/jada, src/precon of the PHIST sources)
 * against libphist_kernels_b200.so: one process (no MPI), row-major mvecs,
 * double and single precision, no complex types, no third-party libraries.
 * Plays the role of the header CMake generates from src/phist_config.h.in. */
#ifndef PHIST_CONFIG_H
#define PHIST_CONFIG_H
#define PHIST_VERSION_STRING "1.12.0-b200"
#define PHIST_VERSION_MAJOR 1
#define PHIST_VERSION_MINOR 12
#define PHIST_VERSION_PATCH 0
#define PHIST_GIT_REVISION "b200"
#define PHIST_INSTALL_INFO "kernel library: b200 (libphist_kernels_b200.so)\n"
#ifndef PHIST_OUTLEV
#define PHIST_OUTLEV 1
#endif
#define PHIST_HAVE_CXX11_LAMBDAS
#define PHIST_HAVE_CXX11_THREADLOCAL
#define PHIST_HAVE_CXX11_MOVEDEFAULT
#define PHIST_HAVE_SP
#define PHIST_BUILTIN_MEMALIGN 64
#define PHIST_KERNEL_LIB_B200
#define PHIST_MVECS_ROW_MAJOR
/* PHIST_TIMEMONITOR is left undefined: its timer registry is one
 * process-wide map, and the served form drives PHIST's solvers from several
 * host threads at once. */
#endif
