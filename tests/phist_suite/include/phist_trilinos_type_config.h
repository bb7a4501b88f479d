/* Stand-in for the header PHIST's CMake generates when Trilinos is present:
 * without Trilinos it defines nothing, so the Belos interface tests of the
 * kernel suite stay compiled out. */
#ifndef PHIST_TRILINOS_TYPE_CONFIG_H
#define PHIST_TRILINOS_TYPE_CONFIG_H
#endif
