/*
 * Build configuration for compiling the PaStiX reference CPU path as a test
 * oracle (the reference's own CMake cannot run: its spm and morse_cmake
 * submodules are empty).  This plays the role of the reference's
 * include/pastix/config.h.in with the options of a single-node, CPU-only,
 * sequential-BLAS build: no MPI, StarPU, PaRSEC, CUDA, hwloc, Scotch or METIS.
 *
 * Test infrastructure only: nothing in the shipped package includes this.
 */
#ifndef _pastix_config_h_
#define _pastix_config_h_

#define PASTIX_VERSION_MAJOR 6
#define PASTIX_VERSION_MINOR 3
#define PASTIX_VERSION_MICRO 0

/* system */
#define HAVE_SCHED_SETAFFINITY
#define HAVE_CLOCK_GETTIME
#define HAVE_ATOMIC_GCC_32_BUILTINS
#define HAVE_ATOMIC_GCC_64_BUILTINS
#define HAVE_STDARG_H
#define HAVE_UNISTD_H
#define HAVE_VA_COPY
#define HAVE_GETOPT_LONG
#define HAVE_GETRUSAGE
#define HAVE_GETOPT_H
#define HAVE_ERRNO_H
#define HAVE_STDDEF_H
#define HAVE_LIMITS_H
#define HAVE_STRING_H
#define HAVE_COMPLEX_H
#define HAVE_FALLTHROUGH
#define HAVE_BUILTIN_EXPECT
#define HAVE_GETLINE
#define HAVE_MKDTEMP

/* Architecture */
#define PASTIX_ARCH_X86
#define PASTIX_ARCH_X86_64

/* Datatypes used: 64-bit integers, the reference's default */
#define PASTIX_INT64

#include <inttypes.h>

#define pastix_attr_fallthrough __attribute__((fallthrough))

#undef BEGIN_C_DECLS
#undef END_C_DECLS
#if defined(c_plusplus) || defined(__cplusplus)
# define BEGIN_C_DECLS extern "C" {
# define END_C_DECLS }
#else
# define BEGIN_C_DECLS
# define END_C_DECLS
#endif

#endif /* _pastix_config_h_ */
