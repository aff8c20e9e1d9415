/* Project-written stand-in for the reference's CMake-configured PLiB/Global.h
 * (template: PLiB/Global.h.in:1-64). Test infrastructure only: it lets the
 * oracle harness compile the reference's CPU hot-path headers from where they
 * lie without running the reference's CMake configure step.
 * Precision follows -DHIDEM_REF_MIXED: defined -> lpReal_t=float (the
 * reference default, SET_FP32 + SET_CT_FP32), else plain FP64. */
#ifndef PHELL_GLOBAL_H
#define PHELL_GLOBAL_H

#define ENABLE_CUDA 0
#define ENABLE_HIP 0
#define ENABLE_SIMD256 0
#define ENABLE_SIMD512 0
#define ENABLE_HDF5
#ifdef _OPENMP
#define ENABLE_OMP
#endif
#ifdef HIDEM_REF_MIXED
#define SET_FP32
#define SET_CT_FP32
#endif

typedef long long int ind_t;
typedef long long int gKey_t;
typedef int pInd_t;
typedef int lInd_t;

#ifdef SET_FP32
typedef float lpReal_t;
#else
typedef double lpReal_t;
#endif
typedef double hpReal_t;

#define REALT_TEMPL
#define REALT_TEMPL_LONG

#endif
