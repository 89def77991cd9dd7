/* Host stand-ins for the CUDA qualifiers and float intrinsics used by the
 * reference's src/mutils/svd_fast3.cuh and src/mutils/dist_g.cuh, so those two
 * headers compile with g++ for pinning the oracle (TEST INFRASTRUCTURE ONLY).
 * __fadd_rn / __fsub_rn / __fmul_rn are single IEEE round-to-nearest float
 * operations (the file is built with -ffp-contract=off); __frsqrt_rn is the
 * correctly rounded 1/sqrt(x), computed in double and rounded once. */
#pragma once
#include <cmath>
#ifndef __device__
#define __device__
#endif
#ifndef __host__
#define __host__
#endif
#ifndef __forceinline__
#define __forceinline__ inline
#endif
#ifndef __inline__
#define __inline__ inline
#endif
static inline float __fadd_rn(float a, float b) { return a + b; }
static inline float __fsub_rn(float a, float b) { return a - b; }
static inline float __fmul_rn(float a, float b) { return a * b; }
static inline float __frsqrt_rn(float a) { return (float)(1.0 / std::sqrt((double)a)); }
/* CUDA's float overload of max (used unqualified by svd_fast3.cuh) is fmaxf. */
static inline float max(float a, float b) { return std::fmax(a, b); }
