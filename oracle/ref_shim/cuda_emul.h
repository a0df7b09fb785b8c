// Host emulation layer for compiling GSAP/kernels.hpp with g++ (test
// infrastructure; see oracle/build_ref.sh).  A __global__ function becomes a
// plain host function; the harness "launches" it by looping threadIdx.x over
// the index range with blockIdx.x = 0 and blockDim.x = 1, so that
// blockIdx.x * blockDim.x + threadIdx.x is the loop index.  __log2f becomes
// the libm log2f (the reference is built with -use_fast_math, so its logs
// differ from these by a few ulp).  The random-number kernels compile but are
// never called.
#pragma once
#include <cmath>
#include <cstddef>
#include <cstdint>

#define __global__
#define __device__
#define __host__
#define __forceinline__ inline

struct emu_dim3 { unsigned x, y, z; };
extern emu_dim3 threadIdx, blockIdx, blockDim;
static const int warpSize = 32;

static inline float emu_log2f(float x) { return log2f(x); }
#define __log2f emu_log2f
template <typename T> static inline T min(T a, T b) { return a < b ? a : b; }
template <typename T> static inline T __shfl_down_sync(unsigned, T v, unsigned) { return v; }

template <typename T> static inline T atomicAdd(T* p, T v) { T o = *p; *p = o + v; return o; }

struct curandState { unsigned s; };
static inline long long clock64() { return 0; }
static inline void curand_init(unsigned long long, unsigned long long, unsigned long long, curandState* st) { st->s = 0; }
static inline unsigned curand(curandState* st) { return st->s; }
static inline float curand_uniform(curandState*) { return 1.0f; }
