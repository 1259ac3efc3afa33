// Host-only stand-in (oracle build of the reference).  curandState_t exists so
// kernels/ssaa.cuh compiles; its random kernels are never launched by prr.cpp.
#pragma once
#include "cuda_runtime.h"
typedef struct { unsigned long long s; } curandState_t;
typedef curandState_t curandState;
static inline void curand_init(unsigned long long seed, unsigned long long seq, unsigned long long, curandState_t *st) { st->s = seed * 6364136223846793005ULL + seq; }
static inline float curand_uniform(curandState_t *st) { st->s = st->s * 6364136223846793005ULL + 1442695040888963407ULL; return ((st->s >> 40) + 1) * (1.0f / 16777217.0f); }
