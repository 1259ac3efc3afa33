// Host-only stand-in for <cuda_runtime.h>, used ONLY to compile the reference
// ParRelRay sources as plain C++ for the CPU oracle (oracle/_ref).  Test
// infrastructure: nothing in the product includes this file.
//
// The reference kernels are written one-thread-per-ray with no shared memory
// and no __syncthreads, so a kernel launch is emulated by running every
// (block, thread) pair of the grid as an ordinary function call, with
// blockIdx/threadIdx held in thread-local storage so OpenMP threads can run
// different blocks concurrently (see prr_ref_launch below).
#pragma once
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <algorithm>

#define __host__
#define __device__
#define __global__
#define __forceinline__ inline

typedef int cudaError_t;
enum { cudaSuccess = 0 };
enum cudaMemcpyKind { cudaMemcpyHostToDevice = 1, cudaMemcpyDeviceToHost = 2, cudaMemcpyDeviceToDevice = 3 };

struct uint3 { unsigned int x, y, z; };
struct dim3 {
    unsigned int x, y, z;
    dim3(unsigned int a = 1, unsigned int b = 1, unsigned int c = 1) : x(a), y(b), z(c) {}
};

extern thread_local uint3 blockIdx;
extern thread_local uint3 threadIdx;
extern thread_local dim3 blockDim;
extern thread_local dim3 gridDim;

static inline cudaError_t cudaMalloc(void **p, size_t n) { *p = calloc(1, n ? n : 1); return *p ? 0 : 2; }
static inline cudaError_t cudaMallocManaged(void **p, size_t n) { return cudaMalloc(p, n); }
static inline cudaError_t cudaFree(void *p) { free(p); return 0; }
static inline cudaError_t cudaMemcpy(void *d, const void *s, size_t n, cudaMemcpyKind) { memcpy(d, s, n); return 0; }
static inline cudaError_t cudaDeviceSynchronize() { return 0; }
static inline cudaError_t cudaDeviceReset() { return 0; }
static inline cudaError_t cudaGetLastError() { return 0; }

// CUDA's device-side min/max on floats are fminf/fmaxf (NaN-ignoring); the
// reference relies on these overloads inside its kernels (solver.cuh:174,
// ssaa.cuh:163-168), so the host build mirrors them.
static inline float min(float a, float b) { return fminf(a, b); }
static inline float max(float a, float b) { return fmaxf(a, b); }
static inline int min(int a, int b) { return a < b ? a : b; }
static inline int max(int a, int b) { return a > b ? a : b; }
