// fma_peak.cu - FP32 / FP64 FMA throughput microbenchmark: the roofline
// denominator for the ALU-bound tracer (no FP32/FP64 peak is published for
// the pool's GPUs).  Each thread runs 8 independent dependent-FMA chains, so
// every SM sub-partition has enough independent FMAs in flight to issue one
// per cycle.  FLOPs = grid * block * iters * 16 * 8 * 2.
#include "kernels.cuh"

namespace prr {

template <class T> __global__ void k_fma_peak(T *sink, int iters, T b, T c)
{
    T a0 = (T)threadIdx.x, a1 = a0 + (T)1, a2 = a0 + (T)2, a3 = a0 + (T)3, a4 = a0 + (T)4, a5 = a0 + (T)5,
      a6 = a0 + (T)6, a7 = a0 + (T)7;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 16; k++) {
            a0 = fma(a0, b, c); a1 = fma(a1, b, c); a2 = fma(a2, b, c); a3 = fma(a3, b, c);
            a4 = fma(a4, b, c); a5 = fma(a5, b, c); a6 = fma(a6, b, c); a7 = fma(a7, b, c);
        }
    }
    T s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
    if (s == (T)-12345.678) sink[blockIdx.x] = s;  // never true; keeps the chains live
}

cudaError_t launch_fma_peak(float *sink, int blocks, int threads, int iters, cudaStream_t st)
{
    k_fma_peak<float><<<blocks, threads, 0, st>>>(sink, iters, 0.9999999f, 1e-7f);
    return cudaGetLastError();
}

cudaError_t launch_dfma_peak(double *sink, int blocks, int threads, int iters, cudaStream_t st)
{
    k_fma_peak<double><<<blocks, threads, 0, st>>>(sink, iters, 0.9999999999, 1e-12);
    return cudaGetLastError();
}

// The reciprocal and reciprocal square root of the PHYSICAL path
// (prr_device.cuh frcp/frsqrt) on x[i]: out[4i .. 4i+3] = FP64 1/x, FP64
// 1/sqrt(x), FP32 1/(float)x, FP32 1/sqrt((float)x), for tests of their
// error against the correctly rounded values.
__global__ void k_check_recip(const double *x, int n, double *out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double v = x[i];
    out[4 * i] = frcp<double>(v);
    out[4 * i + 1] = frsqrt<double>(v);
    out[4 * i + 2] = (double)frcp<float>((float)v);
    out[4 * i + 3] = (double)frsqrt<float>((float)v);
}

cudaError_t launch_check_recip(const double *x, int n, double *out, cudaStream_t st)
{
    k_check_recip<<<(n + 255) / 256, 256, 0, st>>>(x, n, out);
    return cudaGetLastError();
}

}  // namespace prr
