// k_reference.cu - REFERENCE-mode tracing kernel: one thread per ray, with
// ray placement, initRays, trace_RKF/trace_Euler and rayToRGB fused (the
// reference runs them as separate launches, prr.cpp:258-323; fusing them
// changes no arithmetic).  Built with -fmad=false.
#include "kernels.cuh"
#include "ref_stepper.cuh"

namespace prr {

__device__ __forceinline__ void warp_add(unsigned long long *p, unsigned long long v)
{
    unsigned mask = __activemask();
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o);
    if ((threadIdx.x & 31) == (__ffs(mask) - 1)) atomicAdd(p, v);
}

__global__ void __launch_bounds__(128) k_ref_trace(const FrameParams *__restrict__ fps, int frame, long long nrays,
                                                   float *__restrict__ state, float *__restrict__ rgb,
                                                   unsigned long long *__restrict__ counters)
{
    long long rid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (rid >= nrays) return;
    const FrameParams &fp = fps[frame];
    int S = fp.samples;
    long long pix = rid / S;
    int s = (int)(rid - pix * S);
    int x = (int)(pix % fp.width), y = (int)(pix / fp.width);
    RefRay R;
    ref_init(fp, x, y, s, R);
    if (fp.solver == PRR_SOLVER_EULER) ref_euler(fp, R);
    else ref_rkf(fp, R);
    V3<float> c = ray_colour<float>(fp, R.result, R.r, R.u);
    if (state) {
        float *o = state + 12 * rid;
        o[0] = R.uvx; o[1] = R.uvy; o[2] = (float)R.result;
        o[3] = R.r.x; o[4] = R.r.y; o[5] = R.r.z; o[6] = R.r.w;
        o[7] = R.u.x; o[8] = R.u.y; o[9] = R.u.z; o[10] = R.u.w;
        o[11] = (float)R.accepted;
    }
    if (rgb) {
        rgb[3 * rid] = c.x; rgb[3 * rid + 1] = c.y; rgb[3 * rid + 2] = c.z;
    }
    if (counters) {
        warp_add(&counters[C_RAYS], 1ull);
        warp_add(&counters[C_ATTEMPTS], (unsigned long long)R.attempts);
        warp_add(&counters[C_ACCEPTED], (unsigned long long)R.accepted);
        float r = metric_radius<float>(fp, R.r.x, R.r.y, R.r.z);
        int cls = R.result == PRR_RESULT_SUCCESS ? (r >= fp.rout ? C_ESCAPED : C_CAPTURED)
                : R.result == PRR_RESULT_INTERSECTION ? C_INTERSECTION
                : R.result == PRR_RESULT_INFINITE_GEO ? C_INFINITE : C_MATH_ERROR;
        atomicAdd(&counters[cls], 1ull);
    }
}

cudaError_t launch_ref_trace(const FrameParams *d_fp, int frame, long long nrays, float *state, float *rgb,
                             unsigned long long *counters, cudaStream_t st)
{
    if (nrays <= 0) return cudaSuccess;
    const int block = 128;
    long long grid = (nrays + block - 1) / block;
    k_ref_trace<<<(unsigned)grid, block, 0, st>>>(d_fp, frame, nrays, state, rgb, counters);
    return cudaGetLastError();
}

}  // namespace prr
