#pragma once
// prr_plugin.cuh - the REFERENCE-mode and PHYSICAL-mode renderers built
// around an unchanged ParRelRay metric plug-in header.
//
// The reference's "plug-in API" is compile-time: main/metric.h includes one
// header from metrics/ that defines getMetric, getGeod, User_LOOP,
// User_UPDATE, User_ENDLOOP and the rayToRGB kernel, and the solver
// (kernels/solver.cuh) and frame loop (prr.cpp:237-341) call them.  The
// plug-in build (parrelray_b200/build.py: build_metric_plugin) places such a
// header in a directory beside this library's compatibility tree
// (compat/main, compat/cudamaths, compat/scene: the reference's type shapes)
// and compiles one translation unit:
//
//     #include "metrics/<header>"   // the plug-in, unchanged
//     #include "prr_plugin.cuh"     // this file
//
// into libprr_metric_<name>.so.  prr_load_metric_plugin() loads it into a
// context; frames whose metric is the id it returns are traced here:
//   k_plugin_trace  ray placement (createRays_none/regular), initRays with the
//                   header's getMetric, and trace_RKF / trace_Euler with the
//                   header's getGeod and hooks (the library's solver, which
//                   follows kernels/solver.cuh step for step, instantiated on
//                   the header's hooks); writes the 48-byte Ray records;
//   rayToRGB        the header's own kernel, launched as prr.cpp:317-319 does;
//   k_plugin_collect per-sample colours and counters.
// PHYSICAL-mode frames (FP32) run k_plugin_phys instead of k_plugin_trace:
// the same hooks on the persistent, warp-compacted scheduler with the
// PHYSICAL stepper (hook_stepper.cuh).
// SSAA combine, FXAA and quantisation then run in the library as for the
// built-in metrics.
//
// PRR_PLUGIN_PART selects what a translation unit holds: 1 the REFERENCE
// renderer, the colouring (the header's rayToRGB) and the library's metadata
// entry points, built with -fmad=false as the built-in REFERENCE path, so the
// header's FP32 arithmetic is the reference's operation for operation; 2 the
// PHYSICAL renderer, built with contraction on (its bar is the FP64 oracle,
// not the reference's rounding), which colours through part 1's
// prr_plugin_colour; 0 (or undefined) both, in one translation unit.
#include <algorithm>

#include "hook_stepper.cuh"
#include "kernels.cuh"
#include "ref_stepper.cuh"

#ifndef PRR_PLUGIN_NAME
#define PRR_PLUGIN_NAME "plugin"
#endif
#ifndef PRR_PLUGIN_PART
#define PRR_PLUGIN_PART 0
#endif
#define PRR_PLUGIN_HAS_REFERENCE (PRR_PLUGIN_PART == 0 || PRR_PLUGIN_PART == 1)
#define PRR_PLUGIN_HAS_PHYSICAL (PRR_PLUGIN_PART == 0 || PRR_PLUGIN_PART == 2)

namespace prr_plugin {

using prr::FrameParams;
using prr::RefRay;
using prr::V4;

// The reference's by-value kernel arguments for one frame.  `d_fp` is the
// frame's parameter block in device memory (the scene's spheres).
__host__ __device__ inline Camera make_camera(const FrameParams &fp)
{
    Camera c(f3(fp.cam[0], fp.cam[1], fp.cam[2]), fp.alpha, fp.beta, fp.vfov, i2(fp.width, fp.height),
             fp.ssaa == 0 ? SSAA_DISTR::NONE : SSAA_DISTR::REGULAR, fp.samples);
    c.computeVectors();
#ifdef SPHERICAL
    c.spos = pos_cartTOspher(c.pos);  // prr.cpp:250-252
#endif
    return c;
}

__host__ __device__ inline Spacetime make_space(const FrameParams &fp, const FrameParams *d_fp)
{
    Spacetime s;
    s.setBhMass(fp.M);
    s.setBhSpin(fp.a);
    s.fp = d_fp;
    return s;
}

__host__ __device__ inline Tracer make_tracer(const FrameParams &fp)
{
    Tracer t;
    t.h = fp.h; t.hmin = fp.hmin; t.hmax = fp.hmax; t.eps = fp.eps;
    t.sph1.tex = tex2d(fp.bg);
    t.sph1.rout = fp.rout;
    t.sph2.tex = tex2d();
    t.sph2.rout = fp.rout;
    t.solver = fp.solver == PRR_SOLVER_EULER ? SOLVER::EULER : SOLVER::RUNGE_KUTTA_FEHLBERG;
    return t;
}

__device__ inline void to_ray(const RefRay &R, Ray &T)
{
    T.uv = f2(R.uvx, R.uvy);
    T.result = (RESULT)R.result;
    T.r = f4(R.r.x, R.r.y, R.r.z, R.r.w);
    T.u = f4(R.u.x, R.u.y, R.u.z, R.u.w);
    T.I = 0.0f;
}

__device__ inline void from_ray(const Ray &T, RefRay &R)
{
    R.result = (int)T.result;
    R.r = {T.r.x, T.r.y, T.r.z, T.r.w};
    R.u = {T.u.x, T.u.y, T.u.z, T.u.w};
}

// The header's functions as the solver's hook set (ref_stepper.cuh).  A
// header written for SPHERICAL states (r, theta, phi, t) is compiled with
// SPHERICAL defined, as the reference compiles it: its rays then start at
// the camera's spherical position with the spherical rates of the pin-hole
// direction (kernels/solver.cuh:34-37).
struct PluginHooks {
#ifdef SPHERICAL
    static constexpr bool kSpherical = true;
#else
    static constexpr bool kSpherical = false;
#endif
    Camera cam;
    Spacetime space;
    Tracer trace;

    __device__ void spherical_start(RefRay &R, V4<float> &u) const
    {
        Camera c = cam;
        f3 v = vel_cartTOspher(c.pos, c.rayDir_PinHole(f2(R.uvx, R.uvy)));
        u = {v.x, v.y, v.z, 1.0f};
        R.r = {c.spos.x, c.spos.y, c.spos.z, 0.0f};
    }

    __device__ void metric(const RefRay &R, float g[16]) const
    {
        Ray T;
        to_ray(R, T);
        mat4 m = getMetric(&T, space);
        for (int i = 0; i < 16; i++) g[i] = m.e[i];
    }
    __device__ V4<float> geod(const V4<float> &x, const V4<float> &u) const
    {
        f4 d = getGeod(f4(x.x, x.y, x.z, x.w), f4(u.x, u.y, u.z, u.w), space);
        return {d.x, d.y, d.z, d.w};
    }
    __device__ bool loop(RefRay &R) const
    {
        Ray T;
        to_ray(R, T);
        bool go = User_LOOP(&T, cam, space);
        from_ray(T, R);
        return go;
    }
    __device__ bool update(RefRay &R, float h) const
    {
        Ray T;
        to_ray(R, T);
        bool go = User_UPDATE(&T, cam, space, h);
        from_ray(T, R);
        return go;
    }
    __device__ bool endloop(RefRay &R, float trace_h) const
    {
        Ray T;
        to_ray(R, T);
        Tracer t = trace;
        t.h = trace_h;  // trace_RKF passes its tracer with h = the last accepted step (solver.cuh:199)
        bool go = User_ENDLOOP(&T, cam, space, t);
        from_ray(T, R);
        return go;
    }
};

__device__ __forceinline__ void warp_add(unsigned long long *p, unsigned long long v)
{
    unsigned mask = __activemask();
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o);
    if ((threadIdx.x & 31) == (__ffs(mask) - 1)) atomicAdd(p, v);
}

#if PRR_PLUGIN_HAS_REFERENCE
__global__ void __launch_bounds__(128) k_plugin_trace(const FrameParams *__restrict__ fps, int frame, long long nrays,
                                                      Ray *__restrict__ rays, float *__restrict__ state,
                                                      unsigned long long *__restrict__ counters)
{
    long long rid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (rid >= nrays) return;
    const FrameParams &fp = fps[frame];
    const int S = fp.samples;
    long long pix = rid / S;
    int s = (int)(rid - pix * S);
    int x = (int)(pix % fp.width), y = (int)(pix / fp.width);
    PluginHooks hk{make_camera(fp), make_space(fp, &fps[frame]), make_tracer(fp)};
    RefRay R;
    prr::ref_init_h(fp, hk, x, y, s, R);
    if (fp.solver == PRR_SOLVER_EULER) prr::ref_euler_h(fp, hk, R);
    else prr::ref_rkf_h(fp, hk, R);
    Ray T;
    to_ray(R, T);
    rays[rid] = T;
    if (state) {
        float *o = state + 12 * rid;
        o[0] = R.uvx; o[1] = R.uvy; o[2] = (float)R.result;
        o[3] = R.r.x; o[4] = R.r.y; o[5] = R.r.z; o[6] = R.r.w;
        o[7] = R.u.x; o[8] = R.u.y; o[9] = R.u.z; o[10] = R.u.w;
        o[11] = (float)R.accepted;
    }
    if (counters) {
        warp_add(&counters[prr::C_RAYS], 1ull);
        warp_add(&counters[prr::C_ATTEMPTS], (unsigned long long)R.attempts);
        warp_add(&counters[prr::C_ACCEPTED], (unsigned long long)R.accepted);
    }
}

#endif  // PRR_PLUGIN_HAS_REFERENCE

#if PRR_PLUGIN_HAS_PHYSICAL
// PHYSICAL mode through the header's hooks (hook_stepper.cuh) on the
// persistent scheduler: CTAs stay resident and each lane integrates one ray
// at a time, one RKF45 attempt per loop iteration; every `interval` attempts
// (or when the whole warp is idle) the lanes whose ray has ended are refilled
// together - __ballot_sync finds them, one atomicAdd on the frame's work
// counter reserves __popc of them rays, each lane takes base + its rank - so a
// warp never waits for its slowest ray.  Finished rays are written as Ray
// records for the header's rayToRGB, as the reference's pipeline hands them
// on (prr.cpp:317-319).  counters[C_WORK] must be zero at launch.
__global__ void __launch_bounds__(128) k_plugin_phys(const FrameParams *__restrict__ fps, int frame, long long nrays,
                                                     Ray *__restrict__ rays, float *__restrict__ state,
                                                     unsigned long long *__restrict__ counters, int interval)
{
    constexpr unsigned FULL = 0xffffffffu;
    const FrameParams &fp = fps[frame];
    const int lane = threadIdx.x & 31;
    const PluginHooks hk{make_camera(fp), make_space(fp, &fps[frame]), make_tracer(fp)};
    prr::HookRay S;
    long long rid = -1;
    bool busy = false, need = true;
    unsigned long long n_rays = 0, n_att = 0, n_acc = 0;
    const unsigned ci = interval > 1 ? (unsigned)interval : 1u;
    unsigned since = ci;
    while (true) {
        if (++since >= ci || __ballot_sync(FULL, busy) == 0) {
            since = 0;
            const unsigned m = __ballot_sync(FULL, need);
            if (m) {
                const int leader = __ffs(m) - 1;
                unsigned long long base = 0;
                if (lane == leader) base = atomicAdd(&counters[prr::C_WORK], (unsigned long long)__popc(m));
                base = __shfl_sync(FULL, base, leader);
                if (need) {
                    rid = (long long)(base + __popc(m & ((1u << lane) - 1u)));
                    need = false;
                    busy = rid < nrays;
                    if (busy) {
                        const int S_ = fp.samples;
                        const long long pix = rid / S_;
                        prr::hook_phys_init(fp, hk, (int)(pix % fp.width), (int)(pix / fp.width), (int)(rid - pix * S_), S);
                    }
                }
            }
        }
        if (__ballot_sync(FULL, busy) == 0) {
            if (__ballot_sync(FULL, need) == 0) break;  // every lane has drawn past the last ray
            since = ci;
            continue;
        }
        if (!busy) continue;
        if (prr::hook_phys_attempt(fp, hk, S) != prr::STEP_DONE) continue;
        const prr::RefRay &R = S.R;
        Ray T;
        to_ray(R, T);
        rays[rid] = T;
        if (state) {
            float *o = state + 12 * rid;
            o[0] = R.uvx; o[1] = R.uvy; o[2] = (float)R.result;
            o[3] = R.r.x; o[4] = R.r.y; o[5] = R.r.z; o[6] = R.r.w;
            o[7] = R.u.x; o[8] = R.u.y; o[9] = R.u.z; o[10] = R.u.w;
            o[11] = (float)R.accepted;
        }
        n_rays++;
        n_att += (unsigned)R.attempts;
        n_acc += (unsigned)R.accepted;
        busy = false;
        need = true;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        n_rays += __shfl_xor_sync(FULL, n_rays, o);
        n_att += __shfl_xor_sync(FULL, n_att, o);
        n_acc += __shfl_xor_sync(FULL, n_acc, o);
    }
    if (lane == 0 && counters) {
        atomicAdd(&counters[prr::C_RAYS], n_rays);
        atomicAdd(&counters[prr::C_ATTEMPTS], n_att);
        atomicAdd(&counters[prr::C_ACCEPTED], n_acc);
    }
}

#endif  // PRR_PLUGIN_HAS_PHYSICAL

#if PRR_PLUGIN_HAS_REFERENCE
// Per-sample colour (Ray::u after rayToRGB) and outcome counters.
__global__ void k_plugin_collect(const Ray *__restrict__ rays, long long nrays, float rout, float *__restrict__ rgb,
                                 unsigned long long *__restrict__ counters)
{
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nrays) return;
    Ray T = rays[i];
    if (rgb) { rgb[3 * i] = T.u.x; rgb[3 * i + 1] = T.u.y; rgb[3 * i + 2] = T.u.z; }
    if (counters) {
        int cls;
        switch (T.result) {
#ifdef SPHERICAL
        case RESULT::SUCCESS: cls = T.r.x >= rout ? prr::C_ESCAPED : prr::C_CAPTURED; break;
#else
        case RESULT::SUCCESS: cls = T.r.xyz().norm() >= rout ? prr::C_ESCAPED : prr::C_CAPTURED; break;
#endif
        case RESULT::INTERSECTION: cls = prr::C_INTERSECTION; break;
        case RESULT::INFINITE_GEO: cls = prr::C_INFINITE; break;
        default: cls = prr::C_MATH_ERROR;
        }
        atomicAdd(&counters[cls], 1ull);
    }
}

#endif  // PRR_PLUGIN_HAS_REFERENCE

}  // namespace prr_plugin

// ---- the plug-in library's C entry points (loaded by prr_load_metric_plugin) ----

// rayToRGB as renderframe launches it (prr.cpp:317-319) over d_rays, then the
// per-sample colours d_rgb and outcome counters; asynchronous on `stream`.
extern "C" int prr_plugin_colour(const void *h_fp, const void *d_fps, int frame, long long nrays, void *d_rays,
                                 float *d_rgb, unsigned long long *d_counters, void *stream);

#if PRR_PLUGIN_HAS_REFERENCE
extern "C" int prr_plugin_abi_version(void) { return PRR_ABI_VERSION; }
extern "C" size_t prr_plugin_frame_params_size(void) { return sizeof(prr::FrameParams); }
extern "C" size_t prr_plugin_ray_bytes(void) { return sizeof(Ray); }
extern "C" const char *prr_plugin_name(void) { return PRR_PLUGIN_NAME; }

namespace prr_plugin {

inline cudaError_t colour_rays(const FrameParams &fp, const FrameParams *dfp, int frame, long long nrays, Ray *rays,
                               float *d_rgb, unsigned long long *d_counters, cudaStream_t st)
{
    Camera cam = make_camera(fp);
    Spacetime space = make_space(fp, dfp + frame);
    Tracer trace = make_tracer(fp);
    dim3 blocks(fp.samples * fp.width / 8 + 1, fp.height / 8 + 1), threads(8, 8);
    rayToRGB<<<blocks, threads, 0, st>>>(rays, cam, space, trace, fp.samples);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_plugin_collect<<<(unsigned)((nrays + 255) / 256), 256, 0, st>>>(rays, nrays, fp.rout, d_rgb, d_counters);
    return cudaGetLastError();
}

}  // namespace prr_plugin

extern "C" int prr_plugin_colour(const void *h_fp, const void *d_fps, int frame, long long nrays, void *d_rays,
                                 float *d_rgb, unsigned long long *d_counters, void *stream)
{
    return (int)prr_plugin::colour_rays(*(const prr::FrameParams *)h_fp, (const prr::FrameParams *)d_fps, frame,
                                        nrays, (Ray *)d_rays, d_rgb, d_counters, (cudaStream_t)stream);
}

// Traces frame `frame` of the device frame table d_fps (h_fp: the same block
// on the host) into d_rays (nrays Ray records), and writes the per-sample
// colours d_rgb (3 floats/ray) and, when non-null, the per-ray states d_state
// (12 floats/ray) and counters.  Asynchronous on `stream`; returns a
// cudaError_t.
extern "C" int prr_plugin_trace(const void *h_fp, const void *d_fps, int frame, long long nrays, void *d_rays,
                                float *d_state, float *d_rgb, unsigned long long *d_counters, void *stream)
{
    using namespace prr_plugin;
    if (nrays <= 0) return (int)cudaSuccess;
    cudaStream_t st = (cudaStream_t)stream;
    const FrameParams &fp = *(const FrameParams *)h_fp;
    const FrameParams *dfp = (const FrameParams *)d_fps;
    Ray *rays = (Ray *)d_rays;
    const int block = 128;
    k_plugin_trace<<<(unsigned)((nrays + block - 1) / block), block, 0, st>>>(dfp, frame, nrays, rays, d_state, d_counters);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return (int)e;
    return (int)colour_rays(fp, dfp, frame, nrays, rays, d_rgb, d_counters, st);
}
#endif  // PRR_PLUGIN_HAS_REFERENCE

#if PRR_PLUGIN_HAS_PHYSICAL
// PHYSICAL mode (FP32) on the persistent scheduler, same arguments and
// outputs as prr_plugin_trace; d_counters is required (its work counter is
// reset here).  Launches k_plugin_phys with resident CTAs of 128 threads on
// every SM, a warp refill every 16 attempts.
extern "C" int prr_plugin_trace_physical(const void *h_fp, const void *d_fps, int frame, long long nrays, void *d_rays,
                                         float *d_state, float *d_rgb, unsigned long long *d_counters, void *stream)
{
    using namespace prr_plugin;
    if (nrays <= 0) return (int)cudaSuccess;
    if (!d_counters) return (int)cudaErrorInvalidValue;
    cudaStream_t st = (cudaStream_t)stream;
    const FrameParams *dfp = (const FrameParams *)d_fps;
    Ray *rays = (Ray *)d_rays;
    int dev = 0, nsm = 0, bpsm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bpsm, k_plugin_phys, 128, 0);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_counters + prr::C_WORK, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess) return (int)e;
    const long long grid = std::min<long long>((long long)nsm * (bpsm > 0 ? bpsm : 1), (nrays + 127) / 128);
    k_plugin_phys<<<(unsigned)grid, 128, 0, st>>>(dfp, frame, nrays, rays, d_state, d_counters, 16);
    if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;
    return prr_plugin_colour(h_fp, d_fps, frame, nrays, d_rays, d_rgb, d_counters, stream);
}
#endif  // PRR_PLUGIN_HAS_PHYSICAL
