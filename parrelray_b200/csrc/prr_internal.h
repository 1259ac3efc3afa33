// prr_internal.h - the context behind the C ABI and the render plan that
// turns an array of prr_frame_desc into launches.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "kernels.cuh"
#include "prr.h"

struct DevBuf {
    void *p = nullptr;
    size_t cap = 0;
    prr_status ensure(size_t bytes);  // grow-only
    void release();
};

struct TexSlot {
    DevBuf buf;
    int w = 0, h = 0;
};

// The plasma grid of prr_upload_plasma (density, temperature and velocity as
// float4 per node, each on the device; the last two optional).
struct PlasmaGrid {
    DevBuf n, theta, vel;
    bool present = false, has_theta = false, has_vel = false;
    int nx = 0, ny = 0, nz = 0;
    float lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
};

// A loaded metric plug-in library (compat/prr_plugin.cuh).
struct MetricPlugin {
    std::string path, name;
    void *handle = nullptr;
    size_t ray_bytes = 0;
    // REFERENCE mode (prr_plugin_trace) and PHYSICAL mode (prr_plugin_trace_physical), same arguments
    int (*trace)(const void *h_fp, const void *d_fps, int frame, long long nrays, void *d_rays, float *d_state,
                 float *d_rgb, unsigned long long *d_counters, void *stream) = nullptr;
    int (*trace_physical)(const void *h_fp, const void *d_fps, int frame, long long nrays, void *d_rays, float *d_state,
                          float *d_rgb, unsigned long long *d_counters, void *stream) = nullptr;
};

struct prr_ctx {
    int device = 0;
    int nsm = 0;
    int sm_clock_khz = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr, t0 = nullptr, t1 = nullptr;
    std::string err;
    TexSlot tex[PRR_MAX_TEXTURES];
    PlasmaGrid plasma;
    int schedule = PRR_SCHED_PERSISTENT;
    prr_launch_config cfg{};
    int geod_table = -1;  // -1: per schedule (PERSISTENT contraction, PLAIN table); 0: contraction; 1: table
    int hamiltonian = PRR_HAM_FP32 | PRR_HAM_FP64;  // renders in Hamiltonian form (PRR_OPT_HAMILTONIAN)
    long long watchdog_cycles = 0;
    std::vector<MetricPlugin> plugins;
    int *ray_steps_out = nullptr;  // set by prr_adjoint around its forward render: per-ray accepted steps
    int last_launches = 0;
    float last_ms = 0.f;
    float last_trace_ms = 0.f;
    // device scratch, grown on demand and reused across calls
    DevBuf frames, frame_begin, counters, image, sample_rgb, rays, queue, state, out_u8, out_f, scratch, adj_ckpt, adj_dl,
        adj_sort;
    std::vector<DevBuf *> all_buffers()
    {
        return {&frames, &frame_begin, &counters, &image, &sample_rgb, &rays, &queue, &state, &out_u8, &out_f, &scratch,
                &adj_ckpt, &adj_dl, &adj_sort, &plasma.n, &plasma.theta, &plasma.vel};
    }
};

// Host-side description of one render call.
struct RenderPlan {
    std::vector<prr::FrameParams> fp;
    std::vector<long long> pix_begin;  // nframes + 1
    std::vector<long long> ray_begin;  // nframes + 1
    long long total_pixels = 0;
    long long total_rays = 0;
    int mode = PRR_MODE_PHYSICAL;
    int precision = PRR_PREC_FP32;
    bool any_fxaa = false;
    bool any_emission = false;  // some frame has plasma emission
    bool plugin = false;        // the frames use metric plug-ins (then every frame does)
};

// The plug-in of a frame's metric id, or null for a built-in metric.
inline const MetricPlugin *frame_plugin(const prr_ctx *ctx, int metric)
{
    int k = metric - PRR_METRIC_PLUGIN0;
    return (k >= 0 && k < (int)ctx->plugins.size()) ? &ctx->plugins[k] : nullptr;
}

// render.cu
prr_status build_plan(prr_ctx *ctx, const prr_frame_desc *frames, int n, RenderPlan &plan);
// Runs a plan into device outputs (either may be null).  When `timed`, the
// device time between two events around the launches is kept in ctx->last_ms.
prr_status run_plan(prr_ctx *ctx, const RenderPlan &plan, uint8_t *d_rgb8, float *d_rgbf, cudaStream_t st, bool timed);
// Single frame: per-ray states and per-sample colours to host buffers.
prr_status trace_plan(prr_ctx *ctx, const RenderPlan &plan, float *h_state, double *h_state64, float *h_rgb);
prr_status collect_stats(prr_ctx *ctx, const RenderPlan &plan, prr_stats *stats);
// Resident CTAs per SM of the persistent kernel under the context's launch
// configuration (its blocks_per_sm, or the occupancy limit when that is 0).
int resolve_bpsm(prr_ctx *ctx, int precision, bool emission = false);
