// graph.cu - a batch of PHYSICAL-mode frames (a camera trajectory, a set of
// render requests) recorded once into a CUDA graph and replayed.
//
// The graph holds: a memset of the device counters, ONE persistent launch
// over every frame of the batch (the warp-compacted scheduler of
// k_persistent.cu walks all frames from one work counter, so frames of
// uneven cost fill each other's tails), the FP64 re-integration pass for
// split precision, and the per-frame SSAA-combine / FXAA / quantise passes
// where a frame needs them.  Everything it touches on the device is owned
// by the prr_graph object, so the context's own buffers (and later render
// calls on the context) do not disturb it.  The launch shape is the
// context's at creation time (after prr_autotune, the tuned one).
//
// The reference renders a trajectory as a host loop of per-frame pipelines
// (prr.cpp:382-386 calling renderframe, prr.cpp:237-341), each a dozen
// synchronised launches.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "kernels.cuh"
#include "prr_internal.h"

using namespace prr;

struct prr_graph {
    prr_ctx *ctx = nullptr;
    RenderPlan plan;
    DevBuf frames, frame_begin, counters, image, sample_rgb, queue;
    uint8_t *d_rgb8 = nullptr;
    float *d_rgbf = nullptr;
    cudaStream_t capture = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t done = nullptr;  // recorded after each replay
    int launches = 0;
    int bpsm = 1;
    prr_launch_config cfg{};
    bool launched = false;
};

#define PRR_GCK(g, expr)                                                                                   \
    do {                                                                                                   \
        cudaError_t _e = (expr);                                                                           \
        if (_e != cudaSuccess) {                                                                           \
            (g)->ctx->err = std::string(#expr) + ": " + cudaGetErrorString(_e);                           \
            return PRR_ERR_CUDA;                                                                           \
        }                                                                                                  \
    } while (0)

namespace {

prr_status galloc(prr_graph *g, DevBuf &b, size_t bytes, const char *what)
{
    if (b.ensure(bytes) != PRR_OK) {
        g->ctx->err = std::string("prr_graph: out of device memory for ") + what + " (" + std::to_string(bytes) + " bytes)";
        return PRR_ERR_NOMEM;
    }
    return PRR_OK;
}

void release(prr_graph *g)
{
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    if (g->capture) cudaStreamDestroy(g->capture);
    if (g->done) cudaEventDestroy(g->done);
    for (DevBuf *b : {&g->frames, &g->frame_begin, &g->counters, &g->image, &g->sample_rgb, &g->queue}) b->release();
}

// Launches of one replay, issued on `st` (under capture when recording).
prr_status record(prr_graph *g, cudaStream_t st)
{
    prr_ctx *ctx = g->ctx;
    const RenderPlan &plan = g->plan;
    const int n = (int)plan.fp.size();
    g->launches = 0;
    PRR_GCK(g, cudaMemsetAsync(g->counters.p, 0, C_COUNT * sizeof(unsigned long long), st));
    PersistentArgs a;
    memset(&a, 0, sizeof(a));
    a.frames = (const FrameParams *)g->frames.p;
    a.frame_pix_begin = (const long long *)g->frame_begin.p;
    a.nframes = n;
    a.total_pixels = plan.total_pixels;
    a.counters = (unsigned long long *)g->counters.p;
    a.geod_table = ctx->geod_table == 1;
    a.hamiltonian = ctx->hamiltonian;
    a.compaction_interval = g->cfg.compaction_interval;
    a.watchdog_cycles = ctx->watchdog_cycles;
    a.rays_per_thread = g->cfg.rays_per_thread;
    a.emission = plan.any_emission;
    a.image = (float *)g->image.p;
    float *image = (float *)g->image.p;
    if (plan.precision == PRR_PREC_SPLIT) {
        a.sample_rgb = (float *)g->sample_rgb.p;
        a.fp64_queue = (unsigned long long *)g->queue.p;
        a.fp64_capacity = plan.total_rays;
        PRR_GCK(g, launch_persistent(a, PRR_PREC_SPLIT, g->cfg.block_size, g->bpsm, ctx->nsm, st));
        PRR_GCK(g, launch_fp64_requeue(a, 128, ctx->nsm, st));
        g->launches += 2;
        for (int f = 0; f < n; f++) {
            const FrameParams &p = plan.fp[f];
            PRR_GCK(g, launch_combine(a.sample_rgb + 3 * p.ray_begin, p.width, p.height, p.samples, image + 3 * p.pix_begin, st));
            PRR_GCK(g, launch_finish(image + 3 * p.pix_begin, p.width, p.height, p.fxaa,
                                     g->d_rgbf ? g->d_rgbf + 3 * p.pix_begin : nullptr,
                                     g->d_rgb8 ? g->d_rgb8 + 3 * p.pix_begin : nullptr, st));
            g->launches += 2;
        }
        return PRR_OK;
    }
    a.rgb8 = g->d_rgb8;
    PRR_GCK(g, launch_persistent(a, plan.precision, g->cfg.block_size, g->bpsm, ctx->nsm, st));
    g->launches += 1;
    for (int f = 0; f < n; f++) {
        const FrameParams &p = plan.fp[f];
        const size_t npx = (size_t)p.width * p.height;
        float *img = image + 3 * p.pix_begin;
        if (p.fxaa) {
            PRR_GCK(g, launch_finish(img, p.width, p.height, 1, g->d_rgbf ? g->d_rgbf + 3 * p.pix_begin : nullptr,
                                     g->d_rgb8 ? g->d_rgb8 + 3 * p.pix_begin : nullptr, st));
            g->launches += 1;
        } else if (g->d_rgbf) {
            PRR_GCK(g, cudaMemcpyAsync(g->d_rgbf + 3 * p.pix_begin, img, npx * 3 * sizeof(float), cudaMemcpyDeviceToDevice, st));
        }
    }
    return PRR_OK;
}

prr_status upload(prr_graph *g)
{
    const RenderPlan &plan = g->plan;
    const size_t n = plan.fp.size();
    PRR_GCK(g, cudaMemcpy(g->frames.p, plan.fp.data(), n * sizeof(FrameParams), cudaMemcpyHostToDevice));
    PRR_GCK(g, cudaMemcpy(g->frame_begin.p, plan.pix_begin.data(), (n + 1) * sizeof(long long), cudaMemcpyHostToDevice));
    return PRR_OK;
}

}  // namespace

extern "C" prr_status prr_graph_create(prr_ctx *ctx, const prr_frame_desc *frames, int n, uint8_t *d_rgb8, float *d_rgbf,
                                       prr_graph **out)
{
    if (!ctx) return PRR_ERR_INVALID;
    if (!out) { ctx->err = "prr_graph_create: null output handle"; return PRR_ERR_INVALID; }
    *out = nullptr;
    if (!d_rgb8 && !d_rgbf) { ctx->err = "prr_graph_create: need at least one device output"; return PRR_ERR_INVALID; }
    prr_graph *g = new prr_graph();
    g->ctx = ctx;
    prr_status s = build_plan(ctx, frames, n, g->plan);
    if (s == PRR_OK && g->plan.mode != PRR_MODE_PHYSICAL) {
        ctx->err = "prr_graph_create: graphs record the PHYSICAL-mode persistent renderer; REFERENCE frames render with prr_render";
        s = PRR_ERR_UNSUPPORTED;
    }
    if (s == PRR_OK && g->plan.plugin) {
        ctx->err = "prr_graph_create: graphs record the built-in metrics; metric plug-in frames render with prr_render";
        s = PRR_ERR_UNSUPPORTED;
    }
    if (s != PRR_OK) { delete g; return s; }
    if (cudaSetDevice(ctx->device) != cudaSuccess) { ctx->err = "prr_graph_create: cudaSetDevice failed"; delete g; return PRR_ERR_CUDA; }
    const RenderPlan &plan = g->plan;
    const size_t nf = plan.fp.size();
    g->d_rgb8 = d_rgb8;
    g->d_rgbf = d_rgbf;
    g->cfg = ctx->cfg;
    g->bpsm = resolve_bpsm(ctx, plan.precision, plan.any_emission);
    if ((s = galloc(g, g->frames, nf * sizeof(FrameParams), "frame parameters")) != PRR_OK ||
        (s = galloc(g, g->frame_begin, (nf + 1) * sizeof(long long), "frame table")) != PRR_OK ||
        (s = galloc(g, g->counters, C_COUNT * sizeof(unsigned long long), "counters")) != PRR_OK ||
        (s = galloc(g, g->image, (size_t)plan.total_pixels * 3 * sizeof(float), "image")) != PRR_OK) {
        release(g); delete g; return s;
    }
    if (plan.precision == PRR_PREC_SPLIT &&
        ((s = galloc(g, g->sample_rgb, (size_t)plan.total_rays * 3 * sizeof(float), "per-sample colours")) != PRR_OK ||
         (s = galloc(g, g->queue, (size_t)plan.total_rays * sizeof(unsigned long long), "FP64 queue")) != PRR_OK)) {
        release(g); delete g; return s;
    }
    if ((s = upload(g)) != PRR_OK) { release(g); delete g; return s; }
    if (cudaStreamCreateWithFlags(&g->capture, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&g->done, cudaEventDisableTiming) != cudaSuccess) {
        ctx->err = "prr_graph_create: cudaStreamCreate/cudaEventCreate failed"; release(g); delete g; return PRR_ERR_CUDA;
    }
    cudaError_t e = cudaStreamBeginCapture(g->capture, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) { ctx->err = std::string("cudaStreamBeginCapture: ") + cudaGetErrorString(e); release(g); delete g; return PRR_ERR_CUDA; }
    s = record(g, g->capture);
    cudaGraph_t graph = nullptr;
    e = cudaStreamEndCapture(g->capture, &graph);
    g->graph = graph;
    if (s == PRR_OK && e != cudaSuccess) { ctx->err = std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e); s = PRR_ERR_CUDA; }
    if (s == PRR_OK) {
        e = cudaGraphInstantiate(&g->exec, g->graph, 0);
        if (e != cudaSuccess) { ctx->err = std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e); s = PRR_ERR_CUDA; }
    }
    if (s != PRR_OK) { cudaGetLastError(); release(g); delete g; return s; }
    *out = g;
    return PRR_OK;
}

extern "C" prr_status prr_graph_set_frames(prr_graph *g, const prr_frame_desc *frames, int n)
{
    if (!g) return PRR_ERR_INVALID;
    prr_ctx *ctx = g->ctx;
    if (n != (int)g->plan.fp.size()) { ctx->err = "prr_graph_set_frames: frame count differs from the recorded batch"; return PRR_ERR_INVALID; }
    RenderPlan plan;
    prr_status s = build_plan(ctx, frames, n, plan);
    if (s != PRR_OK) return s;
    if (plan.mode != g->plan.mode || plan.precision != g->plan.precision) {
        ctx->err = "prr_graph_set_frames: mode and precision must match the recorded batch";
        return PRR_ERR_INVALID;
    }
    for (int f = 0; f < n; f++) {
        const FrameParams &a = plan.fp[f], &b = g->plan.fp[f];
        if (a.width != b.width || a.height != b.height || a.samples != b.samples || a.fxaa != b.fxaa) {
            ctx->err = "prr_graph_set_frames: frame " + std::to_string(f) + " changes size, samples or FXAA";
            return PRR_ERR_INVALID;
        }
    }
    if (cudaSetDevice(ctx->device) != cudaSuccess) { ctx->err = "prr_graph_set_frames: cudaSetDevice failed"; return PRR_ERR_CUDA; }
    // the previous replay may still read the table
    if (g->launched) PRR_GCK(g, cudaEventSynchronize(g->done));
    g->plan = plan;
    return upload(g);
}

extern "C" prr_status prr_graph_launch(prr_graph *g, void *stream)
{
    if (!g) return PRR_ERR_INVALID;
    cudaStream_t st = (cudaStream_t)stream;
    PRR_GCK(g, cudaGraphLaunch(g->exec, st));
    PRR_GCK(g, cudaEventRecord(g->done, st));
    g->launched = true;
    return PRR_OK;
}

extern "C" prr_status prr_graph_stats(prr_graph *g, prr_stats *stats)
{
    if (!g) return PRR_ERR_INVALID;
    if (!g->launched) { g->ctx->err = "prr_graph_stats: the graph has not been launched"; return PRR_ERR_INVALID; }
    PRR_GCK(g, cudaEventSynchronize(g->done));
    unsigned long long c[C_COUNT];
    PRR_GCK(g, cudaMemcpy(c, g->counters.p, sizeof(c), cudaMemcpyDeviceToHost));
    if (stats) {
        memset(stats, 0, sizeof(*stats));
        stats->rays = g->plan.total_rays;
        stats->attempts = (int64_t)c[C_ATTEMPTS];
        stats->accepted = (int64_t)c[C_ACCEPTED];
        stats->n_escaped = (int64_t)c[C_ESCAPED];
        stats->n_captured = (int64_t)c[C_CAPTURED];
        stats->n_intersection = (int64_t)c[C_INTERSECTION];
        stats->n_infinite = (int64_t)c[C_INFINITE];
        stats->n_math_error = (int64_t)c[C_MATH_ERROR];
        stats->n_fp64 = (int64_t)c[C_FP64];
        stats->kernel_launches = g->launches;
    }
    if (c[C_TIMEOUT]) { g->ctx->err = "device watchdog expired: some rays were not finished"; return PRR_ERR_TIMEOUT; }
    return PRR_OK;
}

extern "C" prr_status prr_graph_get_launch_config(const prr_graph *g, prr_launch_config *cfg)
{
    if (!g || !cfg) return PRR_ERR_INVALID;
    *cfg = g->cfg;
    cfg->blocks_per_sm = g->bpsm;
    return PRR_OK;
}

extern "C" void prr_graph_destroy(prr_graph *g)
{
    if (!g) return;
    cudaSetDevice(g->ctx->device);
    if (g->launched) cudaEventSynchronize(g->done);
    release(g);
    delete g;
}
