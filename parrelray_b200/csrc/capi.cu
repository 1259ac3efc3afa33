// capi.cu - the C ABI of include/prr.h: context, textures, frame
// validation, dispatch to the REFERENCE / PLAIN / PERSISTENT paths, stats.
#include <dlfcn.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "kernels.cuh"
#include "prr.h"
#include "prr_internal.h"

using namespace prr;

namespace {

void fail(prr_ctx *ctx, const std::string &msg)
{
    if (ctx) ctx->err = msg;
}

}  // namespace

#define PRR_CK(ctx, expr)                                                                                  \
    do {                                                                                                   \
        cudaError_t _e = (expr);                                                                           \
        if (_e != cudaSuccess) {                                                                           \
            fail(ctx, std::string(#expr) + ": " + cudaGetErrorString(_e));                                 \
            return PRR_ERR_CUDA;                                                                           \
        }                                                                                                  \
    } while (0)

prr_status DevBuf::ensure(size_t n)
{
    if (n <= cap) return PRR_OK;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    size_t want = std::max(n, (size_t)256);
    if (cudaMalloc(&p, want) != cudaSuccess) { p = nullptr; return PRR_ERR_NOMEM; }
    cap = want;
    return PRR_OK;
}

void DevBuf::release()
{
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
}

extern "C" {

int prr_abi_version(void) { return PRR_ABI_VERSION; }

size_t prr_sizeof(int which)
{
    switch (which) {
    case 0: return sizeof(prr_frame_desc);
    case 1: return sizeof(prr_stats);
    case 2: return sizeof(prr_launch_config);
    case 3: return sizeof(prr_sphere);
    case 4: return sizeof(prr_emission_desc);
    case 5: return sizeof(prr_plasma_desc);
    }
    return 0;
}

const char *prr_status_string(prr_status s)
{
    switch (s) {
    case PRR_OK: return "ok";
    case PRR_ERR_INVALID: return "invalid argument";
    case PRR_ERR_CUDA: return "CUDA error";
    case PRR_ERR_NOMEM: return "out of device memory";
    case PRR_ERR_TIMEOUT: return "device watchdog expired";
    case PRR_ERR_IO: return "I/O error";
    case PRR_ERR_UNSUPPORTED: return "unsupported option";
    case PRR_ERR_NO_DEVICE: return "no usable CUDA device";
    }
    return "unknown status";
}

void prr_frame_desc_defaults(prr_frame_desc *d)
{
    if (!d) return;
    memset(d, 0, sizeof(*d));
    d->width = 320; d->height = 180;
    d->ssaa = PRR_SSAA_NONE; d->samples = 1;
    d->vfov = (float)(60.0 * M_PI / 180.0);
    d->cam_pos[0] = 30.0f;
    d->cam_alpha = (float)M_PI; d->cam_beta = 0.0f;
    d->metric = PRR_METRIC_SCHWARZSCHILD; d->mass = 1.0f; d->spin = 0.0f;
    d->solver = PRR_SOLVER_RKF45; d->mode = PRR_MODE_PHYSICAL; d->precision = PRR_PREC_FP32;
    d->h = 0.01f; d->hmin = 0.0001f; d->hmax = 0.1f;  // input/sim.params:10-12
    d->eps = 0.001f;                                  // input/sim.params:13
    d->rtol = 1e-6f; d->atol = 1e-6f;
    d->rout = 100.0f;
    d->horizon_eps = 0.001f;  // metrics/schwarzschild.cuh:70
    d->max_steps = 10000;
    d->background_id = -1;
    d->bg_filter = PRR_BG_RMS2X2;
    d->fxaa = 0;
    d->fp64_delta = 1e-3f;
    d->fp64_rfac = 1.05f;
    d->nspheres = 0;
    for (int i = 0; i < PRR_MAX_SPHERES; i++) d->spheres[i].texture_id = -1;
    d->emission = PRR_EMISSION_NONE;
    d->emis.index = 2.0f; d->emis.height = 0.3f; d->emis.r_in = 2.0f; d->emis.r_out = 30.0f;
    d->emis.spectral_index = 0.0f; d->emis.absorb = 0.0f; d->emis.gain = 1.0f; d->emis.sense = 1;
    d->emis.temp_power = 0.0f; d->emis.colormap = PRR_CMAP_AFMHOT;
}

prr_status prr_create(int device, prr_ctx **out)
{
    if (!out) return PRR_ERR_INVALID;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) { cudaGetLastError(); return PRR_ERR_NO_DEVICE; }
    if (device < 0 || device >= n) return PRR_ERR_INVALID;
    if (cudaSetDevice(device) != cudaSuccess) { cudaGetLastError(); return PRR_ERR_NO_DEVICE; }
    prr_ctx *ctx = new prr_ctx();
    ctx->device = device;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) { delete ctx; return PRR_ERR_NO_DEVICE; }
    ctx->nsm = prop.multiProcessorCount;
    ctx->sm_clock_khz = prop.clockRate;
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&ctx->e0) != cudaSuccess || cudaEventCreate(&ctx->e1) != cudaSuccess ||
        cudaEventCreate(&ctx->t0) != cudaSuccess || cudaEventCreate(&ctx->t1) != cudaSuccess) {
        delete ctx;
        return PRR_ERR_CUDA;
    }
    ctx->cfg.block_size = 128;
    ctx->cfg.blocks_per_sm = 0;  // 0: occupancy-derived
    ctx->cfg.compaction_interval = 1;
    ctx->cfg.rays_per_thread = 1;
    ctx->schedule = PRR_SCHED_PERSISTENT;
    *out = ctx;
    return PRR_OK;
}

void prr_destroy(prr_ctx *ctx)
{
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (auto &t : ctx->tex) t.buf.release();
    for (DevBuf *b : ctx->all_buffers()) b->release();
    cudaEventDestroy(ctx->e0);
    cudaEventDestroy(ctx->e1);
    cudaEventDestroy(ctx->t0);
    cudaEventDestroy(ctx->t1);
    cudaStreamDestroy(ctx->stream);
    delete ctx;
}

const char *prr_last_error(const prr_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

prr_status prr_load_metric_plugin(prr_ctx *ctx, const char *path, int *metric_id)
{
    if (!ctx) return PRR_ERR_INVALID;
    if (!path || !metric_id) { fail(ctx, "prr_load_metric_plugin: null path or output"); return PRR_ERR_INVALID; }
    for (size_t k = 0; k < ctx->plugins.size(); k++)
        if (ctx->plugins[k].path == path) { *metric_id = PRR_METRIC_PLUGIN0 + (int)k; return PRR_OK; }
    if ((int)ctx->plugins.size() >= PRR_MAX_PLUGINS) { fail(ctx, "prr_load_metric_plugin: PRR_MAX_PLUGINS plug-ins already loaded"); return PRR_ERR_INVALID; }
    void *h = dlopen(path, RTLD_NOW | RTLD_LOCAL);
    if (!h) { fail(ctx, std::string("prr_load_metric_plugin: ") + dlerror()); return PRR_ERR_IO; }
    auto abi = (int (*)(void))dlsym(h, "prr_plugin_abi_version");
    auto fps = (size_t (*)(void))dlsym(h, "prr_plugin_frame_params_size");
    auto rb = (size_t (*)(void))dlsym(h, "prr_plugin_ray_bytes");
    auto nm = (const char *(*)(void))dlsym(h, "prr_plugin_name");
    void *tr = dlsym(h, "prr_plugin_trace");
    void *trp = dlsym(h, "prr_plugin_trace_physical");
    if (!abi || !fps || !rb || !nm || !tr || !trp) {
        dlclose(h);
        fail(ctx, std::string("prr_load_metric_plugin: ") + path + " is not a prr metric plug-in (missing prr_plugin_* symbols)");
        return PRR_ERR_INVALID;
    }
    if (abi() != PRR_ABI_VERSION || fps() != sizeof(FrameParams) || rb() != 48) {
        dlclose(h);
        fail(ctx, std::string("prr_load_metric_plugin: ") + path + " was built for another library version; rebuild it");
        return PRR_ERR_INVALID;
    }
    MetricPlugin pl;
    pl.path = path;
    pl.name = nm();
    pl.handle = h;
    pl.ray_bytes = rb();
    pl.trace = (decltype(pl.trace))tr;
    pl.trace_physical = (decltype(pl.trace_physical))trp;
    ctx->plugins.push_back(pl);
    *metric_id = PRR_METRIC_PLUGIN0 + (int)ctx->plugins.size() - 1;
    return PRR_OK;
}

prr_status prr_upload_texture(prr_ctx *ctx, int id, const uint8_t *rgba8, int w, int h)
{
    if (!ctx) return PRR_ERR_INVALID;
    if (id < 0 || id >= PRR_MAX_TEXTURES || !rgba8 || w < 2 || h < 2 || (long long)w * h > (1LL << 28)) {
        fail(ctx, "prr_upload_texture: bad id, pointer or size (need 0 <= id < PRR_MAX_TEXTURES, w,h >= 2)");
        return PRR_ERR_INVALID;
    }
    PRR_CK(ctx, cudaSetDevice(ctx->device));
    TexSlot &t = ctx->tex[id];
    size_t bytes = (size_t)w * h * 4;
    if (t.buf.ensure(bytes) != PRR_OK) { fail(ctx, "prr_upload_texture: out of device memory"); return PRR_ERR_NOMEM; }
    PRR_CK(ctx, cudaMemcpyAsync(t.buf.p, rgba8, bytes, cudaMemcpyHostToDevice, ctx->stream));
    PRR_CK(ctx, cudaStreamSynchronize(ctx->stream));
    t.w = w; t.h = h;
    return PRR_OK;
}

prr_status prr_upload_plasma(prr_ctx *ctx, const prr_plasma_desc *pd)
{
    if (!ctx) return PRR_ERR_INVALID;
    if (!pd || !pd->density || pd->nx < 2 || pd->ny < 2 || pd->nz < 2) {
        fail(ctx, "prr_upload_plasma: need a density array and nx, ny, nz >= 2");
        return PRR_ERR_INVALID;
    }
    const long long nn = (long long)pd->nx * pd->ny * pd->nz;
    if (nn > (1LL << 28)) { fail(ctx, "prr_upload_plasma: more than 2^28 nodes"); return PRR_ERR_INVALID; }
    for (int k = 0; k < 3; k++)
        if (!std::isfinite(pd->lo[k]) || !std::isfinite(pd->hi[k]) || !(pd->hi[k] > pd->lo[k])) {
            fail(ctx, "prr_upload_plasma: need finite box corners with lo < hi on every axis");
            return PRR_ERR_INVALID;
        }
    for (long long i = 0; i < nn; i++) {
        if (!(pd->density[i] >= 0.0f) || !std::isfinite(pd->density[i])) {
            fail(ctx, "prr_upload_plasma: density must be finite and >= 0 (node " + std::to_string(i) + ")");
            return PRR_ERR_INVALID;
        }
        if (pd->temperature && (!(pd->temperature[i] >= 0.0f) || !std::isfinite(pd->temperature[i]))) {
            fail(ctx, "prr_upload_plasma: temperature must be finite and >= 0 (node " + std::to_string(i) + ")");
            return PRR_ERR_INVALID;
        }
        if (pd->velocity && !(std::isfinite(pd->velocity[3 * i]) && std::isfinite(pd->velocity[3 * i + 1]) &&
                              std::isfinite(pd->velocity[3 * i + 2]))) {
            fail(ctx, "prr_upload_plasma: velocity must be finite (node " + std::to_string(i) + ")");
            return PRR_ERR_INVALID;
        }
    }
    PRR_CK(ctx, cudaSetDevice(ctx->device));
    PlasmaGrid &G = ctx->plasma;
    G.present = false;
    const size_t fb = (size_t)nn * sizeof(float);
    if (G.n.ensure(fb) != PRR_OK || (pd->temperature && G.theta.ensure(fb) != PRR_OK) ||
        (pd->velocity && G.vel.ensure((size_t)nn * sizeof(float4)) != PRR_OK)) {
        fail(ctx, "prr_upload_plasma: out of device memory");
        return PRR_ERR_NOMEM;
    }
    PRR_CK(ctx, cudaMemcpyAsync(G.n.p, pd->density, fb, cudaMemcpyHostToDevice, ctx->stream));
    if (pd->temperature) PRR_CK(ctx, cudaMemcpyAsync(G.theta.p, pd->temperature, fb, cudaMemcpyHostToDevice, ctx->stream));
    std::vector<float4> v4;
    if (pd->velocity) {  // one aligned 16-byte load per node on the device
        v4.resize((size_t)nn);
        for (long long i = 0; i < nn; i++)
            v4[i] = make_float4(pd->velocity[3 * i], pd->velocity[3 * i + 1], pd->velocity[3 * i + 2], 0.0f);
        PRR_CK(ctx, cudaMemcpyAsync(G.vel.p, v4.data(), (size_t)nn * sizeof(float4), cudaMemcpyHostToDevice, ctx->stream));
    }
    PRR_CK(ctx, cudaStreamSynchronize(ctx->stream));
    G.nx = pd->nx; G.ny = pd->ny; G.nz = pd->nz;
    for (int k = 0; k < 3; k++) { G.lo[k] = pd->lo[k]; G.hi[k] = pd->hi[k]; }
    G.has_theta = pd->temperature != nullptr;
    G.has_vel = pd->velocity != nullptr;
    G.present = true;
    return PRR_OK;
}

prr_status prr_set_schedule(prr_ctx *ctx, int schedule, const prr_launch_config *cfg)
{
    if (!ctx) return PRR_ERR_INVALID;
    if (schedule != PRR_SCHED_PLAIN && schedule != PRR_SCHED_PERSISTENT) { fail(ctx, "unknown schedule"); return PRR_ERR_INVALID; }
    if (cfg) {
        if (cfg->block_size < 32 || cfg->block_size > 256 || cfg->block_size % 32 || cfg->blocks_per_sm < 0 ||
            cfg->blocks_per_sm > 64 || cfg->compaction_interval < 1 || cfg->rays_per_thread < 1 || cfg->rays_per_thread > 2) {
            fail(ctx, "prr_set_schedule: block_size must be a multiple of 32 in [32,256], blocks_per_sm in [0,64], "
                      "compaction_interval >= 1, rays_per_thread 1 or 2");
            return PRR_ERR_INVALID;
        }
        ctx->cfg = *cfg;
    }
    ctx->schedule = schedule;
    return PRR_OK;
}

prr_status prr_get_launch_config(prr_ctx *ctx, prr_launch_config *cfg)
{
    if (!ctx || !cfg) return PRR_ERR_INVALID;
    *cfg = ctx->cfg;
    return PRR_OK;
}

prr_status prr_set_option(prr_ctx *ctx, int option, long long value)
{
    if (!ctx) return PRR_ERR_INVALID;
    switch (option) {
    case PRR_OPT_GEOD_TABLE: ctx->geod_table = value < 0 ? -1 : (value ? 1 : 0); return PRR_OK;
    case PRR_OPT_HAMILTONIAN:
        if (value < 0 || value > (PRR_HAM_FP32 | PRR_HAM_FP64)) {
            ctx->err = "PRR_OPT_HAMILTONIAN takes a mask of PRR_HAM_FP32 and PRR_HAM_FP64 (0..3)";
            return PRR_ERR_INVALID;
        }
        ctx->hamiltonian = (int)value;
        return PRR_OK;
    case PRR_OPT_WATCHDOG_CYCLES: ctx->watchdog_cycles = value > 0 ? value : 0; return PRR_OK;
    default: fail(ctx, "prr_set_option: unknown option"); return PRR_ERR_INVALID;
    }
}

prr_status prr_render(prr_ctx *ctx, const prr_frame_desc *frames, int n, uint8_t *out_rgb8, float *out_rgbf, prr_stats *stats)
{
    if (!ctx) return PRR_ERR_INVALID;
    RenderPlan plan;
    prr_status s = build_plan(ctx, frames, n, plan);
    if (s != PRR_OK) return s;
    PRR_CK(ctx, cudaSetDevice(ctx->device));
    size_t npx = (size_t)plan.total_pixels;
    if (ctx->out_u8.ensure(npx * 3) != PRR_OK || ctx->out_f.ensure(npx * 3 * sizeof(float)) != PRR_OK) {
        fail(ctx, "prr_render: out of device memory for outputs");
        return PRR_ERR_NOMEM;
    }
    s = run_plan(ctx, plan, (uint8_t *)ctx->out_u8.p, out_rgbf ? (float *)ctx->out_f.p : nullptr, ctx->stream, true);
    if (s != PRR_OK && s != PRR_ERR_TIMEOUT) return s;
    if (out_rgb8) PRR_CK(ctx, cudaMemcpyAsync(out_rgb8, ctx->out_u8.p, npx * 3, cudaMemcpyDeviceToHost, ctx->stream));
    if (out_rgbf) PRR_CK(ctx, cudaMemcpyAsync(out_rgbf, ctx->out_f.p, npx * 3 * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    PRR_CK(ctx, cudaStreamSynchronize(ctx->stream));
    prr_status s2 = collect_stats(ctx, plan, stats);
    return s != PRR_OK ? s : s2;
}

prr_status prr_render_device(prr_ctx *ctx, const prr_frame_desc *frames, int n, uint8_t *d_rgb8, float *d_rgbf, void *stream)
{
    if (!ctx) return PRR_ERR_INVALID;
    RenderPlan plan;
    prr_status s = build_plan(ctx, frames, n, plan);
    if (s != PRR_OK) return s;
    PRR_CK(ctx, cudaSetDevice(ctx->device));
    return run_plan(ctx, plan, d_rgb8, d_rgbf, stream ? (cudaStream_t)stream : (cudaStream_t)0, false);
}

prr_status prr_trace_rays(prr_ctx *ctx, const prr_frame_desc *frame, float *out_state, float *out_rgb, prr_stats *stats)
{
    if (!ctx) return PRR_ERR_INVALID;
    RenderPlan plan;
    prr_status s = build_plan(ctx, frame, 1, plan);
    if (s != PRR_OK) return s;
    PRR_CK(ctx, cudaSetDevice(ctx->device));
    s = trace_plan(ctx, plan, out_state, nullptr, out_rgb);
    if (s != PRR_OK && s != PRR_ERR_TIMEOUT) return s;
    prr_status s2 = collect_stats(ctx, plan, stats);
    return s != PRR_OK ? s : s2;
}

prr_status prr_trace_rays_f64(prr_ctx *ctx, const prr_frame_desc *frame, double *out_state, double *out_rgb, prr_stats *stats)
{
    if (!ctx) return PRR_ERR_INVALID;
    if (!frame || frame->mode != PRR_MODE_PHYSICAL) { fail(ctx, "prr_trace_rays_f64: PHYSICAL mode only"); return PRR_ERR_INVALID; }
    prr_frame_desc f = *frame;
    f.precision = PRR_PREC_FP64;
    RenderPlan plan;
    prr_status s = build_plan(ctx, &f, 1, plan);
    if (s != PRR_OK) return s;
    PRR_CK(ctx, cudaSetDevice(ctx->device));
    std::vector<float> rgb;
    if (out_rgb) rgb.resize((size_t)plan.total_rays * 3);
    s = trace_plan(ctx, plan, nullptr, out_state, out_rgb ? rgb.data() : nullptr);
    if (s != PRR_OK && s != PRR_ERR_TIMEOUT) return s;
    if (out_rgb) for (size_t i = 0; i < rgb.size(); i++) out_rgb[i] = rgb[i];
    prr_status s2 = collect_stats(ctx, plan, stats);
    return s != PRR_OK ? s : s2;
}

prr_status prr_measure_peak(prr_ctx *ctx, double *fp32_tflops, double *fp64_tflops)
{
    if (!ctx) return PRR_ERR_INVALID;
    PRR_CK(ctx, cudaSetDevice(ctx->device));
    if (ctx->scratch.ensure(4096 * sizeof(double)) != PRR_OK) return PRR_ERR_NOMEM;
    const int threads = 256, blocks = ctx->nsm * 8;
    for (int pass = 0; pass < 2; pass++) {
        double *outp = pass == 0 ? fp32_tflops : fp64_tflops;
        if (!outp) continue;
        int iters = pass == 0 ? 4096 : 1024;
        float best = 1e30f;
        for (int rep = 0; rep < 4; rep++) {
            PRR_CK(ctx, cudaEventRecord(ctx->e0, ctx->stream));
            if (pass == 0) PRR_CK(ctx, launch_fma_peak((float *)ctx->scratch.p, blocks, threads, iters, ctx->stream));
            else PRR_CK(ctx, launch_dfma_peak((double *)ctx->scratch.p, blocks, threads, iters, ctx->stream));
            PRR_CK(ctx, cudaEventRecord(ctx->e1, ctx->stream));
            PRR_CK(ctx, cudaEventSynchronize(ctx->e1));
            float ms = 0;
            PRR_CK(ctx, cudaEventElapsedTime(&ms, ctx->e0, ctx->e1));
            if (rep > 0) best = std::min(best, ms);  // first launch is warm-up
        }
        double flops = (double)blocks * threads * iters * 16.0 * 8.0 * 2.0;
        *outp = flops / (best * 1e-3) / 1e12;
    }
    return PRR_OK;
}

prr_status prr_check_recip(prr_ctx *ctx, const double *x, int n, double *out)
{
    if (!ctx) return PRR_ERR_INVALID;
    if (!x || !out || n < 1 || n > (1 << 20)) {
        ctx->err = "prr_check_recip: needs 1..2^20 inputs and an output of 4 doubles per input";
        return PRR_ERR_INVALID;
    }
    PRR_CK(ctx, cudaSetDevice(ctx->device));
    if (ctx->scratch.ensure((size_t)n * 5 * sizeof(double)) != PRR_OK) return PRR_ERR_NOMEM;
    double *d_x = (double *)ctx->scratch.p, *d_out = d_x + n;
    PRR_CK(ctx, cudaMemcpyAsync(d_x, x, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    PRR_CK(ctx, launch_check_recip(d_x, n, d_out, ctx->stream));
    PRR_CK(ctx, cudaMemcpyAsync(out, d_out, (size_t)n * 4 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    PRR_CK(ctx, cudaStreamSynchronize(ctx->stream));
    return PRR_OK;
}

}  // extern "C"
