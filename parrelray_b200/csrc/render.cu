// render.cu - frame validation, the render plan and its execution on the
// REFERENCE, PLAIN and PERSISTENT paths, ray-state readback, stats and the
// launch-shape autotuner.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "kernels.cuh"
#include "prr_internal.h"

using namespace prr;

#define PRR_CK(ctx, expr)                                                                                  \
    do {                                                                                                   \
        cudaError_t _e = (expr);                                                                           \
        if (_e != cudaSuccess) {                                                                           \
            (ctx)->err = std::string(#expr) + ": " + cudaGetErrorString(_e);                               \
            return PRR_ERR_CUDA;                                                                           \
        }                                                                                                  \
    } while (0)

namespace {

prr_status bad(prr_ctx *ctx, int f, const std::string &msg)
{
    ctx->err = "frame " + std::to_string(f) + ": " + msg;
    return PRR_ERR_INVALID;
}

bool finite_pos(float v) { return std::isfinite(v) && v > 0.0f; }

DevTex dev_tex(prr_ctx *ctx, int id)
{
    DevTex t{nullptr, 0, 0};
    if (id >= 0 && id < PRR_MAX_TEXTURES && ctx->tex[id].buf.p) {
        t.p = (const uint32_t *)ctx->tex[id].buf.p;
        t.w = ctx->tex[id].w;
        t.h = ctx->tex[id].h;
    }
    return t;
}

prr_status alloc(prr_ctx *ctx, DevBuf &b, size_t bytes, const char *what)
{
    if (b.ensure(bytes) != PRR_OK) {
        ctx->err = std::string("out of device memory for ") + what + " (" + std::to_string(bytes) + " bytes)";
        return PRR_ERR_NOMEM;
    }
    return PRR_OK;
}

// Camera::computeVectors (main/Camera.cpp:19-28) in FP32: forward, up and
// right = forward x up, each normalised as cudamaths' normalize does.
void camera_basis(float a, float b, float fwd[3], float right[3], float up[3])
{
    auto nrm = [](float v[3]) {
        float k = 1.0f / sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        v[0] = k * v[0]; v[1] = k * v[1]; v[2] = k * v[2];
    };
    fwd[0] = cosf(b) * cosf(a); fwd[1] = cosf(b) * sinf(a); fwd[2] = -sinf(b);
    nrm(fwd);
    up[0] = cosf(a) * sinf(b); up[1] = sinf(a) * sinf(b); up[2] = cosf(b);
    nrm(up);
    right[0] = fwd[1] * up[2] - fwd[2] * up[1];
    right[1] = fwd[2] * up[0] - fwd[0] * up[2];
    right[2] = fwd[0] * up[1] - fwd[1] * up[0];
    nrm(right);
}

// Validates a frame's emission block and fills its device parameters
// (prr_emission_desc in include/prr.h).
prr_status emission_params(prr_ctx *ctx, int f, const prr_frame_desc &d, EmisParams &em)
{
    memset(&em, 0, sizeof(em));
    em.kind = PRR_EMISSION_NONE;
    if (d.emission == PRR_EMISSION_NONE) return PRR_OK;
    if (d.emission != PRR_EMISSION_DISK && d.emission != PRR_EMISSION_GRID) return bad(ctx, f, "unknown emission model (none, disk, grid)");
    if (d.mode != PRR_MODE_PHYSICAL) return bad(ctx, f, "emission renders in PHYSICAL mode");
    if (d.precision != PRR_PREC_FP32 && d.precision != PRR_PREC_FP64) return bad(ctx, f, "emission renders in FP32 or FP64");
    const prr_emission_desc &e = d.emis;
    if (!(e.r_in >= 0.0f) || !(e.r_out > e.r_in) || !std::isfinite(e.r_out)) return bad(ctx, f, "emission needs 0 <= r_in < r_out (finite)");
    if (d.emission == PRR_EMISSION_DISK && (!(e.r_in > 0.0f) || !finite_pos(e.height) || !std::isfinite(e.index)))
        return bad(ctx, f, "disk emission needs r_in > 0, height > 0 and a finite index");
    if (!std::isfinite(e.spectral_index) || !std::isfinite(e.temp_power)) return bad(ctx, f, "emission exponents must be finite");
    if (!(e.absorb >= 0.0f) || !std::isfinite(e.absorb) || !(e.gain >= 0.0f) || !std::isfinite(e.gain))
        return bad(ctx, f, "emission needs finite absorb >= 0 and gain >= 0");
    if (e.sense != 1 && e.sense != -1) return bad(ctx, f, "emission sense must be +1 (co-rotating) or -1");
    if (e.colormap != PRR_CMAP_AFMHOT && e.colormap != PRR_CMAP_GREY) return bad(ctx, f, "unknown emission colour map");
    if (d.emission == PRR_EMISSION_GRID && !ctx->plasma.present) return bad(ctx, f, "grid emission needs a plasma grid (prr_upload_plasma)");
    // nu_cam is measured by a static observer at the camera: g_tt = f - 1 < 0 there
    const double M = d.metric == PRR_METRIC_FLAT ? 0.0 : d.mass, a = d.metric == PRR_METRIC_KERR ? d.spin : 0.0;
    const double x = d.cam_pos[0], y = d.cam_pos[1], z = d.cam_pos[2];
    const double b = x * x + y * y + z * z - a * a;
    const double r = std::sqrt(0.5 * (b + std::sqrt(b * b + 4.0 * a * a * z * z)));
    const double fc = M > 0.0 ? 2.0 * M * r * r * r / (r * r * r * r + a * a * z * z) : 0.0;
    if (!(fc < 1.0)) return bad(ctx, f, "emission needs the camera outside the ergoregion (a static observer there)");
    em.kind = d.emission;
    em.sense = e.sense;
    em.cmap = e.colormap;
    em.index = e.index; em.height = e.height; em.r_in = e.r_in; em.r_out = e.r_out;
    em.spectral = e.spectral_index; em.absorb = e.absorb; em.gain = e.gain; em.temp_power = e.temp_power;
    if (d.emission == PRR_EMISSION_GRID) {
        const PlasmaGrid &G = ctx->plasma;
        em.grid.n = (const float *)G.n.p;
        em.grid.theta = G.has_theta ? (const float *)G.theta.p : nullptr;
        em.grid.vel = G.has_vel ? (const float4 *)G.vel.p : nullptr;
        em.grid.nx = G.nx; em.grid.ny = G.ny; em.grid.nz = G.nz;
        const int nn[3] = {G.nx, G.ny, G.nz};
        for (int k = 0; k < 3; k++) {
            em.grid.lo[k] = G.lo[k];
            em.grid.inv[k] = (float)(nn[k] - 1) / (G.hi[k] - G.lo[k]);
        }
    }
    return PRR_OK;
}

}  // namespace

int resolve_bpsm(prr_ctx *ctx, int precision, bool emission)
{
    if (ctx->cfg.blocks_per_sm > 0) return ctx->cfg.blocks_per_sm;
    int b = persistent_occupancy(precision, ctx->geod_table == 1, ctx->cfg.block_size, ctx->cfg.rays_per_thread, emission,
                                 ctx->hamiltonian);
    return b > 0 ? b : 1;
}

prr_status build_plan(prr_ctx *ctx, const prr_frame_desc *frames, int n, RenderPlan &plan)
{
    if (!frames || n < 1 || n > (1 << 22)) { ctx->err = "need 1 <= n <= 4194304 frames and a non-null array"; return PRR_ERR_INVALID; }
    plan.fp.resize(n);
    plan.pix_begin.assign(n + 1, 0);
    plan.ray_begin.assign(n + 1, 0);
    plan.mode = frames[0].mode;
    plan.precision = frames[0].precision;
    plan.any_fxaa = false;
    plan.any_emission = false;
    plan.plugin = false;
    for (int f = 0; f < n; f++) {
        const prr_frame_desc &d = frames[f];
        FrameParams &p = plan.fp[f];
        memset(&p, 0, sizeof(p));
        if (d.mode != plan.mode || d.precision != plan.precision) return bad(ctx, f, "all frames of one call need the same mode and precision");
        if (d.width < 1 || d.height < 1 || d.width > 65536 || d.height > 65536) return bad(ctx, f, "width/height must be in [1, 65536]");
        if (d.samples < 1 || d.samples > 64) return bad(ctx, f, "samples must be in [1, 64]");
        if (d.ssaa == PRR_SSAA_NONE) {
            if (d.samples != 1) return bad(ctx, f, "SSAA none needs samples == 1");
            p.nsub = 1;
        } else if (d.ssaa == PRR_SSAA_REGULAR || d.ssaa == PRR_SSAA_JITTERED) {
            int q = (int)std::lround(std::sqrt((double)d.samples));
            if (q * q != d.samples) return bad(ctx, f, "SSAA regular/jittered needs a perfect-square sample count (kernels/ssaa.cuh:41)");
            p.nsub = q;
        } else if (d.ssaa == PRR_SSAA_RANDOM) {
            p.nsub = 1;
        } else return bad(ctx, f, "unknown SSAA distribution (none, regular, random, jittered)");
        if (d.camera < PRR_CAMERA_SPHERICAL || d.camera > PRR_CAMERA_PANORAMA) return bad(ctx, f, "unknown camera model");
        if (d.mode == PRR_MODE_REFERENCE &&
            (d.camera != PRR_CAMERA_SPHERICAL || (d.ssaa != PRR_SSAA_NONE && d.ssaa != PRR_SSAA_REGULAR)))
            return bad(ctx, f, "REFERENCE mode places rays as the reference does: spherical camera, SSAA none or regular");
        if (!finite_pos(d.vfov) || d.vfov >= 6.3f) return bad(ctx, f, "vfov must be in (0, 2*pi) radians");
        for (int k = 0; k < 3; k++) if (!std::isfinite(d.cam_pos[k])) return bad(ctx, f, "camera position is not finite");
        if (!std::isfinite(d.cam_alpha) || !std::isfinite(d.cam_beta)) return bad(ctx, f, "camera angles are not finite");
        const MetricPlugin *plugin = frame_plugin(ctx, d.metric);
        if ((d.metric < PRR_METRIC_FLAT || d.metric > PRR_METRIC_KERR) && !plugin)
            return bad(ctx, f, "unknown metric (built-in 0-2, or an id from prr_load_metric_plugin)");
        if (f == 0) plan.plugin = plugin != nullptr;
        if ((plugin != nullptr) != plan.plugin)
            return bad(ctx, f, "frames with metric plug-ins and frames with built-in metrics need separate calls");
        if (plugin && d.mode == PRR_MODE_PHYSICAL && d.precision != PRR_PREC_FP32)
            return bad(ctx, f, "metric plug-ins render PHYSICAL mode in FP32 (a header's getGeod computes in FP32)");
        if (plugin && d.emission != PRR_EMISSION_NONE) return bad(ctx, f, "metric plug-ins render without plasma emission");
        if (!std::isfinite(d.mass) || d.mass < 0.0f) return bad(ctx, f, "mass must be >= 0");
        // M = 0 is allowed for Schwarzschild: the reference renders its example deck (input/sim.params:30,52) so
        if (d.metric == PRR_METRIC_KERR && d.mass <= 0.0f) return bad(ctx, f, "Kerr needs mass > 0");
        if (d.metric == PRR_METRIC_KERR && !(std::fabs(d.spin) <= d.mass)) return bad(ctx, f, "Kerr needs |spin| <= mass");
        if (d.solver != PRR_SOLVER_EULER && d.solver != PRR_SOLVER_RKF45) return bad(ctx, f, "solver must be euler (0) or rkf45 (2)");
        if (d.mode != PRR_MODE_REFERENCE && d.mode != PRR_MODE_PHYSICAL) return bad(ctx, f, "unknown mode");
        if (d.precision < PRR_PREC_FP32 || d.precision > PRR_PREC_SPLIT) return bad(ctx, f, "unknown precision");
        if (d.mode == PRR_MODE_REFERENCE && d.precision != PRR_PREC_FP32) return bad(ctx, f, "REFERENCE mode is FP32 only");
        if (d.mode == PRR_MODE_PHYSICAL && d.solver == PRR_SOLVER_EULER) return bad(ctx, f, "PHYSICAL mode integrates with rkf45 only");
        if (!finite_pos(d.h) || !finite_pos(d.hmin) || !finite_pos(d.hmax) || d.hmin > d.hmax) return bad(ctx, f, "need 0 < hmin <= hmax and h > 0");
        if (d.mode == PRR_MODE_REFERENCE && !finite_pos(d.eps)) return bad(ctx, f, "REFERENCE mode needs eps > 0");
        if (d.mode == PRR_MODE_PHYSICAL && (!(d.rtol >= 0.0f) || !(d.atol >= 0.0f) || d.rtol + d.atol <= 0.0f)) return bad(ctx, f, "need rtol, atol >= 0, not both 0");
        if (!finite_pos(d.rout)) return bad(ctx, f, "rout must be > 0");
        if (!(d.horizon_eps >= 0.0f)) return bad(ctx, f, "horizon_eps must be >= 0");
        if (d.max_steps < 1) return bad(ctx, f, "max_steps must be >= 1");
        if (d.background_id >= PRR_MAX_TEXTURES || (d.background_id >= 0 && !ctx->tex[d.background_id].buf.p)) return bad(ctx, f, "background texture id not uploaded");
        if (d.bg_filter != PRR_BG_RMS2X2 && d.bg_filter != PRR_BG_BILINEAR) return bad(ctx, f, "unknown background filter");
        if (d.nspheres < 0 || d.nspheres > PRR_MAX_SPHERES) return bad(ctx, f, "nspheres must be in [0, PRR_MAX_SPHERES]");
        for (int s = 0; s < d.nspheres; s++) {
            const prr_sphere &S = d.spheres[s];
            if (!finite_pos(S.radius) || !std::isfinite(S.center[0]) || !std::isfinite(S.center[1]) || !std::isfinite(S.center[2]))
                return bad(ctx, f, "sphere " + std::to_string(s) + " has a bad centre or radius");
            if (S.texture_id >= PRR_MAX_TEXTURES || (S.texture_id >= 0 && !ctx->tex[S.texture_id].buf.p))
                return bad(ctx, f, "sphere " + std::to_string(s) + " texture id not uploaded");
            // a hit with any window h <= hmax needs |p - c|^2 <= ((sqrt(hmax) + R)/2)^2 + R^2
            double reach = 0.5 * (std::sqrt((double)d.hmax) + S.radius);
            float far2 = (float)((reach * reach + (double)S.radius * S.radius) * 1.01 + 1e-3);
            p.sph[s] = {S.center[0], S.center[1], S.center[2], S.radius, dev_tex(ctx, S.texture_id), far2,
                        (float)std::sqrt((double)far2)};
        }
        // the shell that holds every sphere's far radius: |p - c| >= | |p| - |c| |, so a point
        // with |p| > |c| + sqrt(far2) or |p| < |c| - sqrt(far2) is far from that sphere (the bounds
        // widened by 1e-4 relative and absolute against rounding)
        {
            double lo = INFINITY, hi = -1.0;
            for (int s = 0; s < d.nspheres; s++) {
                const DevSphere &S = p.sph[s];
                const double c = std::sqrt((double)S.cx * S.cx + (double)S.cy * S.cy + (double)S.cz * S.cz);
                const double fr = std::sqrt((double)S.far2);
                hi = std::max(hi, c + fr);
                lo = std::min(lo, c - fr);
            }
            if (d.nspheres == 0) {
                p.sph_lo2 = 1.0f; p.sph_hi2 = 0.0f;
            } else {
                hi = hi * (1.0 + 1e-4) + 1e-4;
                lo = lo * (1.0 - 1e-4) - 1e-4;
                p.sph_hi2 = (float)(hi * hi);
                p.sph_lo2 = lo > 0.0 ? (float)(lo * lo) : -1.0f;
            }
        }
        p.width = d.width; p.height = d.height; p.samples = d.samples; p.ssaa = d.ssaa;
        p.vfov = d.vfov; p.cam[0] = d.cam_pos[0]; p.cam[1] = d.cam_pos[1]; p.cam[2] = d.cam_pos[2];
        p.alpha = d.cam_alpha; p.beta = d.cam_beta;
        p.camera = d.camera;
        p.ssaa_seed = d.ssaa_seed;
        // computeVectors takes the pitch with the opposite sign from rayDir_Spherical: evaluate it at -b
        // so every model's centre ray is the spherical model's
        camera_basis(d.cam_alpha, -d.cam_beta, p.cfwd, p.cright, p.cup);
        p.tan_half = tanf(d.vfov / 2.0f);
        p.metric = d.metric; p.M = d.mass; p.a = (d.metric == PRR_METRIC_KERR || plugin) ? d.spin : 0.0f;
        p.rs = 2.0f * d.mass;  // Spacetime::setBhMass (main/Spacetime.h:23)
        float rplus = d.metric == PRR_METRIC_KERR ? kerr_r_plus<float>(d.mass, d.spin) : (d.metric == PRR_METRIC_FLAT ? 0.0f : p.rs);
        p.rstop = rplus + d.horizon_eps;
        p.rblack = rplus * 1.01f;
        p.solver = d.solver; p.mode = d.mode; p.precision = d.precision;
        p.h = d.h; p.hmin = d.hmin; p.hmax = d.hmax; p.eps = d.eps; p.rtol = d.rtol; p.atol = d.atol; p.rout = d.rout;
        p.max_steps = d.max_steps;
        p.bg_filter = d.bg_filter; p.fxaa = d.fxaa ? 1 : 0;
        p.bg = dev_tex(ctx, d.background_id);
        p.fp64_delta = d.precision == PRR_PREC_SPLIT ? d.fp64_delta : 0.0f;
        p.fp64_rfac = d.precision == PRR_PREC_SPLIT ? d.fp64_rfac : 0.0f;
        p.nspheres = d.nspheres;
        prr_status es = emission_params(ctx, f, d, p.em);
        if (es != PRR_OK) return es;
        if (p.em.kind != PRR_EMISSION_NONE) plan.any_emission = true;
        long long npx = (long long)d.width * d.height;
        p.pix_begin = plan.pix_begin[f];
        p.ray_begin = plan.ray_begin[f];
        plan.pix_begin[f + 1] = plan.pix_begin[f] + npx;
        plan.ray_begin[f + 1] = plan.ray_begin[f] + npx * d.samples;
        if (d.fxaa) plan.any_fxaa = true;
    }
    plan.total_pixels = plan.pix_begin[n];
    plan.total_rays = plan.ray_begin[n];
    if (plan.total_rays > (1LL << 38)) { ctx->err = "too many rays in one call"; return PRR_ERR_INVALID; }
    return PRR_OK;
}

static prr_status upload_plan(prr_ctx *ctx, const RenderPlan &plan, cudaStream_t st)
{
    size_t n = plan.fp.size();
    prr_status s;
    if ((s = alloc(ctx, ctx->frames, n * sizeof(FrameParams), "frame parameters")) != PRR_OK) return s;
    if ((s = alloc(ctx, ctx->frame_begin, (n + 1) * sizeof(long long), "frame table")) != PRR_OK) return s;
    if ((s = alloc(ctx, ctx->counters, C_COUNT * sizeof(unsigned long long), "counters")) != PRR_OK) return s;
    PRR_CK(ctx, cudaMemcpyAsync(ctx->frames.p, plan.fp.data(), n * sizeof(FrameParams), cudaMemcpyHostToDevice, st));
    PRR_CK(ctx, cudaMemcpyAsync(ctx->frame_begin.p, plan.pix_begin.data(), (n + 1) * sizeof(long long), cudaMemcpyHostToDevice, st));
    PRR_CK(ctx, cudaMemsetAsync(ctx->counters.p, 0, C_COUNT * sizeof(unsigned long long), st));
    // the host vectors may be freed when the caller returns: make the copies complete first
    PRR_CK(ctx, cudaStreamSynchronize(st));
    return PRR_OK;
}

static PersistentArgs persistent_args(prr_ctx *ctx, const RenderPlan &plan)
{
    PersistentArgs a;
    memset(&a, 0, sizeof(a));
    a.frames = (const FrameParams *)ctx->frames.p;
    a.frame_pix_begin = (const long long *)ctx->frame_begin.p;
    a.nframes = (int)plan.fp.size();
    a.total_pixels = plan.total_pixels;
    a.counters = (unsigned long long *)ctx->counters.p;
    a.geod_table = ctx->geod_table == 1;
    a.hamiltonian = ctx->hamiltonian;
    a.compaction_interval = ctx->cfg.compaction_interval;
    a.watchdog_cycles = ctx->watchdog_cycles;
    a.rays_per_thread = ctx->cfg.rays_per_thread;
    a.ray_steps = ctx->ray_steps_out;
    a.emission = plan.any_emission;
    return a;
}

// Emission runs on the persistent kernels with the register contraction.
static prr_status check_emission_schedule(prr_ctx *ctx, const RenderPlan &plan)
{
    if (!plan.any_emission) return PRR_OK;
    if (ctx->schedule == PRR_SCHED_PLAIN || ctx->geod_table == 1) {
        ctx->err = "emission renders on the persistent schedule with the register contraction";
        return PRR_ERR_UNSUPPORTED;
    }
    return PRR_OK;
}

prr_status run_plan(prr_ctx *ctx, const RenderPlan &plan, uint8_t *d_rgb8, float *d_rgbf, cudaStream_t st, bool timed)
{
    prr_status s = check_emission_schedule(ctx, plan);
    if (s != PRR_OK) return s;
    s = upload_plan(ctx, plan, st);
    if (s != PRR_OK) return s;
    const int n = (int)plan.fp.size();
    unsigned long long *counters = (unsigned long long *)ctx->counters.p;
    int launches = 0;
    if ((s = alloc(ctx, ctx->image, (size_t)plan.total_pixels * 3 * sizeof(float), "image")) != PRR_OK) return s;
    float *image = (float *)ctx->image.p;
    if (timed) PRR_CK(ctx, cudaEventRecord(ctx->e0, st));
    const FrameParams *d_fp = (const FrameParams *)ctx->frames.p;

    auto finish = [&](int f, bool direct_done) -> prr_status {
        const FrameParams &p = plan.fp[f];
        float *img = image + 3 * p.pix_begin;
        float *of = d_rgbf ? d_rgbf + 3 * p.pix_begin : nullptr;
        uint8_t *o8 = d_rgb8 ? d_rgb8 + 3 * p.pix_begin : nullptr;
        if (p.fxaa || !direct_done) {
            PRR_CK(ctx, launch_finish(img, p.width, p.height, p.fxaa, of, o8, st));
            launches++;
        } else if (of) {
            PRR_CK(ctx, cudaMemcpyAsync(of, img, (size_t)p.width * p.height * 3 * sizeof(float), cudaMemcpyDeviceToDevice, st));
        }
        return PRR_OK;
    };

    bool trace_timed = false;
    if (plan.mode == PRR_MODE_REFERENCE || ctx->schedule == PRR_SCHED_PLAIN || plan.plugin) {
        long long max_rays = 0;
        for (const auto &p : plan.fp) max_rays = std::max(max_rays, (long long)p.width * p.height * p.samples);
        if ((s = alloc(ctx, ctx->sample_rgb, (size_t)max_rays * 3 * sizeof(float), "per-sample colours")) != PRR_OK) return s;
        if (plan.mode != PRR_MODE_REFERENCE &&
            (s = alloc(ctx, ctx->rays, (size_t)max_rays * plain_ray_record_bytes(), "ray records")) != PRR_OK) return s;
        float *rgb = (float *)ctx->sample_rgb.p;
        for (int f = 0; f < n; f++) {
            const FrameParams &p = plan.fp[f];
            long long nr = (long long)p.width * p.height * p.samples;
            if (const MetricPlugin *pl = frame_plugin(ctx, p.metric)) {
                if ((s = alloc(ctx, ctx->rays, (size_t)nr * pl->ray_bytes, "plug-in ray records")) != PRR_OK) return s;
                auto tr = p.mode == PRR_MODE_PHYSICAL ? pl->trace_physical : pl->trace;
                PRR_CK(ctx, (cudaError_t)tr(&p, d_fp, f, nr, ctx->rays.p, nullptr, rgb, counters, st));
                launches += 3;
            } else if (plan.mode == PRR_MODE_REFERENCE) {
                PRR_CK(ctx, launch_ref_trace(d_fp, f, nr, nullptr, rgb, counters, st));
                launches++;
            } else {
                PlainBuffers b{ctx->rays.p, rgb};
                PRR_CK(ctx, launch_plain_frame(d_fp, p, f, b, counters, ctx->geod_table != 0, st, &launches));
            }
            PRR_CK(ctx, launch_combine(rgb, p.width, p.height, p.samples, image + 3 * p.pix_begin, st));
            launches++;
            if ((s = finish(f, false)) != PRR_OK) return s;
        }
    } else {
        trace_timed = timed;
        PersistentArgs a = persistent_args(ctx, plan);
        a.image = image;
        const int bpsm = resolve_bpsm(ctx, plan.precision, plan.any_emission);
        if (plan.precision == PRR_PREC_SPLIT) {
            if ((s = alloc(ctx, ctx->sample_rgb, (size_t)plan.total_rays * 3 * sizeof(float), "per-sample colours")) != PRR_OK) return s;
            if ((s = alloc(ctx, ctx->queue, (size_t)plan.total_rays * sizeof(unsigned long long), "FP64 queue")) != PRR_OK) return s;
            a.sample_rgb = (float *)ctx->sample_rgb.p;
            a.fp64_queue = (unsigned long long *)ctx->queue.p;
            a.fp64_capacity = plan.total_rays;
            if (timed) PRR_CK(ctx, cudaEventRecord(ctx->t0, st));
            PRR_CK(ctx, launch_persistent(a, PRR_PREC_SPLIT, ctx->cfg.block_size, bpsm, ctx->nsm, st));
            PRR_CK(ctx, launch_fp64_requeue(a, 128, ctx->nsm, st));
            if (timed) PRR_CK(ctx, cudaEventRecord(ctx->t1, st));
            launches += 2;
            for (int f = 0; f < n; f++) {
                const FrameParams &p = plan.fp[f];
                PRR_CK(ctx, launch_combine(a.sample_rgb + 3 * p.ray_begin, p.width, p.height, p.samples, image + 3 * p.pix_begin, st));
                launches++;
                if ((s = finish(f, false)) != PRR_OK) return s;
            }
        } else {
            a.rgb8 = d_rgb8;
            if (timed) PRR_CK(ctx, cudaEventRecord(ctx->t0, st));
            PRR_CK(ctx, launch_persistent(a, plan.precision, ctx->cfg.block_size, bpsm, ctx->nsm, st));
            if (timed) PRR_CK(ctx, cudaEventRecord(ctx->t1, st));
            launches++;
            for (int f = 0; f < n; f++)
                if ((s = finish(f, true)) != PRR_OK) return s;
        }
    }
    if (timed) {
        PRR_CK(ctx, cudaEventRecord(ctx->e1, st));
        PRR_CK(ctx, cudaEventSynchronize(ctx->e1));
        PRR_CK(ctx, cudaEventElapsedTime(&ctx->last_ms, ctx->e0, ctx->e1));
        ctx->last_trace_ms = ctx->last_ms;
        if (trace_timed) PRR_CK(ctx, cudaEventElapsedTime(&ctx->last_trace_ms, ctx->t0, ctx->t1));
    }
    ctx->last_launches = launches;
    if (ctx->watchdog_cycles > 0) {
        unsigned long long flag = 0;
        PRR_CK(ctx, cudaMemcpyAsync(&flag, counters + C_TIMEOUT, sizeof(flag), cudaMemcpyDeviceToHost, st));
        PRR_CK(ctx, cudaStreamSynchronize(st));
        if (flag) { ctx->err = "device watchdog expired: some rays were not finished"; return PRR_ERR_TIMEOUT; }
    }
    return PRR_OK;
}

prr_status trace_plan(prr_ctx *ctx, const RenderPlan &plan, float *h_state, double *h_state64, float *h_rgb)
{
    cudaStream_t st = ctx->stream;
    prr_status s = check_emission_schedule(ctx, plan);
    if (s != PRR_OK) return s;
    s = upload_plan(ctx, plan, st);
    if (s != PRR_OK) return s;
    const FrameParams &p = plan.fp[0];
    const long long nr = (long long)p.width * p.height * p.samples;
    unsigned long long *counters = (unsigned long long *)ctx->counters.p;
    const FrameParams *d_fp = (const FrameParams *)ctx->frames.p;
    size_t state_bytes = (size_t)nr * 12 * (h_state64 ? sizeof(double) : sizeof(float));
    if ((s = alloc(ctx, ctx->state, state_bytes, "ray states")) != PRR_OK) return s;
    if ((s = alloc(ctx, ctx->sample_rgb, (size_t)nr * 3 * sizeof(float), "per-sample colours")) != PRR_OK) return s;
    float *rgb = (float *)ctx->sample_rgb.p;
    PRR_CK(ctx, cudaEventRecord(ctx->e0, st));
    if (const MetricPlugin *pl = frame_plugin(ctx, p.metric)) {
        if ((s = alloc(ctx, ctx->rays, (size_t)nr * pl->ray_bytes, "plug-in ray records")) != PRR_OK) return s;
        if (h_state64) { ctx->err = "prr_trace_rays_f64: metric plug-ins trace in FP32"; return PRR_ERR_UNSUPPORTED; }
        auto tr = p.mode == PRR_MODE_PHYSICAL ? pl->trace_physical : pl->trace;
        PRR_CK(ctx, (cudaError_t)tr(&p, d_fp, 0, nr, ctx->rays.p, (float *)ctx->state.p, rgb, counters, st));
        ctx->last_launches = 3;
    } else if (plan.mode == PRR_MODE_REFERENCE) {
        PRR_CK(ctx, launch_ref_trace(d_fp, 0, nr, (float *)ctx->state.p, rgb, counters, st));
        ctx->last_launches = 1;
    } else if (ctx->schedule == PRR_SCHED_PLAIN && !h_state64) {
        if ((s = alloc(ctx, ctx->rays, (size_t)nr * plain_ray_record_bytes(), "ray records")) != PRR_OK) return s;
        PlainBuffers b{ctx->rays.p, rgb};
        int launches = 0;
        PRR_CK(ctx, launch_plain_frame(d_fp, p, 0, b, counters, ctx->geod_table != 0, st, &launches));
        ctx->last_launches = launches;
    } else {
        if ((s = alloc(ctx, ctx->image, (size_t)plan.total_pixels * 3 * sizeof(float), "image")) != PRR_OK) return s;
        PersistentArgs a = persistent_args(ctx, plan);
        a.image = (float *)ctx->image.p;
        a.sample_rgb = rgb;
        if (h_state64) a.ray_state64 = (double *)ctx->state.p;
        else a.ray_state = (float *)ctx->state.p;
        int prec = plan.precision == PRR_PREC_FP64 ? PRR_PREC_FP64 : PRR_PREC_FP32;
        PRR_CK(ctx, launch_persistent(a, prec, ctx->cfg.block_size, resolve_bpsm(ctx, prec, plan.any_emission), ctx->nsm, st));
        ctx->last_launches = 1;
    }
    PRR_CK(ctx, cudaEventRecord(ctx->e1, st));
    PRR_CK(ctx, cudaEventSynchronize(ctx->e1));
    PRR_CK(ctx, cudaEventElapsedTime(&ctx->last_ms, ctx->e0, ctx->e1));
    ctx->last_trace_ms = ctx->last_ms;
    if (plan.mode != PRR_MODE_REFERENCE && ctx->schedule == PRR_SCHED_PLAIN && !h_state64) {
        // ray records (48 B, main/base.h:172-176 layout) -> 12-float states
        std::vector<float> rec((size_t)nr * 12);
        PRR_CK(ctx, cudaMemcpy(rec.data(), ctx->rays.p, (size_t)nr * 48, cudaMemcpyDeviceToHost));
        if (h_state)
            for (long long i = 0; i < nr; i++) {
                const float *r = rec.data() + 12 * i;
                float *o = h_state + 12 * i;
                int res;
                memcpy(&res, r + 2, sizeof(int));
                o[0] = r[0]; o[1] = r[1]; o[2] = (float)res;
                for (int k = 0; k < 8; k++) o[3 + k] = r[3 + k];
                o[11] = r[11];
            }
    } else if (h_state) {
        PRR_CK(ctx, cudaMemcpy(h_state, ctx->state.p, (size_t)nr * 12 * sizeof(float), cudaMemcpyDeviceToHost));
    } else if (h_state64) {
        PRR_CK(ctx, cudaMemcpy(h_state64, ctx->state.p, (size_t)nr * 12 * sizeof(double), cudaMemcpyDeviceToHost));
    }
    if (h_rgb) PRR_CK(ctx, cudaMemcpy(h_rgb, rgb, (size_t)nr * 3 * sizeof(float), cudaMemcpyDeviceToHost));
    return PRR_OK;
}

prr_status collect_stats(prr_ctx *ctx, const RenderPlan &plan, prr_stats *stats)
{
    if (!stats) return PRR_OK;
    unsigned long long c[C_COUNT];
    PRR_CK(ctx, cudaMemcpy(c, ctx->counters.p, sizeof(c), cudaMemcpyDeviceToHost));
    memset(stats, 0, sizeof(*stats));
    stats->rays = plan.total_rays;
    stats->attempts = (int64_t)c[C_ATTEMPTS];
    stats->accepted = (int64_t)c[C_ACCEPTED];
    stats->n_escaped = (int64_t)c[C_ESCAPED];
    stats->n_captured = (int64_t)c[C_CAPTURED];
    stats->n_intersection = (int64_t)c[C_INTERSECTION];
    stats->n_infinite = (int64_t)c[C_INFINITE];
    stats->n_math_error = (int64_t)c[C_MATH_ERROR];
    stats->n_fp64 = (int64_t)c[C_FP64];
    stats->kernel_ms = ctx->last_ms;
    stats->kernel_launches = ctx->last_launches;
    stats->trace_ms = ctx->last_trace_ms;
    return PRR_OK;
}

extern "C" prr_status prr_autotune(prr_ctx *ctx, const prr_frame_desc *frame, prr_launch_config *best)
{
    if (!ctx || !frame) return PRR_ERR_INVALID;
    if (frame->mode != PRR_MODE_PHYSICAL) { ctx->err = "prr_autotune: PHYSICAL mode frames only"; return PRR_ERR_INVALID; }
    RenderPlan plan;
    prr_status s = build_plan(ctx, frame, 1, plan);
    if (s != PRR_OK) return s;
    PRR_CK(ctx, cudaSetDevice(ctx->device));
    const prr_launch_config saved = ctx->cfg;
    const int saved_sched = ctx->schedule;
    ctx->schedule = PRR_SCHED_PERSISTENT;
    prr_launch_config winner = saved;
    float best_ms = 1e30f;
    // candidates: CTA size x refill interval x pixel slots per thread, each at the
    // occupancy limit of its kernel; every candidate is timed three times (minimum kept),
    // except that one more than 10 % slower than the best so far on its first run stops there
    const int blocks[3] = {64, 128, 256};
    const int intervals[4] = {8, 16, 32, 64};
    // two pixel slots per thread only where the kernel has them (FP32, register contraction)
    const int nrpt = (plan.precision == PRR_PREC_FP32 && ctx->geod_table != 1 && !plan.any_emission) ? 2 : 1;
    for (int rpt = 1; rpt <= nrpt; rpt++)
        for (int bi = 0; bi < 3; bi++) {
            const int occ = persistent_occupancy(plan.precision, ctx->geod_table == 1, blocks[bi], rpt, plan.any_emission,
                                                 ctx->hamiltonian);
            if (occ < 1) continue;
            for (int ii = 0; ii < 4; ii++) {
                ctx->cfg.block_size = blocks[bi];
                ctx->cfg.blocks_per_sm = occ;
                ctx->cfg.compaction_interval = intervals[ii];
                ctx->cfg.rays_per_thread = rpt;
                float ms = 1e30f;
                for (int rep = 0; rep < 3; rep++) {
                    s = run_plan(ctx, plan, nullptr, nullptr, ctx->stream, true);
                    if (s != PRR_OK) { ctx->cfg = saved; ctx->schedule = saved_sched; return s; }
                    ms = std::min(ms, ctx->last_ms);
                    if (rep == 0 && ms > 1.1f * best_ms) break;
                }
                if (ms < best_ms) { best_ms = ms; winner = ctx->cfg; }
            }
        }
    ctx->cfg = winner;
    ctx->schedule = saved_sched;
    if (best) *best = winner;
    return PRR_OK;
}

// Discrete adjoint of one PHYSICAL frame.  The forward image is rendered in
// FP64 first (its combined colours feed the SSAA-combine derivative), then
// k_adjoint pulls dL/d(image) back to the five parameters.
extern "C" prr_status prr_adjoint(prr_ctx *ctx, const prr_frame_desc *frame, const float *dL_dimage, int sphere_index,
                                  double grads[5], prr_stats *stats)
{
    if (!ctx) return PRR_ERR_INVALID;
    if (!frame || !dL_dimage || !grads) { ctx->err = "prr_adjoint: null frame, gradient or output"; return PRR_ERR_INVALID; }
    const prr_frame_desc &d = *frame;
    if (d.mode != PRR_MODE_PHYSICAL || d.solver != PRR_SOLVER_RKF45) { ctx->err = "prr_adjoint: PHYSICAL mode RKF45 frames only"; return PRR_ERR_INVALID; }
    if (d.fxaa) { ctx->err = "prr_adjoint: FXAA is not differentiated; render the frame without FXAA"; return PRR_ERR_UNSUPPORTED; }
    if (sphere_index < -1 || sphere_index >= d.nspheres) { ctx->err = "prr_adjoint: sphere_index out of range"; return PRR_ERR_INVALID; }
    if (d.camera != PRR_CAMERA_SPHERICAL) { ctx->err = "prr_adjoint: differentiates the spherical camera model only"; return PRR_ERR_UNSUPPORTED; }
    if (d.emission != PRR_EMISSION_NONE) { ctx->err = "prr_adjoint: differentiates frames without plasma emission only"; return PRR_ERR_UNSUPPORTED; }
    // orbit camera: position (r sin i, 0, r cos i), yaw pi, pitch i - pi/2
    double px = d.cam_pos[0], py = d.cam_pos[1], pz = d.cam_pos[2];
    double r = std::sqrt(px * px + py * py + pz * pz);
    if (!(r > 0.0)) { ctx->err = "prr_adjoint: camera at the origin"; return PRR_ERR_INVALID; }
    double incl = std::acos(pz / r);
    if (std::fabs(py) > 1e-6 * r || px < 0.0 || std::fabs(d.cam_alpha - M_PI) > 1e-5 || std::fabs(d.cam_beta - (incl - 0.5 * M_PI)) > 1e-5) {
        ctx->err = "prr_adjoint: needs an orbit camera (position (r sin i, 0, r cos i), yaw pi, pitch i - pi/2)";
        return PRR_ERR_INVALID;
    }
    // forward steps in FP32 for FP32 frames, FP64 otherwise (SPLIT included); the adjoint is FP64
    const int prec = d.precision == PRR_PREC_FP32 ? PRR_PREC_FP32 : PRR_PREC_FP64;
    prr_frame_desc f64 = d;
    f64.precision = prec;
    RenderPlan plan;
    prr_status s = build_plan(ctx, &f64, 1, plan);
    if (s != PRR_OK) return s;
    PRR_CK(ctx, cudaSetDevice(ctx->device));
    const FrameParams &fp = plan.fp[0];
    const long long npx = (long long)fp.width * fp.height, nrays = npx * fp.samples;
    // per-ray step counts of the forward render order the adjoint's rays (longest first)
    const size_t nr4 = ((size_t)nrays * sizeof(int) + 255) / 256 * 256;
    if ((s = alloc(ctx, ctx->adj_sort, 2 * nr4 + adjoint_order_bytes(nrays), "adjoint ray order")) != PRR_OK) return s;
    int *d_steps = (int *)ctx->adj_sort.p;
    unsigned *d_order = (unsigned *)((char *)ctx->adj_sort.p + nr4);
    void *d_sort_scratch = (char *)ctx->adj_sort.p + 2 * nr4;
    const int saved_sched = ctx->schedule;
    ctx->schedule = PRR_SCHED_PERSISTENT;
    ctx->ray_steps_out = d_steps;
    s = run_plan(ctx, plan, nullptr, nullptr, ctx->stream, true);
    ctx->ray_steps_out = nullptr;
    ctx->schedule = saved_sched;
    if (s != PRR_OK) return s;
    const float forward_ms = ctx->last_ms;
    AdjointParamsHost ap{};
    ap.spin = fp.a; ap.mass = fp.M; ap.incl = incl; ap.cam_r = r; ap.sphere = sphere_index;
    if (sphere_index >= 0) {
        const prr_sphere &S = d.spheres[sphere_index];
        ap.sph_R = std::hypot((double)S.center[0], (double)S.center[1]);
        ap.phase = std::atan2((double)S.center[1], (double)S.center[0]);
        ap.sph_z = S.center[2];
    }
    const int threads = ctx->nsm * adjoint_blocks_per_sm(prec) * 128;  // one resident wave
    const int max_ckpt = d.max_steps / ADJ_CHECKPOINT_INTERVAL + 2;
    if ((s = alloc(ctx, ctx->adj_ckpt, (size_t)threads * max_ckpt * adjoint_checkpoint_bytes(prec), "adjoint checkpoints")) != PRR_OK) return s;
    if ((s = alloc(ctx, ctx->adj_dl, (size_t)npx * 3 * sizeof(float) + 8 * sizeof(double), "adjoint inputs")) != PRR_OK) return s;
    float *d_dl = (float *)ctx->adj_dl.p;
    double *d_grad = (double *)((char *)ctx->adj_dl.p + ((size_t)npx * 3 * sizeof(float) + 7) / 8 * 8);
    cudaStream_t st = ctx->stream;
    PRR_CK(ctx, cudaMemcpyAsync(d_dl, dL_dimage, (size_t)npx * 3 * sizeof(float), cudaMemcpyHostToDevice, st));
    PRR_CK(ctx, cudaMemsetAsync(d_grad, 0, 5 * sizeof(double), st));
    PRR_CK(ctx, cudaMemsetAsync(ctx->counters.p, 0, C_COUNT * sizeof(unsigned long long), st));
    PRR_CK(ctx, cudaEventRecord(ctx->e0, st));
    PRR_CK(ctx, launch_adjoint_order(d_steps, nrays, d_order, d_sort_scratch, st));
    PRR_CK(ctx, launch_adjoint((const FrameParams *)ctx->frames.p, ap, d_dl, (const float *)ctx->image.p, ctx->adj_ckpt.p,
                               max_ckpt, threads, d_grad, (unsigned long long *)ctx->counters.p, nrays, d_order, prec, st));
    PRR_CK(ctx, cudaEventRecord(ctx->e1, st));
    PRR_CK(ctx, cudaMemcpyAsync(grads, d_grad, 5 * sizeof(double), cudaMemcpyDeviceToHost, st));
    PRR_CK(ctx, cudaStreamSynchronize(st));
    float adj_ms = 0.f;
    PRR_CK(ctx, cudaEventElapsedTime(&adj_ms, ctx->e0, ctx->e1));
    if (stats) {
        unsigned long long c[C_COUNT];
        PRR_CK(ctx, cudaMemcpy(c, ctx->counters.p, sizeof(c), cudaMemcpyDeviceToHost));
        memset(stats, 0, sizeof(*stats));
        stats->rays = nrays;
        stats->accepted = (int64_t)c[C_ACCEPTED];
        stats->n_math_error = (int64_t)c[C_MATH_ERROR];  // rays dropped: checkpoints did not fit, or a recomputation disagreed
        stats->kernel_ms = adj_ms;
        stats->trace_ms = forward_ms;
        stats->kernel_launches = ctx->last_launches + 2;  // + the ray-order iota and the adjoint (the radix sort's own kernels not counted)
    }
    return PRR_OK;
}
