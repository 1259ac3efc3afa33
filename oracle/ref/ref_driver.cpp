// CPU oracle driver around the reference ParRelRay sources (test
// infrastructure only: used by tests/, the golden-fixture script and the
// bench's CPU-baseline leg; never by the product).
//
// This translation unit is compiled by oracle/ref/build_ref.sh together with
// a patched copy of the reference sources (see that script for the exact,
// minimal patches).  It supplies the three definitions the shipped reference
// lacks (the lowercase `ray`/`tracer` names, `fx`, and `frames`), emulates
// kernel launches on the host with OpenMP, and exposes a small C ABI so
// Python tests can run the reference's own frame pipeline:
//     createRays_none/regular -> initRays -> trace_RKF/trace_Euler (64-row
//     layers) -> rayToRGB -> combineSamples [-> fxaa]
// exactly as prr.cpp:renderframe (prr.cpp:237-341) sequences them, with a
// snapshot of every ray's state between tracing and colouring.
#include "main/base.h"
typedef Ray ray;        // kernels/ssaa.cuh:36, metrics/*.cuh use the lowercase names
typedef Tracer tracer;  // kernels/solver.cuh:68, metrics/*.cuh

// The RKF45 position derivative dx/dlambda = u; called by kernels/solver.cuh:163-168
// but defined nowhere in the reference.
__device__ inline f4 fx(f4 x, f4 u) { (void)x; return u; }

int frames;  // assigned by prr.cpp:354 but never declared there

#include <omp.h>
#include <chrono>

thread_local uint3 blockIdx;
thread_local uint3 threadIdx;
thread_local dim3 blockDim;
thread_local dim3 gridDim;

static int g_threads = 1;

// Emulated <<<grid, block>>> launch: every block is one OpenMP work item,
// threads of a block run sequentially (the reference kernels never
// synchronise within a block).
template <class F>
static void prr_ref_launch(dim3 grid, dim3 block, F f)
{
    const long nb = (long)grid.x * grid.y * grid.z;
#pragma omp parallel for schedule(dynamic, 1) num_threads(g_threads)
    for (long b = 0; b < nb; ++b) {
        gridDim = grid;
        blockDim = block;
        blockIdx.x = (unsigned)(b % grid.x);
        blockIdx.y = (unsigned)((b / grid.x) % grid.y);
        blockIdx.z = (unsigned)(b / ((long)grid.x * grid.y));
        for (unsigned tz = 0; tz < block.z; ++tz)
            for (unsigned ty = 0; ty < block.y; ++ty)
                for (unsigned tx = 0; tx < block.x; ++tx) {
                    threadIdx.x = tx; threadIdx.y = ty; threadIdx.z = tz;
                    f();
                }
    }
}

#define main prr_ref_main
#include "prr.cpp"
#undef main

static bool g_loaded = false;
static Ray *g_rays = nullptr;
static size_t g_nrays = 0;

extern "C" {

// Reads a deck exactly like prr.cpp:main/init (prr.cpp:203-227, 359-365):
// sim deck, then its traj and scene decks, counts frames, builds the scene,
// loads the background texture(s).  Returns the frame count (<=0 on error).
int prr_ref_load(const char *deck_path)
{
    Parameters::get().parameters.clear();
    trace = Tracer();
    spacetime = Spacetime();
    camera = Camera();
    int nf = init(deck_path);
    if (nf <= 0) return nf;
    std::string bpath1 = par("tracer", "bimage1");
    std::string bpath2 = par("tracer", "bimage2");
    if (bpath1 != "") trace.sph1.tex.load(bpath1);
    if (bpath2 != "") trace.sph2.tex.load(bpath2);
    i2 res = camera.getRes();
    size_t n = (size_t)res.x * res.y * camera.getAAsamples();
    free(g_rays);
    g_rays = (Ray *)calloc(n ? n : 1, sizeof(Ray));
    g_nrays = n;
    g_loaded = true;
    frames = nf;
    return nf;
}

void prr_ref_info(int *width, int *height, int *samples)
{
    i2 res = camera.getRes();
    *width = res.x; *height = res.y; *samples = camera.getAAsamples();
}

// One frame of the reference pipeline.  Outputs (any may be NULL):
//   state  [nrays*11]: uv.x uv.y result r.x r.y r.z r.w u.x u.y u.z u.w
//                      after tracing, before rayToRGB;
//   rgb    [nrays*3]  : u.xyz after rayToRGB (the per-sample colour);
//   image  [W*H*3]    : combineSamples output (what tex2d::save quantises);
//   fxaa_im[W*H*3]    : ssaa.cuh:fxaa applied to `image` (never called by
//                       the reference frame loop; rows/cols the kernel does
//                       not write are left at 0).
// rows_stride > 1 traces only every rows_stride-th image row (a bounded
// sample used by the CPU-baseline timing); untraced rays keep their
// initialised state.  Returns the tracing wall time in seconds.
double prr_ref_frame(int frame, int nthreads, int rows_stride,
                     float *state, float *rgb, float *image, float *fxaa_im)
{
    if (!g_loaded) return -1.0;
    g_threads = nthreads > 0 ? nthreads : 1;
    if (rows_stride < 1) rows_stride = 1;
    Ray *rays = g_rays;
    i2 res = camera.getRes();
    int samples = camera.getAAsamples();
    std::string header = "frame" + to_string(frame);

    // prr.cpp:245-253 (with SPHERICAL, 250-252 too)
    camera.pos = f3(parf(header, "x"), parf(header, "y"), parf(header, "z"));
    camera.a = parf(header, "a") * M_PI / 180.0f;
    camera.b = parf(header, "b") * M_PI / 180.0f;
    camera.computeVectors();
    spacetime.updateScene(frame);
#ifdef SPHERICAL
    camera.spos = pos_cartTOspher(camera.pos);
#endif
    spacetime.setBhMass(parf(header, "mass", spacetime.getBhMass()));

    // prr.cpp:258-276
    dim3 blocks(res.x / 8 + 1, res.y / 8 + 1);
    dim3 threads(8, 8);
    switch (camera.getSSAADistr()) {
    case SSAA_DISTR::NONE: prr_ref_launch(blocks, threads, [&] { createRays_none(rays, res); }); break;
    case SSAA_DISTR::REGULAR: prr_ref_launch(blocks, threads, [&] { createRays_regular(rays, res, samples); }); break;
    default: break;
    }
    // prr.cpp:279-285
    blocks = dim3(samples * res.x / 8 + 1, res.y / 8 + 1);
    prr_ref_launch(blocks, threads, [&] { initRays(rays, camera, spacetime, samples); });

    // prr.cpp:289-309 (64-row layers), or a strided row sample through the
    // same kernels with one-row layers.
    auto t0 = std::chrono::steady_clock::now();
    if (rows_stride == 1) {
        int nlines = 64;
        int nlayers = (int)ceil((double)res.y / nlines);
        blocks = dim3(samples * res.x / 8 + 1, nlines / 8 + 1);
        for (int l = 0; l < nlayers; l++) {
            if (trace.solver == SOLVER::EULER)
                prr_ref_launch(blocks, threads, [&] { trace_Euler(rays, camera, spacetime, trace, l, nlines, samples); });
            else if (trace.solver == SOLVER::RUNGE_KUTTA_FEHLBERG)
                prr_ref_launch(blocks, threads, [&] { trace_RKF(rays, camera, spacetime, trace, l, nlines, samples); });
        }
    } else {
        blocks = dim3(samples * res.x / 8 + 1, 1);
        dim3 row_threads(8, 1);
        for (int row = 0; row < res.y; row += rows_stride) {
            if (trace.solver == SOLVER::EULER)
                prr_ref_launch(blocks, row_threads, [&] { trace_Euler(rays, camera, spacetime, trace, row, 1, samples); });
            else if (trace.solver == SOLVER::RUNGE_KUTTA_FEHLBERG)
                prr_ref_launch(blocks, row_threads, [&] { trace_RKF(rays, camera, spacetime, trace, row, 1, samples); });
        }
    }
    double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();

    size_t n = (size_t)res.x * res.y * samples;
    if (state) {
        for (size_t i = 0; i < n; i++) {
            const Ray &R = rays[i];
            float *s = state + 11 * i;
            s[0] = R.uv.x; s[1] = R.uv.y; s[2] = (float)(int)R.result;
            s[3] = R.r.x; s[4] = R.r.y; s[5] = R.r.z; s[6] = R.r.w;
            s[7] = R.u.x; s[8] = R.u.y; s[9] = R.u.z; s[10] = R.u.w;
        }
    }
    // prr.cpp:316-332
    blocks = dim3(samples * res.x / 8 + 1, res.y / 8 + 1);
    prr_ref_launch(blocks, threads, [&] { rayToRGB(rays, camera, spacetime, trace, samples); });
    if (rgb) {
        for (size_t i = 0; i < n; i++) {
            rgb[3 * i] = rays[i].u.x; rgb[3 * i + 1] = rays[i].u.y; rgb[3 * i + 2] = rays[i].u.z;
        }
    }
    tex2d im(res), fim(res);
    blocks = dim3(res.x / 8 + 1, res.y / 8 + 1);
    prr_ref_launch(blocks, threads, [&] { combineSamples(rays, im, res, samples); });
    for (int i = 0; i < res.x * res.y; i++) {
        f3 c = im[i];
        if (image) { image[3 * i] = c.x; image[3 * i + 1] = c.y; image[3 * i + 2] = c.z; }
    }
    if (fxaa_im) {
        prr_ref_launch(blocks, threads, [&] { fxaa(im, fim); });
        for (int i = 0; i < res.x * res.y; i++) {
            f3 c = fim[i];
            fxaa_im[3 * i] = c.x; fxaa_im[3 * i + 1] = c.y; fxaa_im[3 * i + 2] = c.z;
        }
    }
    im.unload();
    fim.unload();
    return secs;
}

// Frame set-up for a sampled trace: camera pose and scene update
// (prr.cpp:245-253), createRays_* and initRays over the whole frame.
int prr_ref_prepare(int frame, int nthreads)
{
    if (!g_loaded) return 1;
    g_threads = nthreads > 0 ? nthreads : 1;
    Ray *rays = g_rays;
    i2 res = camera.getRes();
    int samples = camera.getAAsamples();
    std::string header = "frame" + to_string(frame);
    camera.pos = f3(parf(header, "x"), parf(header, "y"), parf(header, "z"));
    camera.a = parf(header, "a") * M_PI / 180.0f;
    camera.b = parf(header, "b") * M_PI / 180.0f;
    camera.computeVectors();
    spacetime.updateScene(frame);
#ifdef SPHERICAL
    camera.spos = pos_cartTOspher(camera.pos);
#endif
    spacetime.setBhMass(parf(header, "mass", spacetime.getBhMass()));
    dim3 blocks(res.x / 8 + 1, res.y / 8 + 1), threads(8, 8);
    if (camera.getSSAADistr() == SSAA_DISTR::NONE) prr_ref_launch(blocks, threads, [&] { createRays_none(rays, res); });
    else prr_ref_launch(blocks, threads, [&] { createRays_regular(rays, res, samples); });
    blocks = dim3(samples * res.x / 8 + 1, res.y / 8 + 1);
    prr_ref_launch(blocks, threads, [&] { initRays(rays, camera, spacetime, samples); });
    return 0;
}

// Traces a sample of 8-ray blocks with the reference kernel: block k covers
// rays x = 8*bx[k] .. 8*bx[k]+7 of row[k] (in the (samples*width, height)
// ray image), i.e. trace_RKF/trace_Euler launched as a one-row layer with
// blockIdx = (bx[k], 0) and blockDim = (8, 1).  Returns wall seconds.
double prr_ref_trace_blocks(int nthreads, int nblocks, const int *bx, const int *row)
{
    if (!g_loaded) return -1.0;
    Ray *rays = g_rays;
    int samples = camera.getAAsamples();
    auto t0 = std::chrono::steady_clock::now();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads > 0 ? nthreads : 1)
    for (int k = 0; k < nblocks; k++) {
        gridDim = dim3(1, 1);
        blockDim = dim3(8, 1);
        blockIdx.x = (unsigned)bx[k]; blockIdx.y = 0; blockIdx.z = 0;
        for (unsigned tx = 0; tx < 8; ++tx) {
            threadIdx.x = tx; threadIdx.y = 0; threadIdx.z = 0;
            if (trace.solver == SOLVER::EULER) trace_Euler(rays, camera, spacetime, trace, row[k], 1, samples);
            else trace_RKF(rays, camera, spacetime, trace, row[k], 1, samples);
        }
    }
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// Result enum of ray i after tracing.
int prr_ref_ray_result(long long i) { return (g_loaded && i >= 0 && (size_t)i < g_nrays) ? (int)g_rays[i].result : -1; }

// The reference's PNG path (tex2d::save -> Images::savePNGToFile,
// cudamaths/tex2d.cuh:83-99, cudamaths/image.cu:28-39) on a host image.
int prr_ref_save_png(const char *path, const float *image, int w, int h)
{
    return Images::get().savePNGToFile(path, (f3 *)image, i2(w, h)) ? 0 : 1;
}

// ---- the reference's deck parser and getters, for parity tests of the
//      product's deck reader (main/io.h:21-58, main/Parameters.cpp:10-44,
//      prr.cpp:139-153) ----

// readParams of one file into an emptied table (no traj/scene, no scene).
int prr_ref_parse(const char *path)
{
    Parameters::get().parameters.clear();
    readParams(path, &Parameters::get().parameters);
    return 0;
}

int prr_ref_has_block(const char *block) { return headerExists(block) ? 1 : 0; }
int prr_ref_has(const char *block, const char *key) { return parExists(block, key) ? 1 : 0; }

size_t prr_ref_par(const char *block, const char *key, char *buf, size_t len)
{
    std::string v = par(block, key);
    if (buf && len) {
        size_t n = v.size() < len - 1 ? v.size() : len - 1;
        memcpy(buf, v.data(), n);
        buf[n] = 0;
    }
    return v.size();
}

int prr_ref_pari(const char *block, const char *key) { return pari(block, key); }
float prr_ref_parf(const char *block, const char *key) { return parf(block, key); }
float prr_ref_parf_d(const char *block, const char *key, float dflt) { return parf(block, key, dflt); }
int prr_ref_check_frame(void) { return checkFrame(); }

// Number of (block, key) entries and the i-th of them in map order.
int prr_ref_entry_count(void)
{
    int n = 0;
    for (auto &b : Parameters::get().parameters) n += (int)b.second.size();
    return n;
}

int prr_ref_entry(int i, char *block, char *key, char *val, size_t len)
{
    for (auto &b : Parameters::get().parameters)
        for (auto &kv : b.second) {
            if (i-- != 0) continue;
            snprintf(block, len, "%s", b.first.c_str());
            snprintf(key, len, "%s", kv.first.c_str());
            snprintf(val, len, "%s", kv.second.c_str());
            return 0;
        }
    return 1;
}

}  // extern "C"
