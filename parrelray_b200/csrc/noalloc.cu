// noalloc.cu - prr_render_noalloc: the persistent renderer for callers that
// cannot allocate device memory at render time.
//
// Who needs this: applications that own every byte of device memory up front
// - an engine or service that carves its whole budget out of one arena at
// start-up and hands out pieces of it itself, or a real-time loop that cannot
// afford the implicit device synchronisation a cudaMalloc/cudaFree may cause.  prr_render needs a
// context, and a context grows its scratch buffers with cudaMalloc on demand;
// this entry point takes every input and output from the caller and keeps its
// only scratch (the work counters, the frame table and the per-frame pixel
// prefix) in one fixed static device array below.
//
// Limits and sharing rules:
//  * at most PRR_NOALLOC_MAX_FRAMES frames per call (larger n is rejected
//    with PRR_ERR_INVALID before anything is launched);
//  * the scratch array exists once per device for the life of the process
//    (every GPU that loads the library holds its PRR_NOALLOC_SCRATCH_BYTES);
//  * every call on a device shares it and it keeps the previous call's
//    contents, so the counters are cleared at the start of each call, and
//    calls whose GPU work overlaps (different streams, or host threads
//    without ordering) race on it: order them on one stream;
//  * the first call on a device looks up the array's device address
//    (cudaGetSymbolAddress) with that device current; make that first call
//    before any stream capture.
#include <cstring>
#include <mutex>
#include <string>

#include "kernels.cuh"
#include "prr_internal.h"

using namespace prr;

namespace {

constexpr size_t kCountersBytes = C_COUNT * sizeof(unsigned long long);
constexpr size_t kBeginOffset = 256;
constexpr size_t kFramesOffset = 1024;
constexpr size_t kScratchBytes = PRR_NOALLOC_SCRATCH_BYTES;

static_assert(kCountersBytes <= kBeginOffset, "counters overflow their slot");
static_assert(kBeginOffset + (PRR_NOALLOC_MAX_FRAMES + 1) * sizeof(long long) <= kFramesOffset, "frame prefix overflows its slot");
static_assert(kFramesOffset + PRR_NOALLOC_MAX_FRAMES * sizeof(FrameParams) <= kScratchBytes, "scratch array too small");

// The scratch: work counters | pixel prefix (n+1) | frame table (n).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
void *g_scratch_addr[kMaxDevices] = {};

void set_err(char *buf, size_t len, const std::string &msg)
{
    if (!buf || len == 0) return;
    size_t n = msg.size() < len - 1 ? msg.size() : len - 1;
    memcpy(buf, msg.data(), n);
    buf[n] = '\0';
}

}  // namespace

extern "C" prr_status prr_render_noalloc(const prr_frame_desc *frames, int n, const uint8_t *const *d_textures,
                                         const int32_t *tex_w, const int32_t *tex_h, uint8_t *d_rgb8, float *d_rgbf,
                                         void *stream, char *errbuf, size_t errlen)
{
    set_err(errbuf, errlen, "");
    if (!frames || n < 1) { set_err(errbuf, errlen, "need at least one frame"); return PRR_ERR_INVALID; }
    if (n > PRR_NOALLOC_MAX_FRAMES) {
        set_err(errbuf, errlen, "prr_render_noalloc renders at most " + std::to_string(PRR_NOALLOC_MAX_FRAMES) +
                                    " frames per call (its scratch is a fixed static array); got " + std::to_string(n));
        return PRR_ERR_INVALID;
    }
    if (!d_rgb8) { set_err(errbuf, errlen, "d_rgb8 (device output) is required"); return PRR_ERR_INVALID; }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        set_err(errbuf, errlen, "no usable CUDA device");
        return PRR_ERR_NO_DEVICE;
    }
    // once per device, with that device current: the array's device address
    void *scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if (!g_scratch_addr[dev]) {
            cudaError_t e = cudaGetSymbolAddress(&g_scratch_addr[dev], g_noalloc_scratch);
            if (e != cudaSuccess) {
                g_scratch_addr[dev] = nullptr;
                set_err(errbuf, errlen, std::string("cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
                return PRR_ERR_CUDA;
            }
        }
        scratch = g_scratch_addr[dev];
    }
    // Validate and lay out the frames with a context that owns nothing: its
    // texture slots point at the caller's device textures.
    prr_ctx view;
    view.device = dev;
    for (int i = 0; i < PRR_MAX_TEXTURES; i++) {
        if (d_textures && d_textures[i]) {
            if (!tex_w || !tex_h || tex_w[i] < 2 || tex_h[i] < 2) {
                set_err(errbuf, errlen, "texture " + std::to_string(i) + " needs a width and height >= 2");
                return PRR_ERR_INVALID;
            }
            view.tex[i].buf.p = (void *)d_textures[i];
            view.tex[i].buf.cap = (size_t)tex_w[i] * tex_h[i] * 4;
            view.tex[i].w = tex_w[i];
            view.tex[i].h = tex_h[i];
        }
    }
    RenderPlan plan;
    prr_status s = build_plan(&view, frames, n, plan);
    for (auto &t : view.tex) t.buf.p = nullptr;  // the view never owned them
    if (s != PRR_OK) { set_err(errbuf, errlen, view.err); return s; }
    if (plan.mode != PRR_MODE_PHYSICAL || plan.precision == PRR_PREC_SPLIT) {
        set_err(errbuf, errlen, "prr_render_noalloc supports PHYSICAL mode in FP32 or FP64 (not REFERENCE, not SPLIT)");
        return PRR_ERR_UNSUPPORTED;
    }
    if (plan.any_fxaa && !d_rgbf) {
        set_err(errbuf, errlen, "frames with FXAA need d_rgbf: it receives the combined image the FXAA pass reads");
        return PRR_ERR_INVALID;
    }
    cudaStream_t st = (cudaStream_t)stream;
    unsigned char *base = (unsigned char *)scratch;
    unsigned long long *counters = (unsigned long long *)base;
    long long *begin = (long long *)(base + kBeginOffset);
    FrameParams *fps = (FrameParams *)(base + kFramesOffset);
    int nsm = 0;
    cudaError_t e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaMemsetAsync(counters, 0, kCountersBytes, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(begin, plan.pix_begin.data(), (n + 1) * sizeof(long long), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(fps, plan.fp.data(), n * sizeof(FrameParams), cudaMemcpyHostToDevice, st);
    // the host tables are freed on return: complete the copies first
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    PersistentArgs a;
    memset(&a, 0, sizeof(a));
    a.frames = fps;
    a.frame_pix_begin = begin;
    a.nframes = n;
    a.total_pixels = plan.total_pixels;
    a.image = d_rgbf;
    a.rgb8 = d_rgb8;
    a.counters = counters;
    a.compaction_interval = 1;
    a.emission = plan.any_emission;
    const int block = 128;
    int bpsm = persistent_occupancy(plan.precision, 0, block, 1, plan.any_emission);
    if (e == cudaSuccess) e = launch_persistent(a, plan.precision, block, bpsm > 0 ? bpsm : 1, nsm, st);
    for (int f = 0; f < n && e == cudaSuccess; f++) {
        const FrameParams &p = plan.fp[f];
        if (p.fxaa) e = launch_finish(d_rgbf + 3 * p.pix_begin, p.width, p.height, 1, nullptr, d_rgb8 + 3 * p.pix_begin, st);
    }
    if (e != cudaSuccess) {
        set_err(errbuf, errlen, std::string("CUDA error: ") + cudaGetErrorString(e));
        return PRR_ERR_CUDA;
    }
    return PRR_OK;
}
