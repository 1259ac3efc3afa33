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
// The host never waits for the GPU here: the frame table travels to the
// scratch array inside the parameters of a small staging kernel (kernel
// parameters are copied at launch, so the host tables may go away when the
// call returns), and every launch is stream-ordered on the caller's stream.
//
// Limits and sharing rules:
//  * at most PRR_NOALLOC_MAX_FRAMES frames per call (larger n is rejected
//    with PRR_ERR_INVALID before anything is launched);
//  * the scratch array exists once per device for the life of the process
//    (every GPU that loads the library holds its PRR_NOALLOC_SCRATCH_BYTES);
//  * every call on a device shares it and it keeps the previous call's
//    contents, so the staging kernel clears the counters at the start of
//    each call, and calls whose GPU work overlaps (different streams, or host
//    threads without ordering) race on it: order them on one stream;
//  * each call looks up the array's device address with cudaGetSymbolAddress
//    (it allocates nothing), with the calling thread's current device; the
//    first call on a device can load the library's device code there, so
//    make that first call before any stream capture on that device.
#include <cstring>
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

// Frames staged per launch of k_noalloc_stage: the chunk rides in the kernel
// parameters (at most 32,764 bytes of parameters per launch on sm_70 and
// later with CUDA 12.1+ drivers; kept well below that).
constexpr int kChunkFrames = 32;
struct FrameChunk {
    int first, count, nframes, clear;
    long long total_pixels;
    FrameParams f[kChunkFrames];
};
static_assert(sizeof(FrameChunk) + 64 <= 32000, "staging chunk exceeds the kernel parameter space");
static_assert(sizeof(FrameParams) % 4 == 0, "frame parameters are copied as 32-bit words");

// Copies one chunk of the frame table into the scratch array, writes the
// chunk's entries of the pixel prefix (and its end on the last chunk) and,
// on the first chunk, clears the counters.
__global__ void k_noalloc_stage(const FrameChunk c, unsigned char *scratch)
{
    unsigned long long *counters = (unsigned long long *)scratch;
    long long *begin = (long long *)(scratch + kBeginOffset);
    FrameParams *fps = (FrameParams *)(scratch + kFramesOffset);
    const unsigned words = (unsigned)(c.count * sizeof(FrameParams) / 4);
    const unsigned *src = (const unsigned *)c.f;
    unsigned *dst = (unsigned *)(fps + c.first);
    for (unsigned i = threadIdx.x; i < words; i += blockDim.x) dst[i] = src[i];
    if ((int)threadIdx.x < c.count) begin[c.first + threadIdx.x] = c.f[threadIdx.x].pix_begin;
    if (threadIdx.x == 0 && c.first + c.count == c.nframes) begin[c.nframes] = c.total_pixels;
    if (c.clear && threadIdx.x < C_COUNT) counters[threadIdx.x] = 0ull;
}

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
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        set_err(errbuf, errlen, "no usable CUDA device");
        return PRR_ERR_NO_DEVICE;
    }
    // the array's device address on the current device (in host code its
    // name is only a host-side stand-in)
    void *scratch = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&scratch, g_noalloc_scratch);
    if (e != cudaSuccess || !scratch) {
        cudaGetLastError();
        set_err(errbuf, errlen, std::string("cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
        return PRR_ERR_CUDA;
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
    int nsm = 0;
    e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    // the frame table, the pixel prefix and cleared counters, stream-ordered
    for (int first = 0; first < n && e == cudaSuccess; first += kChunkFrames) {
        FrameChunk c;
        memset(&c, 0, sizeof(c));
        c.first = first;
        c.count = n - first < kChunkFrames ? n - first : kChunkFrames;
        c.nframes = n;
        c.clear = first == 0;
        c.total_pixels = plan.total_pixels;
        memcpy(c.f, plan.fp.data() + first, c.count * sizeof(FrameParams));
        k_noalloc_stage<<<1, 256, 0, st>>>(c, base);
        e = cudaGetLastError();
    }
    PersistentArgs a;
    memset(&a, 0, sizeof(a));
    a.frames = (const FrameParams *)(base + kFramesOffset);
    a.frame_pix_begin = (const long long *)(base + kBeginOffset);
    a.nframes = n;
    a.total_pixels = plan.total_pixels;
    a.image = d_rgbf;
    a.rgb8 = d_rgb8;
    a.counters = (unsigned long long *)base;
    a.emission = plan.any_emission;
    a.hamiltonian = PRR_HAM_FP32 | PRR_HAM_FP64;  // a context's default
    // the launch shape prr_autotune picks for the 1080p Kerr workload: CTAs of
    // 64 threads at their occupancy limit, one pixel per thread, a warp refill
    // every 64 attempts
    const int block = 64;
    a.compaction_interval = 64;
    a.rays_per_thread = 1;
    const int bpsm = persistent_occupancy(plan.precision, 0, block, 1, plan.any_emission, a.hamiltonian);
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
