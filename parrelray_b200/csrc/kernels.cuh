// kernels.cuh - host-visible launch wrappers of every kernel in the library
// (each defined in the .cu file named beside it).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "prr_device.cuh"

namespace prr {

// Device counters accumulated by the tracing kernels.
enum Counter {
    C_RAYS = 0,
    C_ATTEMPTS,
    C_ACCEPTED,
    C_ESCAPED,
    C_CAPTURED,
    C_INTERSECTION,
    C_INFINITE,
    C_MATH_ERROR,
    C_FP64,
    C_WORK,          // persistent scheduler: next work item
    C_WORK_FP64,     // split precision: next FP64 work item
    C_FP64_QUEUED,   // split precision: queue length
    C_TIMEOUT,       // watchdog fired
    C_COUNT = 16
};

// k_reference.cu: REFERENCE-mode tracing, one thread per ray of frame
// `frame` (rays [0, nrays)).  state: 12 floats/ray, rgb: 3 floats/ray (either
// may be null).
cudaError_t launch_ref_trace(const FrameParams *d_fp, int frame, long long nrays, float *state, float *rgb,
                             unsigned long long *counters, cudaStream_t st);

// post.cu: SSAA combine of per-sample colours into an FP32 image.
cudaError_t launch_combine(const float *rgb, int w, int h, int samples, float *image, cudaStream_t st);
// post.cu: FXAA (optional) + quantise.  Writes out_f (FP32, may be null) and
// out_u8 (3 bytes/pixel, may be null).  in and out_f must differ when fxaa.
cudaError_t launch_finish(const float *image, int w, int h, int fxaa, float *out_f, uint8_t *out_u8, cudaStream_t st);

// k_persistent.cu: PHYSICAL-mode persistent renderer over a batch of frames.
struct PersistentArgs {
    const FrameParams *frames;   // device array
    const long long *frame_pix_begin;  // device array, nframes+1 prefix of pixel counts
    int nframes;
    long long total_pixels;      // work items (pixels over all frames)
    float *image;                // combined FP32 image, 3 floats/pixel (all frames)
    uint8_t *rgb8;               // optional direct quantised output (frames without FXAA)
    float *sample_rgb;           // per-sample colours (split precision; optional otherwise)
    unsigned long long *fp64_queue;  // split precision: flagged ray ids
    long long fp64_capacity;
    unsigned long long *counters;
    float *ray_state;            // optional per-ray debug state, 12 floats/ray (single frame)
    double *ray_state64;         // optional per-ray debug state, 12 doubles/ray (FP64, single frame)
    int geod_table;              // 1 = Christoffel-table geodesic (for comparisons)
    int compaction_interval;     // attempts between warp refills (>= 1)
    long long watchdog_cycles;   // 0 = off
    int rays_per_thread;         // FP32: pixel slots in flight per thread (1 or 2; 0 = 1)
    int *ray_steps;              // optional: accepted steps per ray (not k_pair; single frame)
    int emission;                // 1 = some frame has plasma emission (the kernels with emission.cuh)
    int hamiltonian;             // PRR_HAM_FP32 | PRR_HAM_FP64 mask: renders that integrate (x, p) in Hamiltonian form (k_ham.cu)
};
// Dispatches to the kernel of the precision: FP32 with one pixel slot per
// thread (emission included) and the FP32 pass of SPLIT with PRR_HAM_FP32 in
// a.hamiltonian, and FP64 with PRR_HAM_FP64 -> k_ham (k_ham.cu); other FP32
// renders with the register contraction -> k_pair (k_pair.cu,
// rays_per_thread slots per thread); other FP64 renders and the
// Christoffel-table variant -> k_persistent.
cudaError_t launch_persistent(const PersistentArgs &a, int precision, int block, int blocks_per_sm, int nsm, cudaStream_t st);

// k_persistent.cu: resident CTAs per SM of the kernel launch_persistent picks.
int persistent_occupancy(int precision, int geod_table, int block, int rays_per_thread = 1, int emission = 0,
                         int hamiltonian = 0);

// k_ham.cu: the renderer in Hamiltonian form (one pixel slot per thread), in
// `precision` PRR_PREC_FP32 or PRR_PREC_FP64; `split`: the FP32 pass of a
// split-precision render (needs sample_rgb and fp64_queue); a.emission: the
// instantiation with plasma emission.
cudaError_t launch_ham(const PersistentArgs &a, int precision, bool split, int block, int blocks_per_sm, int nsm,
                       cudaStream_t st);
int ham_occupancy(int precision, int block, bool split = false, bool emission = false);
// k_ham.cu: the FP64 pass of a split-precision render in Hamiltonian form
// (launch_fp64_requeue calls it when a.hamiltonian has PRR_HAM_FP64).
cudaError_t launch_ham_requeue(const PersistentArgs &a, int nsm, cudaStream_t st);

// k_pair.cu: the FP32 renderer with `rpt` pixel slots per thread; `split`:
// the FP32 pass of a split-precision render (rpt 1; needs sample_rgb and
// fp64_queue); a.emission: the instantiation with plasma emission (rpt 1).
cudaError_t launch_pair(const PersistentArgs &a, int rpt, bool split, int block, int blocks_per_sm, int nsm, cudaStream_t st);
int pair_occupancy(int rpt, bool split, int block, bool emission = false);

// k_persistent.cu: FP64 re-integration of the queued rays of a split render.
cudaError_t launch_fp64_requeue(const PersistentArgs &a, int block, int nsm, cudaStream_t st);

// k_plain.cu: the reference's pipeline structure with PHYSICAL math.
struct PlainBuffers {
    void *rays;      // AoS ray records, one per sample
    float *rgb;      // per-sample colours
};
cudaError_t launch_plain_frame(const FrameParams *d_fp, const FrameParams &h_fp, int frame, PlainBuffers &b,
                               unsigned long long *counters, int geod_table, cudaStream_t st, int *launches);
size_t plain_ray_record_bytes();

// k_adjoint.cu: discrete adjoint of one PHYSICAL frame: forward steps in
// `precision` (PRR_PREC_FP32 or FP64), adjoint and reduction in FP64.
struct AdjointParamsHost {
    double spin, mass, incl, cam_r, phase, sph_R, sph_z;
    int sphere;
};
cudaError_t launch_adjoint(const FrameParams *d_fp, const AdjointParamsHost &p, const float *dL, const float *image,
                           void *ckpt, int max_ckpt, int threads_total, double *grad, unsigned long long *counters,
                           long long nrays, const unsigned *order, int precision, cudaStream_t st);
// k_adjoint.cu: ray order for the adjoint, longest first: `order` receives the
// ray indices sorted by descending accepted-step count `steps` (nrays
// entries), so the rays a warp processes together have similar lengths.
// scratch: adjoint_order_bytes(nrays) bytes.
size_t adjoint_order_bytes(long long nrays);
cudaError_t launch_adjoint_order(const int *steps, long long nrays, unsigned *order, void *scratch, cudaStream_t st);
size_t adjoint_checkpoint_bytes(int precision);
int adjoint_blocks_per_sm(int precision);  // resident 128-thread CTAs of k_adjoint per SM
constexpr int ADJ_CHECKPOINT_INTERVAL = 64;

// fma_peak.cu
cudaError_t launch_fma_peak(float *sink, int blocks, int threads, int iters, cudaStream_t st);
cudaError_t launch_dfma_peak(double *sink, int blocks, int threads, int iters, cudaStream_t st);
// fma_peak.cu: frcp/frsqrt (FP64 and FP32) on n inputs, 4 outputs each
cudaError_t launch_check_recip(const double *x, int n, double *out, cudaStream_t st);

}  // namespace prr
