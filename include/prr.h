/*
 * prr.h - C ABI of prr-b200, the B200-native ParRelRay ray tracer.
 *
 * Plain C, plain pointers and sizes.  Every entry point returns a prr_status
 * (0 = PRR_OK); the message of the last failure on a context is available
 * from prr_last_error().  No exceptions cross this boundary.  The caller owns
 * every host buffer; a context owns its device buffers.  Calls on one
 * context are synchronous unless named *_device (those are asynchronous on
 * the given CUDA stream).  One context per host thread.
 *
 * The reference (GKylian/ParRelRay) has no runtime API: its "plugin" surface
 * is the compile-time metric header (main/metric.h:12) plus the .params
 * deck (main/io.h:21-58).  Each entry point below names the reference code it
 * replaces.
 */
#ifndef PRR_H
#define PRR_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PRR_ABI_VERSION 4
#define PRR_MAX_SPHERES 8
#define PRR_MAX_TEXTURES 32

typedef struct prr_ctx prr_ctx;

typedef enum prr_status {
    PRR_OK = 0,
    PRR_ERR_INVALID = 1,     /* bad argument / descriptor */
    PRR_ERR_CUDA = 2,        /* CUDA runtime error (message in prr_last_error) */
    PRR_ERR_NOMEM = 3,       /* allocation failed */
    PRR_ERR_TIMEOUT = 4,     /* device watchdog expired; rays left unfinished */
    PRR_ERR_IO = 5,          /* file could not be read or written */
    PRR_ERR_UNSUPPORTED = 6, /* option not implemented */
    PRR_ERR_NO_DEVICE = 7    /* no CUDA device / extension unusable */
} prr_status;

/* Integration result per ray; same values as the reference enum RESULT
 * (main/base.h:37-43). */
typedef enum prr_result {
    PRR_RESULT_SUCCESS = 0,
    PRR_RESULT_MATH_ERROR = 1,
    PRR_RESULT_IO_ERROR = 2,
    PRR_RESULT_INFINITE_GEO = 3,
    PRR_RESULT_INTERSECTION = 4
} prr_result;

/* Solver ids; same values as the reference enum SOLVER (main/base.h:26-34).
 * Only EULER and RKF45 are integrators in the reference (prr.cpp:295-305). */
typedef enum prr_solver { PRR_SOLVER_EULER = 0, PRR_SOLVER_RKF45 = 2 } prr_solver;

/* SSAA sample placement; same values as SSAA_DISTR (main/base.h:46-53).
 * NONE and REGULAR are createRays_none/_regular (kernels/ssaa.cuh:92-99,
 * 36-48).  RANDOM (samples uniform in the pixel) and JITTERED (one sample
 * uniform in each cell of an n x n grid, samples = n^2) exist in the
 * reference only as kernels it never launches (ssaa.cuh:55-86, whose random
 * offsets are not scaled to a pixel); here they are PHYSICAL-mode options
 * with offsets from a counter-based hash of (ssaa_seed, pixel, sample), so a
 * frame renders the same on every call. */
typedef enum prr_ssaa { PRR_SSAA_NONE = 0, PRR_SSAA_REGULAR = 1, PRR_SSAA_RANDOM = 2, PRR_SSAA_JITTERED = 4 } prr_ssaa;

/* Ray-direction model (main/Camera.h:30-42).  SPHERICAL is the one the
 * reference's initRays uses (rayDir_Spherical); PINHOLE and PANORAMA are
 * its other two models (rayDir_PinHole, rayDir_Panorama; never called by
 * the reference), PHYSICAL mode only.  Both use the basis of
 * Camera::computeVectors (main/Camera.cpp:19-28) evaluated at pitch -b,
 * because computeVectors takes the pitch with the opposite sign from
 * rayDir_Spherical: so all three models look the same way for one (a, b),
 * and the image's left edge is on the same side.  PANORAMA is the
 * equirectangular model sin(mu) up + cos(mu)(cos(nu) forward + sin(nu) right)
 * with nu growing to the right; the reference's rayDir_Panorama multiplies
 * its up term by mu as well and mirrors nu. */
typedef enum prr_camera { PRR_CAMERA_SPHERICAL = 0, PRR_CAMERA_PINHOLE = 1, PRR_CAMERA_PANORAMA = 2 } prr_camera;

typedef enum prr_metric {
    PRR_METRIC_FLAT = 0,          /* metrics/flat.cuh */
    PRR_METRIC_SCHWARZSCHILD = 1, /* metrics/schwarzschild.cuh (Kerr-Schild form) */
    PRR_METRIC_KERR = 2           /* Kerr-Schild Kerr (new; the reference's is a stub) */
} prr_metric;

/* Integration semantics.
 * REFERENCE: reproduces kernels/solver.cuh exactly, quirks included (stage
 *   inputs of the velocity use h*u, solver.cuh:164-168; the initial 4-velocity
 *   is (dir,1)*u0, solver.cuh:54; absolute error test against eps,
 *   solver.cuh:174-188).  FP32 only.  Used for parity with the reference.
 * PHYSICAL: textbook RKF45 stages, null initial 4-velocity (dir, u^t), and a
 *   mixed error test |y5-y4| <= atol + rtol*|y| that works in FP32 down to
 *   1e-7.  Every other rule (hooks, sphere test, colours) is unchanged. */
typedef enum prr_mode { PRR_MODE_REFERENCE = 0, PRR_MODE_PHYSICAL = 1 } prr_mode;

/* Arithmetic of the integrator (PHYSICAL mode).
 * FP32: FP32 stages with Kahan-compensated state accumulation.
 * FP64: everything in FP64.
 * SPLIT: FP32 pass; rays flagged near the critical impact parameter or near
 *        the horizon are re-integrated in FP64. */
typedef enum prr_precision { PRR_PREC_FP32 = 0, PRR_PREC_FP64 = 1, PRR_PREC_SPLIT = 2 } prr_precision;

/* How rays are scheduled on the GPU.
 * PLAIN: one ray per thread, one kernel per pipeline stage, 64-row layers,
 *        generic Christoffel-table geodesic (the reference's structure).
 * PERSISTENT: persistent CTAs, warp-ballot ray compaction, fused ray
 *        generation/integration/colouring/SSAA combine, Kerr-Schild
 *        contraction in registers. */
typedef enum prr_schedule { PRR_SCHED_PLAIN = 0, PRR_SCHED_PERSISTENT = 1 } prr_schedule;

/* Background lookup.  RMS2X2 is the reference's OutSphere::getColorDefault2
 * (main/base.h:119-162, piecewise constant); BILINEAR is a continuous lookup
 * used for gradients. */
typedef enum prr_bg_filter { PRR_BG_RMS2X2 = 0, PRR_BG_BILINEAR = 1 } prr_bg_filter;

/* Emission from plasma around the hole (PHYSICAL mode, FP32 or FP64).  The
 * reference declares the fields (main/Spacetime.h:50-51: density, pressure,
 * temperature, velocity, magnetic field on a grid of dataDim cells) and a
 * per-ray luminosity integrated along the path (Ray::I, main/base.h:175),
 * and uses neither; this is the model that fills them in.
 *
 * Along each ray, at every accepted step of affine length h, with n the
 * plasma density, u_e the plasma 4-velocity, k the ray's 4-momentum and
 * g = (k.u_cam)/(k.u_e) the frequency ratio (u_cam: a static observer at the
 * camera):
 *     I   += trans * g^(2 + spectral_index) * j * nu_cam * h,  j = n * Theta^temp_power
 *     trans *= exp(-absorb * n * nu_cam * h / g)
 * (nu_cam = -k.u_cam scales h to the affine length of a ray whose camera
 * frequency is 1; this is the invariant transfer equation d(I_nu/nu^3)/dl =
 * j_nu/nu^2 for a spectrum j_nu ~ nu^-spectral_index, with grey absorption.)
 * Points where the flow is not timelike or k.u_e >= 0 emit nothing.  The
 * pixel colour is trans * (the colour without emission) + map(gain * I).
 *
 * Rays are traced forward from the camera (as every mode here and the
 * reference do), so the received picture is the time reverse of the traced
 * scene: in Kerr the hole of spin -a; every flow velocity reversed.  g is
 * invariant under that reversal, so the formula above is exact for it.
 *
 * DISK: n = (r / r_in)^(-index) * exp(-cos^2(theta) / (2 height^2)) for
 *   r_in <= r <= r_out (Kerr-Schild r, cos theta = z / r), 0 elsewhere;
 *   Theta = 1; u_e on circular orbits of angular velocity
 *   Omega = sense sqrt(M) / (r^1.5 + sense a sqrt(M)) about the z axis
 *   (the equatorial Keplerian value at the point's r; sense +1 co-rotates
 *   with the hole).
 * GRID: n, Theta and (optionally) the coordinate velocity dx^i/dt from the
 *   plasma grid of prr_upload_plasma, trilinear between its nodes, 0
 *   outside its box and outside [r_in, r_out]; without a velocity field the
 *   flow is the DISK's. */
typedef enum prr_emission { PRR_EMISSION_NONE = 0, PRR_EMISSION_DISK = 1, PRR_EMISSION_GRID = 2 } prr_emission;

/* map(x) of the emission colour: AFMHOT (clamp(2x), clamp(2x - 1/2),
 * clamp(2x - 1)) or GREY (clamp(x) in all three channels). */
typedef enum prr_colormap { PRR_CMAP_AFMHOT = 0, PRR_CMAP_GREY = 1 } prr_colormap;

typedef struct prr_emission_desc {
    float index;          /* DISK: radial density power law */
    float height;         /* DISK: Gaussian width in cos(theta) (> 0) */
    float r_in, r_out;    /* emitting shell, Kerr-Schild r */
    float spectral_index; /* j_nu ~ nu^-spectral_index */
    float absorb;         /* grey absorption per unit density (>= 0) */
    float gain;           /* colour scale of I */
    int32_t sense;        /* +1 co-rotating, -1 counter-rotating (Keplerian flow) */
    float temp_power;     /* GRID: j = n * Theta^temp_power */
    int32_t colormap;     /* prr_colormap */
    int32_t _pad[2];
} prr_emission_desc;

/* A plasma grid (the reference's density/temperature/velocity fields,
 * main/Spacetime.h:50-51, with its dataDim = (nx, ny, nz)).  Nodes sit at
 * lo + (hi - lo) * (i, j, k) / (n - 1) in Kerr-Schild (x, y, z); arrays are
 * x-fastest (index i + nx * (j + ny * k)).  density is required (>= 0);
 * temperature (NULL: 1 everywhere) and velocity (3 floats per node, the
 * coordinate velocity dx/dt, dy/dt, dz/dt; NULL: the DISK flow) are
 * optional.  The reference's pressure and magnetic field are not used by the
 * emission model. */
typedef struct prr_plasma_desc {
    int32_t nx, ny, nz;   /* >= 2 each */
    float lo[3], hi[3];   /* box corners, lo < hi */
    const float *density;
    const float *temperature;
    const float *velocity;
} prr_plasma_desc;

/* A textured sphere (scene/sphere.h:19-65). */
typedef struct prr_sphere {
    float center[3];
    float radius;
    int32_t texture_id; /* id given to prr_upload_texture; -1 = untextured (grey) */
    int32_t _pad[3];
} prr_sphere;

/* Everything one frame (one render request) needs.  Field meanings follow
 * the reference deck (prr.cpp:159-198, 245-253, Spacetime.cpp:17-44). */
typedef struct prr_frame_desc {
    /* camera (main/Camera.h:39-42) */
    int32_t width, height;
    int32_t ssaa;        /* prr_ssaa */
    int32_t samples;     /* rays per pixel; a perfect square for REGULAR */
    float vfov;          /* vertical field of view, radians */
    float cam_pos[3];    /* camera position (x, y, z) */
    float cam_alpha;     /* yaw a, radians */
    float cam_beta;      /* pitch b, radians */
    /* spacetime */
    int32_t metric;      /* prr_metric */
    float mass;          /* M (rs = 2M) */
    float spin;          /* a (length units; |a| <= M) */
    /* tracer (main/base.h:166-170) */
    int32_t solver;      /* prr_solver */
    int32_t mode;        /* prr_mode */
    int32_t precision;   /* prr_precision (PHYSICAL mode) */
    float h, hmin, hmax; /* initial / minimum / maximum step */
    float eps;           /* REFERENCE mode absolute tolerance */
    float rtol, atol;    /* PHYSICAL mode tolerances */
    float rout;          /* outer sphere radius (Tracer::sph1.rout) */
    float horizon_eps;   /* stop when r <= r_+ + horizon_eps (reference: 0.001) */
    int32_t max_steps;   /* PHYSICAL mode accepted-step cap */
    int32_t background_id; /* texture id of the equirectangular sky; -1 = black */
    int32_t bg_filter;   /* prr_bg_filter */
    int32_t fxaa;        /* 1 = FXAA after the SSAA combine (kernels/ssaa.cuh:150-181) */
    float fp64_delta;    /* SPLIT: flag rays with |b - b_c|/b_c < fp64_delta */
    float fp64_rfac;     /* SPLIT: flag rays reaching r < fp64_rfac * r_+ */
    int32_t nspheres;
    int32_t camera;      /* prr_camera */
    uint32_t ssaa_seed;  /* RANDOM / JITTERED sample offsets */
    int32_t emission;    /* prr_emission (PHYSICAL mode, FP32/FP64, persistent schedule) */
    prr_sphere spheres[PRR_MAX_SPHERES];
    prr_emission_desc emis; /* used when emission != NONE */
} prr_frame_desc;

/* Counters of one render call (summed over frames). */
typedef struct prr_stats {
    int64_t rays;            /* rays traced (width*height*samples per frame) */
    int64_t attempts;        /* integrator attempts (accepted + rejected) */
    int64_t accepted;        /* accepted steps */
    int64_t n_escaped;       /* SUCCESS with r >= rout */
    int64_t n_captured;      /* SUCCESS at the horizon */
    int64_t n_intersection;  /* INTERSECTION */
    int64_t n_infinite;      /* INFINITE_GEO */
    int64_t n_math_error;    /* MATH_ERROR */
    int64_t n_fp64;          /* rays re-integrated in FP64 (SPLIT) */
    double kernel_ms;        /* device time of the render, CUDA events */
    int64_t kernel_launches; /* kernels launched by the call */
    double trace_ms;         /* device time of the tracing kernel(s) alone */
} prr_stats;

/* Launch shape of the persistent scheduler. */
typedef struct prr_launch_config {
    int32_t block_size;          /* threads per CTA (multiple of 32) */
    int32_t blocks_per_sm;       /* resident CTAs per SM requested */
    int32_t compaction_interval; /* attempts between warp refills */
    int32_t rays_per_thread;     /* FP32 renders: pixels in flight per thread, 1 or 2 (2: the two
                                    rays' stages share paired FP32 instructions); results do not
                                    depend on it */
} prr_launch_config;

/* ---- lifetime (replaces prr.cpp:main 345-404, init 203-227) ---- */
int prr_abi_version(void);
const char *prr_status_string(prr_status s);
/* Creates a context on CUDA device `device`; fails with PRR_ERR_NO_DEVICE
 * when no device is usable. */
prr_status prr_create(int device, prr_ctx **out);
void prr_destroy(prr_ctx *ctx);
const char *prr_last_error(const prr_ctx *ctx);

/* ---- textures (replaces tex2d::load, cudamaths/tex2d.cuh:50-80) ----
 * rgba8: w*h*4 bytes, row-major, row 0 first.  Texel value = byte/255 (the
 * reference loads with stbi_ldr_to_hdr_gamma(1), cudamaths/image.cu:15).
 * Alpha is ignored.  Re-uploading an id replaces it. */
prr_status prr_upload_texture(prr_ctx *ctx, int id, const uint8_t *rgba8, int w, int h);

/* ---- plasma (the grid behind the reference's Spacetime::setDataDimensions
 * and its density/temperature/velocity pointers, main/Spacetime.h:28,50-51;
 * the reference never fills them) ----
 * Copies the grid to the device; replaces the previous one.  Frames with
 * emission = GRID sample the grid present when they are rendered. */
prr_status prr_upload_plasma(prr_ctx *ctx, const prr_plasma_desc *plasma);

/* ---- rendering (replaces prr.cpp:renderframe 237-341 and the frame loop
 *      382-386) ----
 * Renders n frames in one batched launch.  Outputs are concatenated per
 * frame, each width*height pixels, row-major:
 *   out_rgb8: 3 bytes/pixel, round(255*x) (cudamaths/image.cu:31), may be NULL
 *   out_rgbf: 3 floats/pixel, the combined (and FXAA'd) colour, may be NULL
 * Synchronous; host buffers. */
prr_status prr_render(prr_ctx *ctx, const prr_frame_desc *frames, int n,
                      uint8_t *out_rgb8, float *out_rgbf, prr_stats *stats);

/* Same, with DEVICE output buffers, asynchronous on `stream` (a
 * cudaStream_t, NULL = legacy default stream).  `frames` is read before the
 * call returns.  Stats are not produced. */
prr_status prr_render_device(prr_ctx *ctx, const prr_frame_desc *frames, int n,
                             uint8_t *d_rgb8, float *d_rgbf, void *stream);

/* Per-ray final states of one frame, for parity checks (the Ray struct of
 * main/base.h:172-176 after trace_RKF, solver.cuh:142-219, and after
 * rayToRGB, metrics/schwarzschild.cuh:151-183).  Host buffers, may be NULL:
 *   out_state: 12 floats/ray = uv.x uv.y result r.x r.y r.z r.w u.x u.y u.z
 *              u.w accepted_steps
 *   out_rgb:   3 floats/ray, the per-sample colour
 * Ray order is the reference's: ((y*width + x)*samples + sample). */
prr_status prr_trace_rays(prr_ctx *ctx, const prr_frame_desc *frame,
                          float *out_state, float *out_rgb, prr_stats *stats);

/* FP64 variant of prr_trace_rays (state in doubles), PHYSICAL mode only. */
prr_status prr_trace_rays_f64(prr_ctx *ctx, const prr_frame_desc *frame,
                              double *out_state, double *out_rgb, prr_stats *stats);

/* ---- gradients (new; the reference has no derivative path) ----
 * Discrete adjoint of a PHYSICAL-mode RKF45 frame (no FXAA): given
 * dL_dimage (host, width*height*3 floats, the derivative of a scalar loss
 * with respect to the combined image), returns in grads[5] the derivatives of
 * the loss with respect to (spin a, mass M, camera inclination i [radians],
 * camera distance r, orbital phase of sphere `sphere_index` about z
 * [radians]; 0 when sphere_index is -1).  The frame must use an orbit camera:
 * position (r sin i, 0, r cos i), yaw pi, pitch i - pi/2.  Step sizes and
 * discrete events (accept/reject, termination, which sphere is hit) are
 * frozen at the forward run.  The forward run is in the frame's precision
 * (an FP32 frame takes FP32 RKF45 steps and checkpoints, FP64 and SPLIT
 * frames FP64 ones); the reverse sweep (recomputed stages and their
 * vector-Jacobian products) and the reduction are FP64 in both.  The RMS2X2
 * sky is piecewise constant (zero gradient); use PRR_BG_BILINEAR for sky
 * gradients.  The rays are visited longest first (ordered by their forward
 * step counts) so rays sharing a warp have similar lengths.
 * stats->kernel_ms is the device time of that ordering plus the adjoint
 * kernel, stats->trace_ms the forward render time, stats->accepted the
 * adjoint's forward steps and stats->n_math_error the rays it dropped (their
 * checkpoints did not fit max_steps, or a recomputed segment disagreed with
 * the forward steps; neither happens on valid frames). */
prr_status prr_adjoint(prr_ctx *ctx, const prr_frame_desc *frame, const float *dL_dimage, int sphere_index,
                       double grads[5], prr_stats *stats);

/* ---- rendering without device allocation ----
 * No counterpart in the reference (which allocates everything itself in
 * main(), prr.cpp:359-378).  For callers that cannot allocate device memory
 * while rendering - an application that reserves its whole device budget up
 * front and hands out pieces of it itself, or a real-time loop that must not
 * pay cudaMalloc's implicit synchronisation.  Every input and output is the
 * caller's: the frames (host array), the textures (PRR_MAX_TEXTURES device
 * pointers to RGBA8 data, NULL = absent, with their sizes) and the outputs
 * (device d_rgb8, and device d_rgbf, which frames with FXAA require: it
 * receives the combined image the FXAA pass reads; without FXAA it receives
 * the final float image and may be NULL).  PHYSICAL mode, FP32 or FP64,
 * persistent schedule, no context, launch shape 64-thread CTAs at their
 * occupancy limit with a warp refill every 64 attempts.  The only scratch is
 * one static device array of PRR_NOALLOC_SCRATCH_BYTES per device, so at
 * most PRR_NOALLOC_MAX_FRAMES frames per call (more is PRR_ERR_INVALID).
 * Calls share that array and it keeps the last call's contents (each call
 * clears what must start at zero): calls whose GPU work overlaps race, so
 * order them on one stream.  Each call looks up the array's device address
 * on the current device (cudaGetSymbolAddress, no allocation); the first call
 * on a device can load the library's device code, so make it before any
 * stream capture on that device.  Asynchronous on `stream` (NULL = legacy
 * default stream): the frame table reaches the device in the parameters of a
 * staging kernel, so the host never waits for the GPU and `frames` may be
 * reused when the call returns.  On failure a message is written to errbuf
 * (errlen bytes, may be NULL). */
#define PRR_NOALLOC_MAX_FRAMES 64
#define PRR_NOALLOC_SCRATCH_BYTES 65536
prr_status prr_render_noalloc(const prr_frame_desc *frames, int n, const uint8_t *const *d_textures,
                              const int32_t *tex_w, const int32_t *tex_h, uint8_t *d_rgb8, float *d_rgbf,
                              void *stream, char *errbuf, size_t errlen);

/* ---- recorded batches (new; replaces the per-frame host loop of
 *      prr.cpp:382-386, each iteration of which runs renderframe,
 *      prr.cpp:237-341, as a dozen synchronised launches) ----
 * prr_graph_create records the render of n PHYSICAL-mode frames (a camera
 * trajectory, a set of uneven requests) into a CUDA graph: a counter reset,
 * ONE persistent launch over all frames (frames fill each other's tails),
 * the FP64 pass of SPLIT precision, and the per-frame combine/FXAA passes
 * the frames need.  Outputs are device buffers, frames concatenated as in
 * prr_render; at least one must be non-NULL.  The graph owns its device
 * scratch and keeps the context's launch configuration of creation time
 * (call prr_autotune first for a tuned shape).  It embeds the device
 * addresses of the uploaded textures: do not re-upload a texture the frames
 * use while the graph lives (or call prr_graph_set_frames afterwards).  The
 * graph must be destroyed before its context.
 * prr_graph_launch replays it asynchronously on `stream` (NULL = legacy
 * default stream); replays on one graph must not overlap in time.
 * prr_graph_set_frames replaces the frame parameters (same count, and per
 * frame the same width, height, samples, FXAA flag, mode and precision),
 * e.g. the next trajectory segment, without re-recording.
 * prr_graph_stats waits for the last replay and returns its counters
 * (kernel_ms is 0: time replays with events on your stream); it returns
 * PRR_ERR_TIMEOUT when the context's watchdog fired during that replay. */
typedef struct prr_graph prr_graph;
prr_status prr_graph_create(prr_ctx *ctx, const prr_frame_desc *frames, int n, uint8_t *d_rgb8, float *d_rgbf,
                            prr_graph **out);
prr_status prr_graph_set_frames(prr_graph *g, const prr_frame_desc *frames, int n);
prr_status prr_graph_launch(prr_graph *g, void *stream);
prr_status prr_graph_stats(prr_graph *g, prr_stats *stats);
/* The launch shape recorded in the graph (blocks_per_sm resolved). */
prr_status prr_graph_get_launch_config(const prr_graph *g, prr_launch_config *cfg);
void prr_graph_destroy(prr_graph *g);

/* ---- metric plug-ins (replaces the compile-time selection of
 *      main/metric.h:12; the hooks a plug-in defines are the ones
 *      kernels/solver.cuh:43,81,87,96,106,154,163-168,197,209 and
 *      prr.cpp:319 call) ----
 * A metric header written for the reference - getMetric, getGeod,
 * User_LOOP, User_UPDATE, User_ENDLOOP and the rayToRGB kernel, including
 * "../main/base.h", "../main/Camera.h", "../main/Spacetime.h" and
 * "../cudamaths/mats.h" - is compiled UNCHANGED against this library's
 * compatibility tree (parrelray_b200/compat) into libprr_metric_<name>.so
 * (python -m parrelray_b200.build --metric <header>).  prr_load_metric_plugin
 * loads such a library into the context and returns in *metric_id the value
 * to put in prr_frame_desc.metric (PRR_METRIC_PLUGIN0 + k).  Plug-in frames
 * render in either mode through the header's hooks, then the header's
 * rayToRGB, then the usual SSAA combine / FXAA / quantisation:
 *   REFERENCE - the solver of kernels/solver.cuh (one thread per ray);
 *   PHYSICAL  - FP32 only (a header's getGeod computes in FP32): the
 *               persistent warp-compacted scheduler with PHYSICAL semantics
 *               (textbook stages, null initial data from the header's
 *               getMetric, atol/rtol control, Kahan-compensated state,
 *               max_steps) and the header's User_UPDATE / User_ENDLOOP
 *               deciding hits and termination as in trace_RKF.
 * A call's frames are all plug-in frames or all built-in ones; plug-in
 * frames take no emission, no FP64/SPLIT and no recorded graph.  The
 * Spacetime the hooks see carries mass, spin (prr_frame_desc.spin, for any
 * plug-in) and the frame's spheres.  Loading the same path twice returns the
 * same id; libraries stay loaded until the process exits. */
#define PRR_METRIC_PLUGIN0 16
#define PRR_MAX_PLUGINS 8
prr_status prr_load_metric_plugin(prr_ctx *ctx, const char *path, int *metric_id);

/* ---- scheduler tuning (new) ---- */
prr_status prr_set_schedule(prr_ctx *ctx, int schedule, const prr_launch_config *cfg);
prr_status prr_get_launch_config(prr_ctx *ctx, prr_launch_config *cfg);
/* Times candidate launch shapes on `frame` and keeps the fastest. */
prr_status prr_autotune(prr_ctx *ctx, const prr_frame_desc *frame, prr_launch_config *best);

/* Context options (values for prr_set_option). */
#define PRR_OPT_GEOD_TABLE 1      /* geodesic form: -1 (default) PERSISTENT uses the register contraction and
                                     PLAIN the Christoffel table; 0: contraction everywhere; 1: table
                                     everywhere (A/B runs) */
#define PRR_OPT_WATCHDOG_CYCLES 2 /* >0: persistent kernels stop after this many SM clock cycles and the
                                     call returns PRR_ERR_TIMEOUT; 0: off (default) */
#define PRR_OPT_HAMILTONIAN 3     /* which PHYSICAL renders integrate (x, p) in Hamiltonian form (p_t
                                     conserved, six state components) instead of (x, u) with the geodesic
                                     contraction: a bit mask of PRR_HAM_FP32 (FP32 renders with one pixel
                                     per thread, emission frames and the FP32 pass of SPLIT included) and
                                     PRR_HAM_FP64 (FP64 renders); default both (3), 0 for neither.  Both
                                     forms use the same tableau, error test (over their own state), caps,
                                     hooks and colours; in the Hamiltonian form the coordinate time is not
                                     integrated, so r.w of prr_trace_rays(_f64) is 0 there.  PRR_HAM_FP64
                                     also covers the FP64 pass of SPLIT; the adjoint always steps (x, u) */
#define PRR_HAM_FP32 1
#define PRR_HAM_FP64 2
prr_status prr_set_option(prr_ctx *ctx, int option, long long value);

/* Measures FP32 and FP64 FMA throughput (TFLOP/s) of the context's device
 * with a dependent-chain FMA kernel; either pointer may be NULL. */
prr_status prr_measure_peak(prr_ctx *ctx, double *fp32_tflops, double *fp64_tflops);

/* Evaluates on the device the reciprocal and reciprocal square root that the
 * PHYSICAL-mode kernels use, for checking their error: for each of the n
 * inputs x[i] (1 <= n <= 2^20), out[4i .. 4i+3] = FP64 1/x, FP64 1/sqrt(x),
 * FP32 1/(float)x, FP32 1/sqrt((float)x) (the FP32 values widened). */
prr_status prr_check_recip(prr_ctx *ctx, const double *x, int n, double *out);

/* ---- input decks (replaces main/io.h:21-58 readParams, the getters of
 *      main/Parameters.cpp:20-44, checkFrame prr.cpp:139-153, createScene
 *      prr.cpp:159-198, Spacetime::setupScene/updateScene
 *      main/Spacetime.cpp:17-44 and renderframe's set-up prr.cpp:245-253).
 *      No GPU needed. ----
 * Decks are read with the reference's rules, quirks included: a line with
 * neither '_' nor '<' is skipped; ANY line containing '_' opens a block named
 * by the text between its first and last '_'; otherwise the key is the text
 * between the first '<' and '>' left of '=', the value the same right of it.
 * prr_deck_load also reads the decks named by tracer.traj and tracer.scene
 * (paths relative to the working directory; an unreadable one adds nothing,
 * as in the reference).  errbuf (errlen bytes) receives a message on failure
 * and may be NULL. */
typedef struct prr_deck prr_deck;
prr_status prr_deck_load(const char *path, prr_deck **out, char *errbuf, size_t errlen);
/* Same rules over an in-memory deck (no traj/scene files are followed). */
prr_status prr_deck_parse_string(const char *text, prr_deck **out);
void prr_deck_free(prr_deck *d);
/* headerExists / parExists (main/Parameters.cpp:10-18): 1 or 0. */
int prr_deck_has_block(const prr_deck *d, const char *block);
int prr_deck_has(const prr_deck *d, const char *block, const char *key);
/* par (main/Parameters.cpp:20-25): copies the value ("" when missing) into
 * buf (len bytes, NUL-terminated, may be NULL) and returns its length. */
size_t prr_deck_get(const prr_deck *d, const char *block, const char *key, char *buf, size_t len);
/* pari / parf (main/Parameters.cpp:26-44): std::stoi / std::stof of the
 * value; 0 (pari) or `dflt` (parf) when the key is missing or unparsable. */
int prr_deck_geti(const prr_deck *d, const char *block, const char *key);
float prr_deck_getf(const prr_deck *d, const char *block, const char *key, float dflt);
/* checkFrame (prr.cpp:139-153): the first i without all of frame<i>.x y z a b. */
int prr_deck_frame_count(const prr_deck *d);
/* Spheres in the scene: the first i without a sphere<i> block. */
int prr_deck_sphere_count(const prr_deck *d);
/* sphere<i>.tex into buf as prr_deck_get; returns its length. */
size_t prr_deck_sphere_texture(const prr_deck *d, int sphere, char *buf, size_t len);
/* The descriptor of frame `frame`: camera, spacetime and tracer from their
 * blocks; sphere<i> centres and radii after updateScene(0..frame), a key the
 * deck lacks keeping the previous frame's value; frame<i>.mass overriding
 * the mass from that frame on.  Angles in degrees are converted as the
 * reference does (float(deg * M_PI / 180.0f)).  Texture ids: 0 = the sky
 * (tracer.bimage1), 1, 2, ... = distinct sphere textures in sphere order,
 * -1 = none.  Deck keys the reference lacks, all optional with defaults that
 * reproduce it: spacetime.metric (flat|schwarzschild|kerr, or the path of a
 * metric plug-in library "*.so", for which the descriptor's metric is
 * PRR_METRIC_PLUGIN0 until the caller puts the id prr_load_metric_plugin
 * returned - prr_run_deck does; schwarzschild by default, as main/metric.h:12
 * selects; no black hole = flat), tracer.mode
 * (reference|physical), tracer.precision (fp32|fp64|split), tracer.rtol and
 * tracer.atol (eps), tracer.maxsteps (10000), tracer.horizon (0.001, as
 * metrics/schwarzschild.cuh:70), tracer.fxaa (0), tracer.bgfilter
 * (rms2x2|bilinear), camera.model (spherical|pinhole|panorama), camera.seed
 * (RANDOM/JITTERED offsets).  SSAA random and jittered map to the PHYSICAL-
 * mode placements of prr_ssaa.  Solvers rk/adams/gragg/dormand/taylor and
 * SSAA poisson/rotated have no implementation (in the reference either) and
 * return PRR_ERR_UNSUPPORTED; unknown names fall back to euler and regular
 * as Parameters::getSolver/getSSAA do. */
prr_status prr_deck_frame(const prr_deck *d, int frame, prr_frame_desc *out, char *errbuf, size_t errlen);

/* The reference's main (prr.cpp:345-404): loads the deck at `path`, uploads
 * the textures it names (prr_image_load), renders frames [first,
 * first+count) (count < 0: to the last) in batches of `batch` frames per
 * prr_render call (< 1: 16), and writes each as <prefix>image_<i>.png, the
 * reference's name (prr.cpp:336); prefix NULL = tracer.out.  Texture ids 0 ..
 * are (re)uploaded on the context.  stats (may be NULL) sums the calls. */
prr_status prr_run_deck(prr_ctx *ctx, const char *path, int first, int count, const char *prefix, int batch,
                        prr_stats *stats);

/* ---- image files (replaces cudamaths/image.cu:13-39) ----
 * prr_image_load decodes PNG (1/2/4/8/16-bit grey, grey+alpha, RGB, RGBA,
 * palette; interlaced or not) and binary PNM (P6, P5; maxval <= 255) to
 * RGBA8 (*rgba8 from malloc; free with prr_image_free), with stb_image's
 * channel rules: grey replicated to RGB, 16-bit samples keep their high
 * byte, low-bit grey scaled to 0..255.  JPEG returns PRR_ERR_UNSUPPORTED.
 * prr_png_write writes 8-bit RGB rows (3*w bytes each) as a PNG file. */
prr_status prr_image_load(const char *path, uint8_t **rgba8, int *w, int *h, char *errbuf, size_t errlen);
void prr_image_free(uint8_t *rgba8);
prr_status prr_png_write(const char *path, const uint8_t *rgb8, int w, int h);

/* ---- host helpers (no GPU needed) ---- */
/* Seeded procedural RGBA8 textures.  kind 0: sphere texture (checkerboard +
 * value noise); kind 1: equirectangular starfield (Poisson point stars with
 * log-normal brightness on a dark gradient). */
prr_status prr_make_texture(int kind, uint32_t seed, int w, int h, uint8_t *out_rgba8);
/* Fills `d` with the defaults used where a deck is silent. */
void prr_frame_desc_defaults(prr_frame_desc *d);
/* sizeof of the ABI structs, for binding checks: 0 prr_frame_desc,
 * 1 prr_stats, 2 prr_launch_config, 3 prr_sphere, 4 prr_emission_desc,
 * 5 prr_plasma_desc; 0 for other values. */
size_t prr_sizeof(int which);

#ifdef __cplusplus
}
#endif
#endif /* PRR_H */
