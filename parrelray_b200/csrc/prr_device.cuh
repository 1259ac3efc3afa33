// prr_device.cuh - device-side building blocks shared by every kernel:
// small vector types, the per-frame parameter block, RGBA8 texture access,
// the metrics, the sphere hit test and the background lookup.
//
// Reference correspondence (paths relative to the reference project):
//   Camera::rayDir_Spherical      main/Camera.h:39-42
//   createRays_none / _regular    kernels/ssaa.cuh:92-99, 36-48
//   initRays                      kernels/solver.cuh:26-56
//   getGeod / getMetric (Schw.)   metrics/schwarzschild.cuh:90-141
//   Sphere::intersects/getColor   scene/sphere.h:34-64
//   Spacetime::IntersectsScene    main/Spacetime.h:38-46
//   tex2d::operator[]             cudamaths/tex2d.cuh:112-131
//   OutSphere::getColorDefault2   main/base.h:119-162
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "prr.h"

#define PRR_DEV __device__ __forceinline__
#define PRR_HD __host__ __device__ __forceinline__

namespace prr {

constexpr double PI_BASE = 3.14159265358979323846;  // main/base.h:20
constexpr double PI_SPHERE = 3.14159265359;          // scene/sphere.h:16 (redefines PI)

template <class T> struct V3 { T x, y, z; };
template <class T> struct V4 { T x, y, z, w; };

// Reciprocal, reciprocal square root and power for the PHYSICAL-mode hot
// loop.  FP32 issues the SFU approximations directly (PTX rcp.approx.ftz,
// rsqrt.approx.ftz, lg2.approx.ftz and ex2.approx.ftz: relative errors of
// about 2^-23, far below the 1e-6 integration tolerance), with subnormal
// inputs and results flushed to zero, so no range or subnormal fix-up
// instructions surround them; the arguments on this path (squared radii,
// norms, error ratios) are normal numbers or 0.  FP64 starts from the SFU's
// double-precision seeds (PTX rcp.approx.ftz.f64 / rsqrt.approx.ftz.f64, good
// to about 2^-22) and refines them with two Newton-Raphson steps on DFMA
// (x <- x + x (1 - v x) for 1/v; y <- y + y (1/2 - (v/2) y^2) for 1/sqrt(v);
// each step doubles the correct bits, Markstein's formulation of the
// iterations with a fused multiply-add), to within an ulp or two of the
// correctly rounded values, for normal positive arguments.
PRR_DEV float sfu_rcp(float v) { float r; asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(v)); return r; }
PRR_DEV float sfu_rsqrt(float v) { float r; asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(v)); return r; }
PRR_DEV float sfu_lg2(float v) { float r; asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(v)); return r; }
PRR_DEV float sfu_ex2(float v) { float r; asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(v)); return r; }
PRR_DEV double nr_rcp(double v)
{
    double x;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(x) : "d"(v));
    double e = __fma_rn(-v, x, 1.0);
    x = __fma_rn(x, e, x);
    e = __fma_rn(-v, x, 1.0);
    return __fma_rn(x, e, x);
}
PRR_DEV double nr_rsqrt(double v)
{
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(v));
    const double hv = 0.5 * v;
    double r = __fma_rn(-hv * y, y, 0.5);
    y = __fma_rn(y, r, y);
    r = __fma_rn(-hv * y, y, 0.5);
    return __fma_rn(y, r, y);
}
template <class T> PRR_DEV T frcp(T v) { return (T)1 / v; }
template <> PRR_DEV float frcp<float>(float v) { return sfu_rcp(v); }
template <> PRR_DEV double frcp<double>(double v) { return nr_rcp(v); }
template <class T> PRR_DEV T frsqrt(T v) { return (T)1 / sqrt(v); }
template <> PRR_DEV float frsqrt<float>(float v) { return sfu_rsqrt(v); }
template <> PRR_DEV double frsqrt<double>(double v) { return nr_rsqrt(v); }
template <class T> PRR_DEV T fpow(T b, T e) { return pow(b, e); }
template <> PRR_DEV float fpow<float>(float b, float e) { return sfu_ex2(e * sfu_lg2(b)); }

template <class T> PRR_HD V4<T> v4add(const V4<T> &a, const V4<T> &b) { return {a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }
// f4 scaled by t; the reference's operator*(float, f4) multiplies each
// component by t (cudamaths/f4.cuh:52).
template <class T> PRR_HD V4<T> v4scl(T t, const V4<T> &a) { return {a.x * t, a.y * t, a.z * t, a.w * t}; }

// ------------------------------------------------------------- textures

struct DevTex {
    const uint32_t *p;  // RGBA8 texels, row-major
    int w, h;
};

// Texel as the reference stores it: byte/255 in FP32 (cudamaths/image.cu:15
// loads with gamma 1, so texel = byte/255.0f exactly).
template <class T> PRR_DEV V3<T> texel(const DevTex &t, int i, int j)
{
    uint32_t v = __ldg(t.p + (size_t)j * t.w + i);
    float r = (float)(v & 255u) / 255.0f, g = (float)((v >> 8) & 255u) / 255.0f, b = (float)((v >> 16) & 255u) / 255.0f;
    return {(T)r, (T)g, (T)b};
}

// tex2d::operator[](i2): index clamped to [0, res-1].
template <class T> PRR_DEV V3<T> tex_at(const DevTex &t, int i, int j)
{
    i = min(max(i, 0), t.w - 1);
    j = min(max(j, 0), t.h - 1);
    return texel<T>(t, i, j);
}

// tex2d::operator[](f2): bilinear, cell clamped to [0, res-2] after the
// fraction is taken (edge extrapolation quirk kept).
template <class T> PRR_DEV V3<T> tex_bilinear(const DevTex &t, T u, T v)
{
    T ux = u * (T)t.w, uy = v * (T)t.h;
    int ix = (int)floor(ux), iy = (int)floor(uy);
    T px = ux - (T)ix, py = uy - (T)iy;
    ix = min(max(ix, 0), t.w - 2);
    iy = min(max(iy, 0), t.h - 2);
    V3<T> a = texel<T>(t, ix, iy), b = texel<T>(t, ix + 1, iy), c = texel<T>(t, ix, iy + 1), d = texel<T>(t, ix + 1, iy + 1);
    const T one = (T)1;
    V3<T> r;
    r.x = a.x * (one - px) * (one - py) + b.x * px * (one - py) + c.x * (one - px) * py + d.x * px * py;
    r.y = a.y * (one - px) * (one - py) + b.y * px * (one - py) + c.y * (one - px) * py + d.y * px * py;
    r.z = a.z * (one - px) * (one - py) + b.z * px * (one - py) + c.z * (one - px) * py + d.z * px * py;
    return r;
}

// ------------------------------------------------------------- frame block

struct DevSphere {
    float cx, cy, cz, r;
    DevTex tex;  // tex.p == nullptr: untextured (grey 0.5)
    float far2;  // squared distance beyond which no hit test can pass (PHYSICAL-mode early out)
    float far;   // sqrt(far2)
};

// Everything a kernel needs about one frame, prepared on the host from a
// prr_frame_desc.
// The plasma grid of prr_upload_plasma on the device (nodes x-fastest).
struct DevPlasma {
    const float *n;       // density
    const float *theta;   // temperature (nullptr: 1)
    const float4 *vel;    // coordinate velocity (vx, vy, vz, 0) (nullptr: the DISK flow)
    int nx, ny, nz;
    float lo[3], inv[3];  // box corner and (n - 1) / (hi - lo) per axis
};

// prr_emission_desc plus the grid, for one frame.
struct EmisParams {
    int kind;             // prr_emission
    int sense, cmap;
    float index, height, r_in, r_out, spectral, absorb, gain, temp_power;
    DevPlasma grid;
};

struct FrameParams {
    int width, height, samples, ssaa, nsub;
    float vfov, cam[3], alpha, beta;
    int metric;
    float M, a, rs;
    float rstop;    // terminate at r <= rstop (horizon + horizon_eps)
    float rblack;   // reference colour rule: SUCCESS with r <= rblack is black
    int solver, mode, precision;
    float h, hmin, hmax, eps, rtol, atol, rout;
    int max_steps;
    int bg_filter, fxaa;
    DevTex bg;      // bg.p == nullptr: black sky
    float fp64_delta, fp64_rfac;
    int nspheres;
    // every sphere is far (sphere_far) from a point p with |p|^2 outside
    // [sph_lo2, sph_hi2] (Euclidean |p|; empty when there are no spheres)
    float sph_lo2, sph_hi2;
    int camera;           // prr_camera
    unsigned ssaa_seed;   // RANDOM / JITTERED offsets
    float cfwd[3], cright[3], cup[3];  // Camera::computeVectors basis (PINHOLE, PANORAMA)
    float tan_half;       // tanf(vfov / 2) (PINHOLE)
    EmisParams em;        // em.kind == PRR_EMISSION_NONE: no plasma
    DevSphere sph[PRR_MAX_SPHERES];
    long long ray_begin;  // first ray (work) index of this frame in a batch
    long long pix_begin;  // first output pixel of this frame in a batch
};

// ------------------------------------------------------------- camera / rays

// Counter-based hash for stochastic sample placement: the PCG output
// permutation applied to an LCG step of the input ("pcg_hash", Jarzynski &
// Olano, "Hash Functions for GPU Rendering", JCGT 2020).
PRR_HD uint32_t pcg_hash(uint32_t v)
{
    uint32_t state = v * 747796405u + 2891336453u;
    uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
    return (word >> 22u) ^ word;
}

// Two uniforms in [0, 1) for sample s of pixel p (24-bit mantissas).
PRR_HD void sample_offsets(uint32_t seed, long long p, int s, float &r0, float &r1)
{
    uint32_t h = pcg_hash(seed ^ pcg_hash((uint32_t)p ^ pcg_hash((uint32_t)(p >> 32) + 0x9e3779b9u * (uint32_t)(s + 1))));
    uint32_t g = pcg_hash(h);
    r0 = (float)(h >> 8) * (1.0f / 16777216.0f);
    r1 = (float)(g >> 8) * (1.0f / 16777216.0f);
}

// Sub-pixel position of ray `s` of pixel (x, y): createRays_none/regular
// (kernels/ssaa.cuh:92-99, 36-48), and the RANDOM / JITTERED placements.
PRR_DEV void ray_uv(const FrameParams &fp, int x, int y, int s, float &uvx, float &uvy)
{
    if (fp.ssaa == PRR_SSAA_NONE) {
        uvx = (float)x / fp.width + (1.0f / fp.width) * 0.5f;
        uvy = (float)y / fp.height + (1.0f / fp.height) * 0.5f;
    } else if (fp.ssaa == PRR_SSAA_REGULAR) {
        int n = fp.nsub;
        float dux = (1.0f / fp.width) / (n + 1.0f), duy = (1.0f / fp.height) / (n + 1.0f);
        int i = s % n, j = s / n;
        uvx = (float)x / fp.width + (float)(i + 1) * dux;
        uvy = (float)y / fp.height + (float)(j + 1) * duy;
    } else {
        float r0, r1;
        sample_offsets(fp.ssaa_seed, (long long)y * fp.width + x, s, r0, r1);
        if (fp.ssaa == PRR_SSAA_JITTERED) {
            const int n = fp.nsub;
            r0 = ((float)(s % n) + r0) / (float)n;
            r1 = ((float)(s / n) + r1) / (float)n;
        }
        uvx = ((float)x + r0) / (float)fp.width;
        uvy = ((float)y + r1) / (float)fp.height;
    }
}

// Ray direction for the screen position (uvx, uvy): Camera::rayDir_Spherical
// (main/Camera.h:39-42, FP32 as in the reference), rayDir_PinHole (30-33) and
// the equirectangular panorama (34-37, see prr_camera).
PRR_DEV V3<float> ray_dir(const FrameParams &fp, float uvx, float uvy)
{
    V3<float> v;
    if (fp.camera == PRR_CAMERA_PINHOLE) {
        const float sx = (2.0f * uvx - 1.0f) * fp.tan_half * (float)fp.width / (float)fp.height;
        const float sy = (1.0f - 2.0f * uvy) * fp.tan_half;
        v = {fp.cfwd[0] + sx * fp.cright[0] + sy * fp.cup[0], fp.cfwd[1] + sx * fp.cright[1] + sy * fp.cup[1],
             fp.cfwd[2] + sx * fp.cright[2] + sy * fp.cup[2]};
    } else if (fp.camera == PRR_CAMERA_PANORAMA) {
        const float mu = (0.5f - uvy) * fp.vfov;
        const float nu = (uvx - 0.5f) * (float)fp.width / (float)fp.height * fp.vfov;
        const float cm = cosf(mu), a = cm * cosf(nu), b = cm * sinf(nu), c = sinf(mu);
        v = {a * fp.cfwd[0] + b * fp.cright[0] + c * fp.cup[0], a * fp.cfwd[1] + b * fp.cright[1] + c * fp.cup[1],
             a * fp.cfwd[2] + b * fp.cright[2] + c * fp.cup[2]};
    } else {
        float nu = (0.5f - uvy) * fp.vfov;
        float mu = (0.5f - uvx) * (float)fp.width / (float)fp.height * fp.vfov;
        float cb = cosf(fp.beta + nu);
        v = {cb * cosf(fp.alpha + mu), cb * sinf(fp.alpha + mu), sinf(fp.beta + nu)};
    }
    float k = 1.0f / sqrtf(v.x * v.x + v.y * v.y + v.z * v.z);
    return {v.x * k, v.y * k, v.z * k};
}

// ------------------------------------------------------------- metrics

template <class T> PRR_DEV T ks_radius(T x, T y, T z, T a)
{
    T R2 = x * x + y * y + z * z;
    T b = R2 - a * a;
    T S = sqrt(b * b + (T)4 * a * a * z * z);
    return sqrt((T)0.5 * (b + S));
}

template <class T> PRR_HD T kerr_r_plus(T M, T a)
{
    T d = M * M - a * a;
    return M + sqrt(d > (T)0 ? d : (T)0);
}

// Radius used by the termination and colour rules: |x| for flat and
// Schwarzschild (metrics/schwarzschild.cuh:68), Kerr-Schild r for Kerr.
template <class T> PRR_DEV T metric_radius(const FrameParams &fp, T x, T y, T z)
{
    if (fp.metric == PRR_METRIC_KERR) return ks_radius<T>(x, y, z, (T)fp.a);
    return sqrt(x * x + y * y + z * z);
}

// metrics/schwarzschild.cuh:123-141 (FP32 order).
PRR_DEV void metric_schw_ref(float px, float py, float pz, float rs, float g[16])
{
    float ir = 1.0f / sqrtf(px * px + py * py + pz * pz);
    float ir2 = ir * ir, ir3 = ir2 * ir;
    g[0] = 1.0f + rs * px * px * ir3; g[1] = rs * px * py * ir3; g[2] = rs * px * pz * ir3; g[3] = rs * px * ir2;
    g[4] = g[1]; g[5] = 1.0f + rs * py * py * ir3; g[6] = rs * py * pz * ir3; g[7] = rs * py * ir2;
    g[8] = g[2]; g[9] = g[6]; g[10] = 1 + rs * pz * pz * ir3; g[11] = rs * pz * ir2;
    g[12] = g[3]; g[13] = g[7]; g[14] = g[11]; g[15] = -1 + rs * ir;
}

// Kerr-Schild g = eta + f l l, (x, y, z, t) order (flat: M = 0).
template <class T> PRR_DEV void metric_ks(T px, T py, T pz, T M, T a, T g[16])
{
    T f = 0, l[4] = {0, 0, 0, 1};
    if (M != (T)0) {
        T r = ks_radius<T>(px, py, pz, a), r2 = r * r, q = r2 + a * a;
        f = (T)2 * M * r2 * r / (r2 * r2 + a * a * pz * pz);
        l[0] = (r * px + a * py) / q; l[1] = (r * py - a * px) / q; l[2] = pz / r;
    }
#pragma unroll
    for (int m = 0; m < 4; m++)
#pragma unroll
        for (int n = 0; n < 4; n++) g[m * 4 + n] = (m == n ? (m == 3 ? (T)-1 : (T)1) : (T)0) + f * l[m] * l[n];
}

// metrics/schwarzschild.cuh:90-119 in the reference's FP32 operation order.
PRR_DEV V4<float> geod_schw_ref(const V4<float> &p, const V4<float> &u, float rs)
{
    V4<float> du;
    float r = sqrtf(p.x * p.x + p.y * p.y + p.z * p.z);
    float x2 = p.x * p.x, y2 = p.y * p.y, z2 = p.z * p.z;
    float Phi = (r * (x2 - 2.0f * y2 - 2.0f * z2) + rs * x2) * u.x * u.x
              + (r * (-2.0f * x2 + y2 - 2.0f * z2) + rs * y2) * u.y * u.y
              + (r * (-2.0f * x2 - 2.0f * y2 + z2) + rs * z2) * u.z * u.z
              + 2.0f * (3.0f * r + rs) * (p.x * p.y * u.x * u.y + p.x * p.z * u.x * u.z + p.y * p.z * u.y * u.z)
              + r * r * (rs - r) * u.w * u.w + 2.0f * r * rs * u.w * (p.x * u.x + p.y * u.y + p.z * u.z);
    Phi *= rs / (2.0f * powf(r, 6.0f));
    du.x = p.x * Phi;
    du.y = p.y * Phi;
    du.z = p.z * Phi;
    du.w = (2.0f * r * (-x2 + y2 + z2) - rs * x2) * u.x * u.x
         + (2.0f * r * (x2 - y2 + z2) - rs * y2) * u.y * u.y
         + (2.0f * r * (x2 + y2 - z2) - rs * z2) * u.z * u.z
         - 2.0f * (4.0f * r + rs) * (p.x * p.y * u.x * u.y + p.x * p.z * u.x * u.z + p.y * p.z * u.y * u.z)
         - r * r * rs * u.w * u.w - 2.0f * r * (r + rs) * u.w * (p.x * u.x + p.y * u.y + p.z * u.z);
    du.w *= rs / (2.0f * powf(r, 5.0f));
    return du;
}

// Geodesic acceleration du/dlambda = -Gamma^k_{mn} u^m u^n for the
// Kerr-Schild metric g = eta + f l(x)l, evaluated WITHOUT forming the
// Christoffel table.  With L = l.u, D = u^k d_k (d_t = 0):
//   G_m = Gamma_{m ab} u^a u^b = l_m (L Df + f DL) + f L D(l_m)
//                                - 1/2 L^2 d_m f - f L d_m(L)|_u
//   du^k = -g^{km} G_m,  g^{km} = eta^{km} - f l^k l^m  (l^k = eta^{kk} l_k)
// All quantities are scalars or 3-vectors held in registers.  Cost is about
// 110 FP32 operations + 2 sqrt + 4 divisions (vs. ~1000 for the table).
// FAST selects the SFU reciprocal / rsqrt forms (PHYSICAL mode); the
// REFERENCE-mode Kerr path keeps IEEE division and square root.
#ifdef PRR_GEOD_NOINLINE
#define PRR_GEOD_FN __device__ __noinline__
#else
#define PRR_GEOD_FN PRR_DEV
#endif
template <class T, bool FAST = false> PRR_GEOD_FN V4<T> geod_ks(const V4<T> &p, const V4<T> &u, T M, T a)
{
    const T X = p.x, Y = p.y, Z = p.z;
    const T a2 = a * a;
    const T R2 = X * X + Y * Y + Z * Z;
    const T b = R2 - a2;
    const T S2 = b * b + (T)4 * a2 * Z * Z;
    T S, iS, r2, r, ir;
    if (FAST) {
        iS = frsqrt<T>(S2);
        S = S2 * iS;
        r2 = (T)0.5 * (b + S);
        ir = frsqrt<T>(r2);
        r = r2 * ir;
    } else {
        S = sqrt(S2);
        iS = (T)1 / S;
        r2 = (T)0.5 * (b + S);
        r = sqrt(r2);
        ir = (T)1 / r;
    }
    const T q = r2 + a2, iq = FAST ? frcp<T>(q) : (T)1 / q;
    const T Sig = r2 * r2 + a2 * Z * Z, iSig = FAST ? frcp<T>(Sig) : (T)1 / Sig;
    // radius gradient
    const T rS = r * iS;
    const T drx = X * rS, dry = Y * rS, drz = Z * q * iS * ir;
    // f and its gradient
    const T f = (T)2 * M * r2 * r * iSig;
    const T c1 = f * ((T)3 * ir - (T)4 * r2 * r * iSig);
    const T dfx = c1 * drx, dfy = c1 * dry, dfz = c1 * drz - (T)2 * f * a2 * Z * iSig;
    // null vector l (l_t = 1)
    const T lx = (r * X + a * Y) * iq, ly = (r * Y - a * X) * iq, lz = Z * ir;
    // directional derivatives along the spatial velocity
    const T ux = u.x, uy = u.y, uz = u.z, ut = u.w;
    const T Dr = ux * drx + uy * dry + uz * drz;
    const T Dq = (T)2 * r * Dr;
    const T Dlx = (Dr * X + r * ux + a * uy - lx * Dq) * iq;
    const T Dly = (Dr * Y + r * uy - a * ux - ly * Dq) * iq;
    const T Dlz = (uz - lz * Dr) * ir;
    const T Df = ux * dfx + uy * dfy + uz * dfz;
    const T L = lx * ux + ly * uy + lz * uz + ut;
    const T DL = ux * Dlx + uy * Dly + uz * Dlz;
    // gradient of L at fixed u
    const T P = (ux * X + uy * Y - (T)2 * r * (ux * lx + uy * ly)) * iq - uz * lz * ir;
    const T dLx = drx * P + (r * ux - a * uy) * iq;
    const T dLy = dry * P + (a * ux + r * uy) * iq;
    const T dLz = drz * P + uz * ir;
    // lowered contraction, then raise with g^{-1}
    const T A = L * Df + f * DL;
    const T fL = f * L, hL2 = (T)0.5 * L * L;
    const T Gx = lx * A + fL * Dlx - hL2 * dfx - fL * dLx;
    const T Gy = ly * A + fL * Dly - hL2 * dfy - fL * dLy;
    const T Gz = lz * A + fL * Dlz - hL2 * dfz - fL * dLz;
    const T Gt = A;
    const T Lam = lx * Gx + ly * Gy + lz * Gz - Gt;
    const T fLam = f * Lam;
    return {fLam * lx - Gx, fLam * ly - Gy, fLam * lz - Gz, Gt - fLam};
}

// ------------------------------------------------------------- scene

struct Hit {
    bool hit;
    float r, g, b;
};

// Sphere::intersects (scene/sphere.h:34-50) for every sphere, closest hit by
// the reference's distance d (Spacetime::IntersectsScene), colour from
// Sphere::getColor (sphere.h:59-64).  The factor 2 in d and the acceptance
// window d*d <= |v|^2 h are the reference's.
template <class T> PRR_DEV Hit intersect_scene(const FrameParams &fp, T px, T py, T pz, T vx, T vy, T vz, T h)
{
    Hit out;
    out.hit = false;
    out.r = out.g = out.b = -1.0f;
    if (fp.nspheres == 0) return out;
    T k = (T)1 / sqrt(vx * vx + vy * vy + vz * vz);
    vx *= k; vy *= k; vz *= k;
    T best = (T)100000000000.0;
    for (int s = 0; s < fp.nspheres; s++) {
        const DevSphere &S = fp.sph[s];
        T cx = (T)S.cx, cy = (T)S.cy, cz = (T)S.cz, rad = (T)S.r;
        T v2 = vx * vx + vy * vy + vz * vz;
        T dx = px - cx, dy = py - cy, dz = pz - cz;
        T dvp = vx * dx + vy * dy + vz * dz;
        T disc = dvp * dvp - v2 * ((dx * dx + dy * dy + dz * dz) - rad * rad);
        if (disc < (T)0) continue;
        T d = ((T)-2.0f * dvp - sqrt(disc)) / v2;
        if (d * d > v2 * h) continue;
        if (d < (T)0) continue;
        T ix = (px + vx * d) - cx, iy = (py + vy * d) - cy, iz = (pz + vz * d) - cz;
        T theta = acos(iz / rad);
        T phi = (T)((double)atan2(iy, ix) + PI_SPHERE);
        T uu = (T)((double)phi / (2.0 * PI_SPHERE)), vv = (T)((double)theta / PI_SPHERE);
        const T uvmax = (T)0.999999999f;
        uu = fmin(fmax(uu, (T)0), uvmax);
        vv = fmin(fmax(vv, (T)0), uvmax);
        V3<T> col = {(T)0.5, (T)0.5, (T)0.5};
        if (S.tex.p) col = tex_bilinear<T>(S.tex, uu, vv);
        T shade = fmax((T)0, fmin((T)0.5 + (T)0.5 * iz / rad, (T)1));
        col.x *= shade; col.y *= shade; col.z *= shade;
        if (col.x >= (T)0 && d <= best) {
            best = d;
            out.hit = true;
            out.r = (float)col.x; out.g = (float)col.y; out.b = (float)col.z;
        }
    }
    return out;
}

// OutSphere::getColorDefault2: RMS of the 2x2 block at floor(uv).
template <class T> PRR_DEV V3<float> background_rms(const DevTex &t, T ux_, T uy_, T uz_)
{
    T k = (T)1 / sqrt(ux_ * ux_ + uy_ * uy_ + uz_ * uz_);
    T nx = ux_ * k, ny = uy_ * k, nz = uz_ * k;
    T theta = acos(nz);
    T phi = atan2(ny, nx);
    phi = (phi >= (T)0 ? phi : (T)((double)phi + 2.0 * PI_BASE));
    if ((double)phi > 2.0 * PI_BASE || phi < (T)0) return {0.5f, 0.5f, 0.0f};
    if (theta < (T)0 || (double)theta > PI_BASE) return {0.0f, 0.5f, 0.8f};
    T fx = (T)((double)phi / (2.0 * PI_BASE) * t.w), fy = (T)((double)theta / PI_BASE * t.h);
    int px = (int)floor(fx), py = (int)floor(fy);
    if (px == t.w) px -= 1;
    if (py == t.h) py -= 1;
    if (px < 0 || px >= t.w || py < 0 || py >= t.h) return {0.0f, 0.5f, 0.0f};
    if (px == t.w - 1 || py == t.h - 1) return tex_at<float>(t, px, py);
    V3<float> a = tex_at<float>(t, px, py), b = tex_at<float>(t, px, py + 1);
    V3<float> c = tex_at<float>(t, px + 1, py), d = tex_at<float>(t, px + 1, py + 1);
    return {sqrtf(0.25f * (a.x * a.x + b.x * b.x + c.x * c.x + d.x * d.x)),
            sqrtf(0.25f * (a.y * a.y + b.y * b.y + c.y * c.y + d.y * d.y)),
            sqrtf(0.25f * (a.z * a.z + b.z * b.z + c.z * c.z + d.z * d.z))};
}

// Continuous background (PRR_BG_BILINEAR): bilinear over texel centres,
// wrapping in longitude, clamped in latitude.
template <class T> PRR_DEV V3<T> background_bilinear(const DevTex &t, T ux_, T uy_, T uz_)
{
    T k = (T)1 / sqrt(ux_ * ux_ + uy_ * uy_ + uz_ * uz_);
    T nz = fmin(fmax(uz_ * k, (T)-1), (T)1);
    T theta = acos(nz);
    T phi = atan2(uy_, ux_);
    if (phi < (T)0) phi += (T)(2.0 * PI_BASE);
    T fx = phi / (T)(2.0 * PI_BASE) * (T)t.w - (T)0.5, fy = theta / (T)PI_BASE * (T)t.h - (T)0.5;
    T flx = floor(fx), fly = floor(fy);
    T wx = fx - flx, wy = fy - fly;
    int x0 = (int)flx, y0 = (int)fly;
    int x1 = x0 + 1, y1 = y0 + 1;
    x0 = ((x0 % t.w) + t.w) % t.w; x1 = ((x1 % t.w) + t.w) % t.w;
    y0 = min(max(y0, 0), t.h - 1); y1 = min(max(y1, 0), t.h - 1);
    V3<T> a = texel<T>(t, x0, y0), b = texel<T>(t, x1, y0), c = texel<T>(t, x0, y1), d = texel<T>(t, x1, y1);
    T w00 = ((T)1 - wx) * ((T)1 - wy), w10 = wx * ((T)1 - wy), w01 = ((T)1 - wx) * wy, w11 = wx * wy;
    return {a.x * w00 + b.x * w10 + c.x * w01 + d.x * w11, a.y * w00 + b.y * w10 + c.y * w01 + d.y * w11,
            a.z * w00 + b.z * w10 + c.z * w01 + d.z * w11};
}

// Final colour of a terminated ray (rayToRGB, metrics/schwarzschild.cuh:151-183).
// REFERENCE mode keeps the reference's rule (a SUCCESS ray between rblack and
// rout keeps its velocity as colour); PHYSICAL mode blacks every captured ray.
template <class T> PRR_DEV V3<float> ray_colour(const FrameParams &fp, int result, const V4<T> &x, const V4<T> &u)
{
    V3<float> c = {(float)u.x, (float)u.y, (float)u.z};
    if (result == PRR_RESULT_SUCCESS) {
        T r = metric_radius<T>(fp, x.x, x.y, x.z);
        bool black;
        if (fp.mode == PRR_MODE_REFERENCE) black = fp.metric != PRR_METRIC_FLAT && r <= (T)fp.rblack;
        else black = r < (T)fp.rout;
        if (black) return {0.0f, 0.0f, 0.0f};
        if (r >= (T)fp.rout) {
            if (!fp.bg.p) return {0.0f, 0.0f, 0.0f};
            if (fp.bg_filter == PRR_BG_BILINEAR) {
                V3<T> b = background_bilinear<T>(fp.bg, u.x, u.y, u.z);
                return {(float)b.x, (float)b.y, (float)b.z};
            }
            return background_rms<T>(fp.bg, u.x, u.y, u.z);
        }
        return c;
    }
    if (result == PRR_RESULT_INTERSECTION) return c;
    return {0.0f, 0.0f, 0.0f};
}

}  // namespace prr
