// k_plain.cu - the PLAIN schedule: the reference's pipeline structure
// (prr.cpp:258-332) with PHYSICAL-mode arithmetic, the "plain
// one-ray-per-thread form" the persistent renderer is measured against.
//   createRays (ssaa.cuh:36-48/92-99) -> initRays (solver.cuh:26-56)
//   -> trace in 64-row layers (prr.cpp:289-309, solver.cuh:142-219)
//   -> rayToRGB (schwarzschild.cuh:151-183) -> combineSamples -> FXAA
// Rays live in HBM as 48-byte records like the reference's Ray
// (base.h:172-176), 8x8 thread blocks, one kernel per stage.  The RKF45
// stages are the textbook ones (both kx and ku kept), the geodesic is the
// Christoffel-table form (or the contraction, for A/B runs), and each
// accepted step runs the two sphere tests separately, as the hooks do.
#include "kernels.cuh"
#include "phys_stepper.cuh"

namespace prr {

struct PlainRay {
    float uvx, uvy;
    int result;
    float r[4], u[4];
    float I;
};
static_assert(sizeof(PlainRay) == 48, "ray record must be 48 bytes");

size_t plain_ray_record_bytes() { return sizeof(PlainRay); }

__global__ void k_plain_create(const FrameParams *__restrict__ fps, int frame, PlainRay *rays)
{
    const FrameParams &fp = fps[frame];
    int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= fp.width || y >= fp.height) return;
    for (int s = 0; s < fp.samples; s++) {
        PlainRay &R = rays[((size_t)y * fp.width + x) * fp.samples + s];
        ray_uv(fp, x, y, s, R.uvx, R.uvy);
    }
}

__global__ void k_plain_init(const FrameParams *__restrict__ fps, int frame, PlainRay *rays)
{
    const FrameParams &fp = fps[frame];
    int ix = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix >= fp.width * fp.samples || y >= fp.height) return;
    PlainRay &R = rays[(size_t)y * fp.width * fp.samples + ix];
    V3<float> dir = ray_dir(fp, R.uvx, R.uvy);
    float g[16];
    metric_ks<float>(fp.cam[0], fp.cam[1], fp.cam[2], fp.metric == PRR_METRIC_FLAT ? 0.f : fp.M,
                     fp.metric == PRR_METRIC_KERR ? fp.a : 0.f, g);
    float a = g[15], b = 2.0f * (g[12] * dir.x + g[13] * dir.y + g[14] * dir.z);
    float c = g[0] * dir.x * dir.x + g[5] * dir.y * dir.y + g[10] * dir.z * dir.z +
              2.0f * (g[1] * dir.x * dir.y + g[2] * dir.x * dir.z + g[6] * dir.y * dir.z);
    float rt = sqrtf(b * b - 4.0f * a * c);
    float u0 = fmaxf((-b + rt) / (2.0f * a), (-b - rt) / (2.0f * a));
    if (u0 < 0.0f) u0 = 1.0f;
    R.r[0] = fp.cam[0]; R.r[1] = fp.cam[1]; R.r[2] = fp.cam[2]; R.r[3] = 0.f;
    R.u[0] = dir.x; R.u[1] = dir.y; R.u[2] = dir.z; R.u[3] = u0;
    R.result = PRR_RESULT_SUCCESS;
    R.I = 0.f;
}

template <int GEOD> __device__ __forceinline__ V4<float> pgeod(const Hot<float> &q, const V4<float> &x, const V4<float> &u)
{
    return phys_geod<float, GEOD>(q, x, u);
}

__device__ __forceinline__ bool plain_scene(const FrameParams &fp, const V4<float> &x, const V4<float> &u, float h, V3<float> *col)
{
    Hit c = intersect_scene<float>(fp, x.x, x.y, x.z, u.x, u.y, u.z, h);
    if (c.hit && col) *col = {c.r, c.g, c.b};
    return c.hit;
}

template <int GEOD>
__global__ void __launch_bounds__(64) k_plain_trace(const FrameParams *__restrict__ fps, int frame, PlainRay *rays, int layer,
                                                    int nlines, unsigned long long *counters)
{
    using F = Fehlberg;
    const FrameParams &fp = fps[frame];
    int ix = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y + layer * nlines;
    if (ix >= fp.samples * fp.width || y >= fp.height || y >= (layer + 1) * nlines) return;
    PlainRay &RR = rays[(size_t)y * fp.samples * fp.width + ix];
    Hot<float> q = make_hot<float>(fp);
    V4<float> x = {RR.r[0], RR.r[1], RR.r[2], RR.r[3]}, u = {RR.u[0], RR.u[1], RR.u[2], RR.u[3]};
    float h = fp.h, trace_h = fp.h;
    bool intersect = false;
    int i = 0, accepted = 0, result = PRR_RESULT_INFINITE_GEO;
    V3<float> hitcol = {0, 0, 0};
    bool have_col = false;
    for (float l = 0.0f; l < 1000.0f;) {
        i += 1;
        V4<float> kx1 = v4scl(h, u), ku1 = v4scl(h, pgeod<GEOD>(q, x, u));
        V4<float> z2x = v4add(x, v4scl((float)F::A21, kx1)), z2u = v4add(u, v4scl((float)F::A21, ku1));
        V4<float> kx2 = v4scl(h, z2u), ku2 = v4scl(h, pgeod<GEOD>(q, z2x, z2u));
        V4<float> z3x = v4add(v4add(x, v4scl((float)F::A31, kx1)), v4scl((float)F::A32, kx2));
        V4<float> z3u = v4add(v4add(u, v4scl((float)F::A31, ku1)), v4scl((float)F::A32, ku2));
        V4<float> kx3 = v4scl(h, z3u), ku3 = v4scl(h, pgeod<GEOD>(q, z3x, z3u));
        V4<float> z4x = v4add(v4add(v4add(x, v4scl((float)F::A41, kx1)), v4scl((float)F::A42, kx2)), v4scl((float)F::A43, kx3));
        V4<float> z4u = v4add(v4add(v4add(u, v4scl((float)F::A41, ku1)), v4scl((float)F::A42, ku2)), v4scl((float)F::A43, ku3));
        V4<float> kx4 = v4scl(h, z4u), ku4 = v4scl(h, pgeod<GEOD>(q, z4x, z4u));
        V4<float> z5x = v4add(v4add(v4add(v4add(x, v4scl((float)F::A51, kx1)), v4scl((float)F::A52, kx2)), v4scl((float)F::A53, kx3)), v4scl((float)F::A54, kx4));
        V4<float> z5u = v4add(v4add(v4add(v4add(u, v4scl((float)F::A51, ku1)), v4scl((float)F::A52, ku2)), v4scl((float)F::A53, ku3)), v4scl((float)F::A54, ku4));
        V4<float> kx5 = v4scl(h, z5u), ku5 = v4scl(h, pgeod<GEOD>(q, z5x, z5u));
        V4<float> z6x = v4add(v4add(v4add(v4add(v4add(x, v4scl((float)F::A61, kx1)), v4scl((float)F::A62, kx2)), v4scl((float)F::A63, kx3)), v4scl((float)F::A64, kx4)), v4scl((float)F::A65, kx5));
        V4<float> z6u = v4add(v4add(v4add(v4add(v4add(u, v4scl((float)F::A61, ku1)), v4scl((float)F::A62, ku2)), v4scl((float)F::A63, ku3)), v4scl((float)F::A64, ku4)), v4scl((float)F::A65, ku5));
        V4<float> kx6 = v4scl(h, z6u), ku6 = v4scl(h, pgeod<GEOD>(q, z6x, z6u));
        float xs4[4], us4[4], xs5[4], us5[4];
        const float *X = &x.x, *U = &u.x;
        const V4<float> *KX[6] = {&kx1, &kx2, &kx3, &kx4, &kx5, &kx6}, *KU[6] = {&ku1, &ku2, &ku3, &ku4, &ku5, &ku6};
        const float K4[6] = {(float)F::K41, (float)F::K42, (float)F::K43, (float)F::K44, (float)F::K45, (float)F::K46};
        const float K5[6] = {(float)F::K51, (float)F::K52, (float)F::K53, (float)F::K54, (float)F::K55, (float)F::K56};
        float err = 0.f;
#pragma unroll
        for (int c = 0; c < 4; c++) {
            float a4 = X[c], b4 = U[c], a5 = X[c], b5 = U[c];
#pragma unroll
            for (int j = 0; j < 6; j++) {
                a4 += K4[j] * (&KX[j]->x)[c]; b4 += K4[j] * (&KU[j]->x)[c];
                a5 += K5[j] * (&KX[j]->x)[c]; b5 += K5[j] * (&KU[j]->x)[c];
            }
            xs4[c] = a4; us4[c] = b4; xs5[c] = a5; us5[c] = b5;
            float sx = q.atol + q.rtol * fmaxf(fabsf(X[c]), fabsf(a4)), su = q.atol + q.rtol * fmaxf(fabsf(U[c]), fabsf(b4));
            err = fmaxf(err, fabsf(a5 - a4) / sx);
            err = fmaxf(err, fabsf(b5 - b4) / su);
        }
        float hn = fminf(fmaxf(0.9f * h * powf(err, -0.2f), q.hmin), q.hmax);
        if (intersect && i > 10000) intersect = false;
        if (i > 8 * q.max_steps) break;
        if (err > 1.0f && h != q.hmin && !intersect) { h = hn; continue; }
        V4<float> xn = {xs4[0], xs4[1], xs4[2], xs4[3]}, un = {us4[0], us4[1], us4[2], us4[3]};
        if (isnan(xn.x + xn.y + xn.z + xn.w + un.x + un.y + un.z + un.w)) { result = PRR_RESULT_MATH_ERROR; break; }
        // User_UPDATE
        if (!plain_scene(fp, xn, un, h, nullptr)) {
            if (!intersect) h = hn;
            x = xn; u = un; trace_h = h;
        } else if (!intersect) {
            intersect = true; h = q.hmin; continue;
        } else {
            x = xn; u = un;
        }
        accepted++;
        // User_ENDLOOP
        float r = metric_radius<float>(fp, x.x, x.y, x.z);
        if (r >= q.rout || (q.metric != PRR_METRIC_FLAT && r <= q.rstop)) { result = PRR_RESULT_SUCCESS; break; }
        if (plain_scene(fp, x, u, trace_h, &hitcol)) { result = PRR_RESULT_INTERSECTION; have_col = true; break; }
        l += h;
        if (accepted >= q.max_steps) break;
    }
    RR.r[0] = x.x; RR.r[1] = x.y; RR.r[2] = x.z; RR.r[3] = x.w;
    if (have_col) { RR.u[0] = hitcol.x; RR.u[1] = hitcol.y; RR.u[2] = hitcol.z; RR.u[3] = 0.f; }
    else { RR.u[0] = u.x; RR.u[1] = u.y; RR.u[2] = u.z; RR.u[3] = u.w; }
    RR.result = result;
    RR.I = (float)accepted;
    if (counters) {
        atomicAdd(&counters[C_ATTEMPTS], (unsigned long long)i);
        atomicAdd(&counters[C_ACCEPTED], (unsigned long long)accepted);
        atomicAdd(&counters[C_RAYS], 1ull);
    }
}

__global__ void k_plain_colour(const FrameParams *__restrict__ fps, int frame, const PlainRay *rays, float *rgb)
{
    const FrameParams &fp = fps[frame];
    int ix = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix >= fp.width * fp.samples || y >= fp.height) return;
    size_t id = (size_t)y * fp.width * fp.samples + ix;
    const PlainRay &R = rays[id];
    V4<float> x = {R.r[0], R.r[1], R.r[2], R.r[3]}, u = {R.u[0], R.u[1], R.u[2], R.u[3]};
    V3<float> c = ray_colour<float>(fp, R.result, x, u);
    rgb[3 * id] = c.x; rgb[3 * id + 1] = c.y; rgb[3 * id + 2] = c.z;
}

cudaError_t launch_plain_frame(const FrameParams *d_fp, const FrameParams &h_fp, int frame, PlainBuffers &b,
                               unsigned long long *counters, int geod_table, cudaStream_t st, int *launches)
{
    PlainRay *rays = (PlainRay *)b.rays;
    const int W = h_fp.width, H = h_fp.height, S = h_fp.samples;
    dim3 thr(8, 8);
    int n = 0;
    k_plain_create<<<dim3(W / 8 + 1, H / 8 + 1), thr, 0, st>>>(d_fp, frame, rays); n++;
    k_plain_init<<<dim3(S * W / 8 + 1, H / 8 + 1), thr, 0, st>>>(d_fp, frame, rays); n++;
    const int nlines = 64;
    int nlayers = (H + nlines - 1) / nlines;
    dim3 lg(S * W / 8 + 1, nlines / 8 + 1);
    for (int l = 0; l < nlayers; l++) {
        if (geod_table) k_plain_trace<1><<<lg, thr, 0, st>>>(d_fp, frame, rays, l, nlines, counters);
        else k_plain_trace<0><<<lg, thr, 0, st>>>(d_fp, frame, rays, l, nlines, counters);
        n++;
    }
    k_plain_colour<<<dim3(S * W / 8 + 1, H / 8 + 1), thr, 0, st>>>(d_fp, frame, rays, b.rgb); n++;
    if (launches) *launches += n;
    return cudaGetLastError();
}

}  // namespace prr
