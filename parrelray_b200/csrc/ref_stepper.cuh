// ref_stepper.cuh - REFERENCE-mode integration of one ray: the control flow
// and FP32 arithmetic of kernels/solver.cuh (initRays 26-56, trace_Euler
// 68-116, trace_RKF 142-219) and the Schwarzschild/flat hooks
// (metrics/schwarzschild.cuh:55-79, metrics/flat.cuh:55-79), quirks included:
//   * the velocity stage inputs use h*u (kx) where h*du (ku) belongs
//     (solver.cuh:164-168);
//   * the initial 4-velocity is (dir, 1) scaled by the larger root u0
//     (solver.cuh:52-54);
//   * absolute error test max|y5 - y4| <= eps (solver.cuh:174-188);
//   * the NaN test looks at the state before the step (solver.cuh:190).
// Compiled with -fmad=false so the FP32 operation sequence is the one the
// source spells out.
#pragma once
#include "prr_device.cuh"

namespace prr {

struct RefRay {
    float uvx, uvy;
    int result;
    V4<float> r, u;  // Ray::r, Ray::u
    int accepted, attempts;
};

// Tableau of solver.cuh:125-131: double literals stored as float.
struct RefTab {
    static constexpr float A21 = (float)(1.0 / 4.0), A31 = (float)(3.0 / 32.0), A32 = (float)(9.0 / 32.0),
                           A41 = (float)(1932.0 / 2197.0), A42 = (float)(-7200.0 / 2197.0), A43 = (float)(7296.0 / 2197.0),
                           A51 = (float)(439.0 / 216.0), A52 = (float)(-8.0), A53 = (float)(3680.0 / 513.0),
                           A54 = (float)(-845.0 / 4104.0), A61 = (float)(-8.0 / 27.0), A62 = (float)(2.0),
                           A63 = (float)(-3544.0 / 2565.0), A64 = (float)(1859.0 / 4104.0), A65 = (float)(-11.0 / 40.0),
                           K41 = (float)(25.0 / 216.0), K42 = 0.0f, K43 = (float)(1408.0 / 2565.0),
                           K44 = (float)(2197.0 / 4104.0), K45 = (float)(-1.0 / 5.0), K46 = 0.0f,
                           K51 = (float)(16.0 / 135.0), K52 = 0.0f, K53 = (float)(6656.0 / 12825.0),
                           K54 = (float)(28561.0 / 56430.0), K55 = (float)(-9.0 / 50.0), K56 = (float)(2.0 / 55.0);
};

PRR_DEV V4<float> ref_geod(const FrameParams &fp, const V4<float> &x, const V4<float> &u)
{
    if (fp.metric == PRR_METRIC_FLAT) return {0.0f, 0.0f, 0.0f, 0.0f};
    if (fp.metric == PRR_METRIC_SCHWARZSCHILD) return geod_schw_ref(x, u, fp.rs);
    return geod_ks<float>(x, u, fp.M, fp.a);
}

PRR_DEV bool isnan4(const V4<float> &a) { return isnan(a.x) || isnan(a.y) || isnan(a.z) || isnan(a.w); }

// The solver below calls the metric through a hooks object H with the
// reference's hook set (kernels/solver.cuh:43,81,87,96,106,154,163-168,197,
// 209): metric(R, g) = getMetric, geod(x, u) = getGeod, loop(R) = User_LOOP,
// update(R, h) = User_UPDATE, endloop(R, trace_h) = User_ENDLOOP.
// BuiltinHooks are the library's flat / Schwarzschild / Kerr hooks; a metric
// plug-in header supplies its own (parrelray_b200/compat/prr_plugin.cuh).

// initRays
template <class H> PRR_DEV void ref_init_h(const FrameParams &fp, const H &hk, int x, int y, int s, RefRay &R)
{
    ray_uv(fp, x, y, s, R.uvx, R.uvy);
    V4<float> u;
    if constexpr (H::kSpherical) {
        // a hook set in spherical coordinates places the ray itself
        // (kernels/solver.cuh:34-37)
        hk.spherical_start(R, u);
    } else {
        V3<float> dir = ray_dir(fp, R.uvx, R.uvy);
        R.r = {fp.cam[0], fp.cam[1], fp.cam[2], 0.0f};
        u = {dir.x, dir.y, dir.z, 1.0f};
    }
    R.u = {0.0f, 0.0f, 0.0f, 0.0f};
    R.result = PRR_RESULT_SUCCESS;
    float g[16];
    hk.metric(R, g);
    float a = g[15];
    float b = 2.0f * (g[12] * u.x + g[13] * u.y + g[14] * u.z);
    float c = g[0] * u.x * u.x + g[5] * u.y * u.y + g[10] * u.z * u.z + 2.0f * (g[1] * u.x * u.y + g[2] * u.x * u.z + g[6] * u.y * u.z);
    float rt = sqrtf(b * b - 4.0f * a * c);
    float u0 = fmaxf((-b + rt) / (2.0f * a), (-b - rt) / (2.0f * a));
    if (u0 < 0.0f) u0 = 1.0f;
    R.u = v4scl(u0, u);
    R.result = PRR_RESULT_SUCCESS;
    R.accepted = 0;
    R.attempts = 0;
}

PRR_DEV void ref_metric(const FrameParams &fp, const RefRay &R, float g[16])
{
    if (fp.metric == PRR_METRIC_SCHWARZSCHILD) metric_schw_ref(R.r.x, R.r.y, R.r.z, fp.rs, g);
    else metric_ks<float>(R.r.x, R.r.y, R.r.z, fp.metric == PRR_METRIC_FLAT ? 0.0f : fp.M, fp.a, g);
}

// User_UPDATE
PRR_DEV bool ref_update(const FrameParams &fp, RefRay &R, float h)
{
    Hit c = intersect_scene<float>(fp, R.r.x, R.r.y, R.r.z, R.u.x, R.u.y, R.u.z, h);
    if (c.hit) { R.result = PRR_RESULT_INTERSECTION; return false; }
    return true;
}

// User_ENDLOOP
PRR_DEV bool ref_endloop(const FrameParams &fp, RefRay &R, float th)
{
    float r = metric_radius<float>(fp, R.r.x, R.r.y, R.r.z);
    if (r >= fp.rout || (fp.metric != PRR_METRIC_FLAT && r <= fp.rstop)) { R.result = PRR_RESULT_SUCCESS; return false; }
    Hit c = intersect_scene<float>(fp, R.r.x, R.r.y, R.r.z, R.u.x, R.u.y, R.u.z, th);
    if (c.hit) { R.u = {c.r, c.g, c.b, 0.0f}; R.result = PRR_RESULT_INTERSECTION; return false; }
    return true;
}

struct BuiltinHooks {
    static constexpr bool kSpherical = false;  // Cartesian (x, y, z, t) states
    const FrameParams &fp;
    PRR_DEV void metric(const RefRay &R, float g[16]) const { ref_metric(fp, R, g); }
    PRR_DEV V4<float> geod(const V4<float> &x, const V4<float> &u) const { return ref_geod(fp, x, u); }
    PRR_DEV bool loop(RefRay &) const { return true; }
    PRR_DEV bool update(RefRay &R, float h) const { return ref_update(fp, R, h); }
    PRR_DEV bool endloop(RefRay &R, float trace_h) const { return ref_endloop(fp, R, trace_h); }
};

// trace_RKF
template <class H> PRR_DEV void ref_rkf_h(const FrameParams &fp, const H &hk, RefRay &R)
{
    using K = RefTab;
    if (!hk.loop(R)) { R.result = PRR_RESULT_INFINITE_GEO; return; }
    float h = fp.h, hmin = fp.hmin, hmax = fp.hmax, _h = h, eps = fp.eps, trace_h = fp.h;
    V4<float> x = R.r, u = R.u, _x = x, _u = u, __x, __u;
    bool intersect = false;
    int i = 0;
    for (float l = 0.0f; l < 1000.0f;) {
        i += 1;
        R.attempts = i;
        V4<float> kx1 = v4scl(h, u);
        V4<float> ku1 = v4scl(h, hk.geod(x, u));
        V4<float> z2x = v4add(x, v4scl(K::A21, kx1)), z2u = v4add(u, v4scl(K::A21, kx1));
        V4<float> kx2 = v4scl(h, z2u), ku2 = v4scl(h, hk.geod(z2x, z2u));
        V4<float> z3x = v4add(v4add(x, v4scl(K::A31, kx1)), v4scl(K::A32, kx2));
        V4<float> z3u = v4add(v4add(u, v4scl(K::A31, kx1)), v4scl(K::A32, ku2));
        V4<float> kx3 = v4scl(h, z3u), ku3 = v4scl(h, hk.geod(z3x, z3u));
        V4<float> z4x = v4add(v4add(v4add(x, v4scl(K::A41, kx1)), v4scl(K::A42, kx2)), v4scl(K::A43, kx3));
        V4<float> z4u = v4add(v4add(v4add(u, v4scl(K::A41, kx1)), v4scl(K::A42, ku2)), v4scl(K::A43, ku3));
        V4<float> kx4 = v4scl(h, z4u), ku4 = v4scl(h, hk.geod(z4x, z4u));
        V4<float> z5x = v4add(v4add(v4add(v4add(x, v4scl(K::A51, kx1)), v4scl(K::A52, kx2)), v4scl(K::A53, kx3)), v4scl(K::A54, kx4));
        V4<float> z5u = v4add(v4add(v4add(v4add(u, v4scl(K::A51, kx1)), v4scl(K::A52, ku2)), v4scl(K::A53, ku3)), v4scl(K::A54, ku4));
        V4<float> kx5 = v4scl(h, z5u), ku5 = v4scl(h, hk.geod(z5x, z5u));
        V4<float> z6x = v4add(v4add(v4add(v4add(v4add(x, v4scl(K::A61, kx1)), v4scl(K::A62, kx2)), v4scl(K::A63, kx3)), v4scl(K::A64, kx4)), v4scl(K::A65, kx5));
        V4<float> z6u = v4add(v4add(v4add(v4add(v4add(u, v4scl(K::A61, kx1)), v4scl(K::A62, ku2)), v4scl(K::A63, ku3)), v4scl(K::A64, ku4)), v4scl(K::A65, ku5));
        V4<float> kx6 = v4scl(h, z6u), ku6 = v4scl(h, hk.geod(z6x, z6u));

        _x = v4add(v4add(v4add(v4add(v4add(v4add(x, v4scl(K::K41, kx1)), v4scl(K::K42, kx2)), v4scl(K::K43, kx3)), v4scl(K::K44, kx4)), v4scl(K::K45, kx5)), v4scl(K::K46, kx6));
        _u = v4add(v4add(v4add(v4add(v4add(v4add(u, v4scl(K::K41, ku1)), v4scl(K::K42, ku2)), v4scl(K::K43, ku3)), v4scl(K::K44, ku4)), v4scl(K::K45, ku5)), v4scl(K::K46, ku6));
        __x = v4add(v4add(v4add(v4add(v4add(v4add(x, v4scl(K::K51, kx1)), v4scl(K::K52, kx2)), v4scl(K::K53, kx3)), v4scl(K::K54, kx4)), v4scl(K::K55, kx5)), v4scl(K::K56, kx6));
        __u = v4add(v4add(v4add(v4add(v4add(v4add(u, v4scl(K::K51, ku1)), v4scl(K::K52, ku2)), v4scl(K::K53, ku3)), v4scl(K::K54, ku4)), v4scl(K::K55, ku5)), v4scl(K::K56, ku6));

        float ex = fmaxf(fmaxf(fmaxf(fabsf(__x.x - _x.x), fabsf(__x.y - _x.y)), fabsf(__x.z - _x.z)), fabsf(__x.w - _x.w));
        float eu = fmaxf(fmaxf(fmaxf(fabsf(__u.x - _u.x), fabsf(__u.y - _u.y)), fabsf(__u.z - _u.z)), fabsf(__u.w - _u.w));
        float maxerr = fmaxf(ex, eu);
        _h = 0.9f * h * powf(eps / maxerr, 0.2f);
        _h = fminf(fmaxf(_h, hmin), hmax);

        if (intersect && i > 10000) intersect = false;
        if (i > 1000000) break;
        if (maxerr > eps && h != hmin && !intersect) { h = _h; continue; }
        if (isnan4(x) || isnan4(u)) { R.result = PRR_RESULT_MATH_ERROR; return; }

        R.r = _x; R.u = _u;
        R.accepted += 1;
        if (hk.update(R, h)) {
            if (!intersect) h = _h;
            x = _x; u = _u; R.r = x; R.u = u; trace_h = h;
        } else if (R.result == PRR_RESULT_INTERSECTION && !intersect) {
            intersect = true; h = hmin; continue;
        }
        if (!hk.endloop(R, trace_h)) return;
        x = R.r; u = R.u;
        l += h;
    }
    R.result = PRR_RESULT_INFINITE_GEO;
}

// trace_Euler
template <class H> PRR_DEV void ref_euler_h(const FrameParams &fp, const H &hk, RefRay &R)
{
    if (!hk.loop(R)) { R.result = PRR_RESULT_INFINITE_GEO; return; }
    bool intersect = false;
    float h = fp.h;
    for (float l = 0.0f; l < 5000.0f; l += h) {
        V4<float> du = hk.geod(R.r, R.u);
        R.attempts += 1;
        if (isnan4(du)) { R.result = PRR_RESULT_MATH_ERROR; return; }
        R.r = v4add(R.r, v4scl(h, R.u));
        R.u = v4add(R.u, v4scl(h, du));
        R.accepted += 1;
        if (!hk.update(R, h)) {
            if (R.result == PRR_RESULT_INTERSECTION && !intersect) { intersect = true; h = fp.hmin; continue; }
        }
        if (!hk.endloop(R, fp.h)) return;
    }
    R.result = PRR_RESULT_INFINITE_GEO;
}

PRR_DEV void ref_init(const FrameParams &fp, int x, int y, int s, RefRay &R) { ref_init_h(fp, BuiltinHooks{fp}, x, y, s, R); }
PRR_DEV void ref_rkf(const FrameParams &fp, RefRay &R) { ref_rkf_h(fp, BuiltinHooks{fp}, R); }
PRR_DEV void ref_euler(const FrameParams &fp, RefRay &R) { ref_euler_h(fp, BuiltinHooks{fp}, R); }

}  // namespace prr
