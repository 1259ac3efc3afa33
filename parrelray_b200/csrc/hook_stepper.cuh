// hook_stepper.cuh - PHYSICAL-mode integration of one ray through a hook set
// H: the same hook objects ref_stepper.cuh drives in REFERENCE mode
// (metric = getMetric, geod = getGeod, loop = User_LOOP, update =
// User_UPDATE, endloop = User_ENDLOOP, kernels/solver.cuh:43,81,87,96,106,
// 154,163-168,197,209), so a metric plug-in header written for the reference
// runs on the persistent, warp-compacted scheduler with PHYSICAL semantics.
//
// One call = one RKF45 attempt (the persistent kernel refills lanes whose ray
// ended).  Control flow is trace_RKF's (solver.cuh:142-219): reject while
// the error is too large (unless h is already hmin or the ray is in
// intersection mode), User_UPDATE with the step h (a hit enters intersection
// mode and retries at hmin), User_ENDLOOP with the last accepted step (the
// header decides termination and the hit colour), l += h, l < 1000.  What
// PHYSICAL mode changes, as for the built-in metrics (phys_stepper.cuh):
//  * textbook Fehlberg stages (the reference feeds h*u into the velocity
//    stages, solver.cuh:164-168), with the position stages linear in the
//    velocity increments (x' = u holds in any coordinates a header uses);
//  * null initial data: u = (dir, u^t) with g(u, u) = 0 for the header's
//    getMetric (the reference scales the whole (dir, 1) by u^t, solver.cuh:54);
//  * error test max_i |y5_i - y4_i| / (atol + rtol max(|y_i|, |y4_i|)) <= 1;
//  * a NaN in the new state ends the ray with MATH_ERROR;
//  * at most max_steps accepted steps and 8 max_steps attempts.
// A header's geodesic is FP32 (its getGeod takes and returns f4), so this
// path is FP32; the state is accumulated with Kahan compensation, which is
// reset whenever a hook rewrites the state (e.g. a pole flip).  Stage and
// update arithmetic use explicit fused multiply-adds, so the result does not
// depend on the -fmad setting the header is compiled with.
#pragma once
#include "phys_stepper.cuh"
#include "ref_stepper.cuh"

namespace prr {

struct HookRay {
    RefRay R;      // uv, result, r, u (the header's Ray fields), counters
    V4<float> cx, cu;  // Kahan compensation of r and u
    float h, trace_h, l;
    int intersect;
};

template <class H> PRR_DEV void hook_phys_init(const FrameParams &fp, const H &hk, int px, int py, int s, HookRay &S)
{
    RefRay &R = S.R;
    ray_uv(fp, px, py, s, R.uvx, R.uvy);
    V4<float> u;
    if constexpr (H::kSpherical) {
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
    // the larger root u^t of g_tt (u^t)^2 + 2 g_ti u^i u^t + g_ij u^i u^j = 0
    const float a = g[15];
    const float b = 2.0f * (g[12] * u.x + g[13] * u.y + g[14] * u.z);
    const float c = g[0] * u.x * u.x + g[5] * u.y * u.y + g[10] * u.z * u.z +
                    2.0f * (g[1] * u.x * u.y + g[2] * u.x * u.z + g[6] * u.y * u.z);
    const float rt = sqrtf(fmaxf(b * b - 4.0f * a * c, 0.0f));
    float u0 = fmaxf((-b + rt) / (2.0f * a), (-b - rt) / (2.0f * a));
    if (!(u0 >= 0.0f)) u0 = 1.0f;
    R.u = {u.x, u.y, u.z, u0};
    R.accepted = 0;
    R.attempts = 0;
    S.cx = {0.0f, 0.0f, 0.0f, 0.0f};
    S.cu = {0.0f, 0.0f, 0.0f, 0.0f};
    S.h = fp.h;
    S.trace_h = fp.h;
    S.l = 0.0f;
    S.intersect = 0;
}

PRR_DEV float hfma(float a, float b, float c) { return __fmaf_rn(a, b, c); }

PRR_DEV bool same4(const V4<float> &a, const V4<float> &b) { return a.x == b.x && a.y == b.y && a.z == b.z && a.w == b.w; }

// One attempt.  Returns STEP_DONE when the ray has ended (S.R.result set, and
// S.R holds the state the header's rayToRGB colours), STEP_CONTINUE
// otherwise.
template <class H> PRR_DEV int hook_phys_attempt(const FrameParams &fp, const H &hk, HookRay &S)
{
    using F = Fehlberg;
    RefRay &R = S.R;
    if (R.attempts == 0 && !hk.loop(R)) { R.result = PRR_RESULT_INFINITE_GEO; return STEP_DONE; }
    if (!(S.l < 1000.0f)) { R.result = PRR_RESULT_INFINITE_GEO; return STEP_DONE; }
    R.attempts += 1;
    if (R.attempts > 8 * fp.max_steps) { R.result = PRR_RESULT_INFINITE_GEO; return STEP_DONE; }
    const float h = S.h;
    const V4<float> x = R.r, u = R.u;
#define PRR_C(v) ((float)(v))
#define PRR_EACH(OP) OP(x) OP(y) OP(z) OP(w)
    V4<float> zx, zu;
    const V4<float> k1 = v4scl(h, hk.geod(x, u));
#define S2(c) zx.c = hfma(h, PRR_C(F::c2) * u.c, x.c); zu.c = hfma(PRR_C(F::A21), k1.c, u.c);
    PRR_EACH(S2)
#undef S2
    const V4<float> k2 = v4scl(h, hk.geod(zx, zu));
#define S3(c)                                                                                                      \
    zx.c = hfma(h, hfma(PRR_C(F::c3), u.c, PRR_C(F::B31) * k1.c), x.c);                                          \
    zu.c = hfma(PRR_C(F::A32), k2.c, hfma(PRR_C(F::A31), k1.c, u.c));
    PRR_EACH(S3)
#undef S3
    const V4<float> k3 = v4scl(h, hk.geod(zx, zu));
#define S4(c)                                                                                                      \
    zx.c = hfma(h, hfma(PRR_C(F::c4), u.c, hfma(PRR_C(F::B42), k2.c, PRR_C(F::B41) * k1.c)), x.c);              \
    zu.c = hfma(PRR_C(F::A43), k3.c, hfma(PRR_C(F::A42), k2.c, hfma(PRR_C(F::A41), k1.c, u.c)));
    PRR_EACH(S4)
#undef S4
    const V4<float> k4 = v4scl(h, hk.geod(zx, zu));
#define S5(c)                                                                                                      \
    zx.c = hfma(h, hfma(PRR_C(F::c5), u.c, hfma(PRR_C(F::B53), k3.c, hfma(PRR_C(F::B52), k2.c,                   \
                                                                        PRR_C(F::B51) * k1.c))), x.c);            \
    zu.c = hfma(PRR_C(F::A54), k4.c, hfma(PRR_C(F::A53), k3.c, hfma(PRR_C(F::A52), k2.c, hfma(PRR_C(F::A51), k1.c, u.c))));
    PRR_EACH(S5)
#undef S5
    const V4<float> k5 = v4scl(h, hk.geod(zx, zu));
#define S6(c)                                                                                                      \
    zx.c = hfma(h, hfma(PRR_C(F::c6), u.c, hfma(PRR_C(F::B64), k4.c, hfma(PRR_C(F::B63), k3.c,                   \
                hfma(PRR_C(F::B62), k2.c, PRR_C(F::B61) * k1.c)))), x.c);                                          \
    zu.c = hfma(PRR_C(F::A65), k5.c, hfma(PRR_C(F::A64), k4.c, hfma(PRR_C(F::A63), k3.c,                          \
                hfma(PRR_C(F::A62), k2.c, hfma(PRR_C(F::A61), k1.c, u.c)))));
    PRR_EACH(S6)
#undef S6
    const V4<float> k6 = v4scl(h, hk.geod(zx, zu));
    float dxv[4], duv[4], err = 0.0f;
    const float xs[4] = {x.x, x.y, x.z, x.w}, us[4] = {u.x, u.y, u.z, u.w};
    const float K1[4] = {k1.x, k1.y, k1.z, k1.w}, K2[4] = {k2.x, k2.y, k2.z, k2.w}, K3[4] = {k3.x, k3.y, k3.z, k3.w},
                K4[4] = {k4.x, k4.y, k4.z, k4.w}, K5[4] = {k5.x, k5.y, k5.z, k5.w}, K6[4] = {k6.x, k6.y, k6.z, k6.w};
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const float du = hfma(PRR_C(F::K45), K5[j], hfma(PRR_C(F::K44), K4[j], hfma(PRR_C(F::K43), K3[j], PRR_C(F::K41) * K1[j])));
        const float dx = h * hfma(PRR_C(F::b4), K4[j], hfma(PRR_C(F::b3), K3[j], hfma(PRR_C(F::b2), K2[j],
                                                                                       hfma(PRR_C(F::b1), K1[j], us[j]))));
        const float eu = hfma(PRR_C(F::E6), K6[j], hfma(PRR_C(F::E5), K5[j], hfma(PRR_C(F::E4), K4[j],
                                                                                    hfma(PRR_C(F::E3), K3[j], PRR_C(F::E1) * K1[j]))));
        const float ex = h * hfma(PRR_C(F::e5), K5[j], hfma(PRR_C(F::e4), K4[j], hfma(PRR_C(F::e3), K3[j],
                                                                                       hfma(PRR_C(F::e2), K2[j], PRR_C(F::e1) * K1[j]))));
        const float sx = hfma(fp.rtol, fmaxf(fabsf(xs[j]), fabsf(xs[j] + dx)), fp.atol);
        const float su = hfma(fp.rtol, fmaxf(fabsf(us[j]), fabsf(us[j] + du)), fp.atol);
        err = fmaxf(err, fmaxf(fabsf(ex) / sx, fabsf(eu) / su));
        dxv[j] = dx;
        duv[j] = du;
    }
#undef PRR_EACH
#undef PRR_C
    float hn = 0.9f * h * fpow<float>(err, -0.2f);
    hn = fminf(fmaxf(hn, fp.hmin), fp.hmax);
    if (S.intersect && R.attempts > 10000) S.intersect = 0;
    if (err > 1.0f && h != fp.hmin && !S.intersect) { S.h = hn; return STEP_CONTINUE; }

    // the new state, compensated
    V4<float> xn = x, un = u, cxn = S.cx, cun = S.cu;
    kahan_add(xn.x, cxn.x, dxv[0]); kahan_add(xn.y, cxn.y, dxv[1]); kahan_add(xn.z, cxn.z, dxv[2]); kahan_add(xn.w, cxn.w, dxv[3]);
    kahan_add(un.x, cun.x, duv[0]); kahan_add(un.y, cun.y, duv[1]); kahan_add(un.z, cun.z, duv[2]); kahan_add(un.w, cun.w, duv[3]);
    if (isnan4(xn) || isnan4(un)) { R.result = PRR_RESULT_MATH_ERROR; return STEP_DONE; }

    R.r = xn; R.u = un;
    R.accepted += 1;
    if (hk.update(R, h)) {
        if (!S.intersect) S.h = hn;
        S.trace_h = S.h;
    } else if (R.result == PRR_RESULT_INTERSECTION && !S.intersect) {
        // enter intersection mode: back to the accepted state, retry at hmin
        S.intersect = 1;
        S.h = fp.hmin;
        R.r = x; R.u = u;
        R.accepted -= 1;
        return STEP_CONTINUE;
    }
    const V4<float> xh = R.r, uh = R.u;
    if (!hk.endloop(R, S.trace_h)) return STEP_DONE;
    if (!same4(R.r, xh) || !same4(R.u, uh) || !same4(xh, xn) || !same4(uh, un)) {
        S.cx = {0.0f, 0.0f, 0.0f, 0.0f};  // a hook rewrote the state: its compensation no longer applies
        S.cu = {0.0f, 0.0f, 0.0f, 0.0f};
    } else {
        S.cx = cxn; S.cu = cun;
    }
    S.l += S.h;
    if (R.accepted >= fp.max_steps) { R.result = PRR_RESULT_INFINITE_GEO; return STEP_DONE; }
    return STEP_CONTINUE;
}

}  // namespace prr
