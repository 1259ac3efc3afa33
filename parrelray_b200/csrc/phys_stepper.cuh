// phys_stepper.cuh - PHYSICAL-mode integration of one ray as a state machine
// that advances by one RKF45 attempt per call, so a warp can keep each lane
// on its own ray (the persistent scheduler refills lanes whose ray ended).
//
// Relative to the reference trace_RKF (kernels/solver.cuh:142-219) the
// control flow - accept/reject, intersection mode, hooks, caps - is the
// same.  What differs, on purpose:
//  * stages are the textbook Fehlberg ones (the reference feeds h*u into the
//    velocity stages, solver.cuh:164-168);
//  * initial data are null: u = (dir, u^t) with g(u,u) = 0 (the reference
//    scales the whole (dir, 1) by u^t, solver.cuh:54);
//  * error test: max_i |y5_i - y4_i| / (atol + rtol*max(|y_i|, |y4_i|)) <= 1;
//  * a NaN in the new state ends the ray with MATH_ERROR at once;
//  * step cap max_steps accepted steps (and 8*max_steps attempts).
// Implementation (B200): the system is second order (x' = u, u' = G), so the
// position stages are linear in the velocity stages:
//   z_i^x = x + h (c_i u + sum_m B_im ku_m),  B = A*A,  c = A*1,
//   x4 = x + h (u + sum_m beta_m ku_m),       beta = K4^T A,
//   x5 - x4 = h sum_m eps_m ku_m,             eps = (K5-K4)^T A,
// so only the six velocity increments ku_m are kept in registers (the
// reference keeps kx and ku).  In FP32 the state is accumulated with Kahan
// compensation.  The two sphere tests of an accepted step (User_UPDATE with
// the step h, User_ENDLOOP with the next step) share one geometry pass.
#pragma once
#include "emission.cuh"
#include "geod_table.cuh"
#include "prr_device.cuh"

namespace prr {

struct Fehlberg {
    static constexpr double A21 = 1.0 / 4.0, A31 = 3.0 / 32.0, A32 = 9.0 / 32.0, A41 = 1932.0 / 2197.0,
                            A42 = -7200.0 / 2197.0, A43 = 7296.0 / 2197.0, A51 = 439.0 / 216.0, A52 = -8.0,
                            A53 = 3680.0 / 513.0, A54 = -845.0 / 4104.0, A61 = -8.0 / 27.0, A62 = 2.0,
                            A63 = -3544.0 / 2565.0, A64 = 1859.0 / 4104.0, A65 = -11.0 / 40.0;
    static constexpr double K41 = 25.0 / 216.0, K42 = 0.0, K43 = 1408.0 / 2565.0, K44 = 2197.0 / 4104.0,
                            K45 = -1.0 / 5.0, K46 = 0.0;
    static constexpr double K51 = 16.0 / 135.0, K52 = 0.0, K53 = 6656.0 / 12825.0, K54 = 28561.0 / 56430.0,
                            K55 = -9.0 / 50.0, K56 = 2.0 / 55.0;
    // row sums
    static constexpr double c2 = A21, c3 = A31 + A32, c4 = A41 + A42 + A43, c5 = A51 + A52 + A53 + A54,
                            c6 = A61 + A62 + A63 + A64 + A65;
    // B = A*A
    static constexpr double B31 = A32 * A21;
    static constexpr double B41 = A42 * A21 + A43 * A31, B42 = A43 * A32;
    static constexpr double B51 = A52 * A21 + A53 * A31 + A54 * A41, B52 = A53 * A32 + A54 * A42, B53 = A54 * A43;
    static constexpr double B61 = A62 * A21 + A63 * A31 + A64 * A41 + A65 * A51,
                            B62 = A63 * A32 + A64 * A42 + A65 * A52, B63 = A64 * A43 + A65 * A53, B64 = A65 * A54;
    // beta = K4^T A, eps = (K5-K4)^T A, E = K5-K4
    static constexpr double E1 = K51 - K41, E2 = K52 - K42, E3 = K53 - K43, E4 = K54 - K44, E5 = K55 - K45,
                            E6 = K56 - K46;
    static constexpr double b1 = K42 * A21 + K43 * A31 + K44 * A41 + K45 * A51 + K46 * A61,
                            b2 = K43 * A32 + K44 * A42 + K45 * A52 + K46 * A62, b3 = K44 * A43 + K45 * A53 + K46 * A63,
                            b4 = K45 * A54 + K46 * A64, b5 = K46 * A65;
    static constexpr double e1 = E2 * A21 + E3 * A31 + E4 * A41 + E5 * A51 + E6 * A61,
                            e2 = E3 * A32 + E4 * A42 + E5 * A52 + E6 * A62, e3 = E4 * A43 + E5 * A53 + E6 * A63,
                            e4 = E5 * A54 + E6 * A64, e5 = E6 * A65;
};

template <class T> struct PhysRay {
    V4<T> x, u;    // accepted state
    V4<T> cx, cu;  // Kahan compensation (FP32 only)
    T h, trace_h, l;
    int i, accepted;
    int intersect;
};

// Per-ray copy of the frame's scalars used every attempt.
template <class T> struct Hot {
    T M, a, hmin, hmax, rtol, atol, rout, rstop;
    int metric, max_steps, nspheres;
};

template <class T> PRR_DEV Hot<T> make_hot(const FrameParams &fp)
{
    Hot<T> q;
    q.M = fp.metric == PRR_METRIC_FLAT ? (T)0 : (T)fp.M;
    q.a = fp.metric == PRR_METRIC_KERR ? (T)fp.a : (T)0;
    q.hmin = (T)fp.hmin; q.hmax = (T)fp.hmax; q.rtol = (T)fp.rtol; q.atol = (T)fp.atol;
    q.rout = (T)fp.rout; q.rstop = (T)fp.rstop;
    q.metric = fp.metric; q.max_steps = fp.max_steps; q.nspheres = fp.nspheres;
    return q;
}




// Null initial data: position = camera, u = (dir, u^t), u^t the larger root
// of g_tt (u^t)^2 + 2 g_ti u^i u^t + g_ij u^i u^j = 0 (initRays solves the
// same quadratic, solver.cuh:48-53).
template <class T> PRR_DEV void phys_init(const FrameParams &fp, int px, int py, int s, PhysRay<T> &R, float *uv_out = nullptr)
{
    float uvx, uvy;
    ray_uv(fp, px, py, s, uvx, uvy);
    if (uv_out) { uv_out[0] = uvx; uv_out[1] = uvy; }
    V3<float> dir = ray_dir(fp, uvx, uvy);
    R.x = {(T)fp.cam[0], (T)fp.cam[1], (T)fp.cam[2], (T)0};
    R.u = {(T)dir.x, (T)dir.y, (T)dir.z, (T)1};
    T g[16];
    metric_ks<T>(R.x.x, R.x.y, R.x.z, fp.metric == PRR_METRIC_FLAT ? (T)0 : (T)fp.M,
                 fp.metric == PRR_METRIC_KERR ? (T)fp.a : (T)0, g);
    const V4<T> &u = R.u;
    T a = g[15];
    T b = (T)2 * (g[12] * u.x + g[13] * u.y + g[14] * u.z);
    T c = g[0] * u.x * u.x + g[5] * u.y * u.y + g[10] * u.z * u.z + (T)2 * (g[1] * u.x * u.y + g[2] * u.x * u.z + g[6] * u.y * u.z);
    T rt = sqrt(b * b - (T)4 * a * c);
    T u0 = fmax((-b + rt) / ((T)2 * a), (-b - rt) / ((T)2 * a));
    if (u0 < (T)0) u0 = (T)1;
    R.u.w = u0;
    R.cx = {0, 0, 0, 0};
    R.cu = {0, 0, 0, 0};
    R.h = (T)fp.h; R.trace_h = (T)fp.h; R.l = 0;
    R.i = 0; R.accepted = 0; R.intersect = 0;
}

template <class T, int GEOD> PRR_DEV V4<T> phys_geod(const Hot<T> &q, const V4<T> &x, const V4<T> &u)
{
    if (q.metric == PRR_METRIC_FLAT) return {0, 0, 0, 0};
    if (GEOD == 1) return geod_table<T>(x, u, q.M, q.a);
    return geod_ks<T, true>(x, u, q.M, q.a);
}

// Distance d of Sphere::intersects (scene/sphere.h:40-48) along the unit
// velocity v; returns false when the sphere is missed (disc < 0 or d < 0).
template <class T> PRR_DEV bool sphere_d(const DevSphere &S, T px, T py, T pz, T vx, T vy, T vz, T v2, T &d)
{
    T dx = px - (T)S.cx, dy = py - (T)S.cy, dz = pz - (T)S.cz, rad = (T)S.r;
    T dvp = vx * dx + vy * dy + vz * dz;
    T disc = dvp * dvp - v2 * ((dx * dx + dy * dy + dz * dz) - rad * rad);
    if (disc < (T)0) return false;
    T sd = disc > (T)0 ? disc * frsqrt<T>(disc) : (T)0;
    d = ((T)-2.0f * dvp - sd) * frcp<T>(v2);
    return d >= (T)0;
}

// True when the point p is too far from sphere S for Sphere::intersects to
// accept it with any window h <= hmax: a hit needs the distance to the
// centre D to satisfy D^2 <= ((sqrt(hmax) + R)/2)^2 + R^2 (S.far2 holds
// that bound with a rounding margin), so skipping the test changes nothing.
template <class T> PRR_DEV bool sphere_far(const DevSphere &S, T px, T py, T pz)
{
    T dx = px - (T)S.cx, dy = py - (T)S.cy, dz = pz - (T)S.cz;
    return dx * dx + dy * dy + dz * dz > (T)S.far2;
}

// Sphere::getColor at p + v d (scene/sphere.h:59-64).
template <class T> PRR_DEV V3<float> sphere_colour(const DevSphere &S, T px, T py, T pz, T vx, T vy, T vz, T d)
{
    T ix = (px + vx * d) - (T)S.cx, iy = (py + vy * d) - (T)S.cy, iz = (pz + vz * d) - (T)S.cz, rad = (T)S.r;
    T theta = acos(iz / rad);
    T phi = (T)((double)atan2(iy, ix) + PI_SPHERE);
    T uu = (T)((double)phi / (2.0 * PI_SPHERE)), vv = (T)((double)theta / PI_SPHERE);
    const T uvmax = (T)0.999999999f;
    uu = fmin(fmax(uu, (T)0), uvmax);
    vv = fmin(fmax(vv, (T)0), uvmax);
    V3<T> col = {(T)0.5, (T)0.5, (T)0.5};
    if (S.tex.p) col = tex_bilinear<T>(S.tex, uu, vv);
    T shade = fmax((T)0, fmin((T)0.5 + (T)0.5 * iz / rad, (T)1));
    return {(float)(col.x * shade), (float)(col.y * shade), (float)(col.z * shade)};
}

// Sky colour of an escaped ray from its direction of flight.
template <class T> PRR_DEV V3<float> escape_colour(const FrameParams &fp, const V4<T> &u)
{
    if (!fp.bg.p) return {0.0f, 0.0f, 0.0f};
    if (fp.bg_filter == PRR_BG_BILINEAR) {
        V3<T> b = background_bilinear<T>(fp.bg, u.x, u.y, u.z);
        return {(float)b.x, (float)b.y, (float)b.z};
    }
    return background_rms<T>(fp.bg, u.x, u.y, u.z);
}

template <class T> PRR_DEV void kahan_add(T &s, T &c, T v)
{
    T y = v - c;
    T t = s + y;
    c = (t - s) - y;
    s = t;
}

enum StepStatus { STEP_CONTINUE = 0, STEP_DONE = 1, STEP_FLAG64 = 2 };

// One RKF45 attempt plus, when accepted, the hooks.  Returns STEP_DONE with
// `result` and `colour` set when the ray has terminated, STEP_FLAG64 when a
// split-precision render must re-integrate it in FP64.
// hit_sphere: when non-null, an INTERSECTION stores the hit sphere's index
// there and leaves the final state in R (otherwise R.u receives the colour,
// as User_ENDLOOP does).
// em: when non-null, every accepted step adds its plasma emission
// (emission.cuh) before the termination tests.
// An attempt is split in three parts so the FP32 path can evaluate the
// stages of two rays at once (phys_pair.cuh): phys_precheck (caps before
// the attempt), the stages (increments dxv/duv, scaled error err and next
// step hn), and phys_accept (accept/reject, state update, hooks).

// The loop bound of trace_RKF (l < 1000, solver.cuh:158) and the attempt
// counter; STEP_DONE when the ray ends before this attempt.
template <class T> PRR_DEV int phys_precheck(PhysRay<T> &R, int &result, V3<float> &colour)
{
    if (!(R.l < (T)1000)) { result = PRR_RESULT_INFINITE_GEO; colour = {0, 0, 0}; return STEP_DONE; }
    R.i += 1;
    return STEP_CONTINUE;
}

template <class T>
PRR_DEV int phys_accept(const FrameParams &fp, const Hot<T> &q, PhysRay<T> &R, const T dxv[4], const T duv[4], T err,
                        T hn, int &result, V3<float> &colour, T flag_r, int *hit_sphere, EmisRay<T> *em = nullptr);

template <class T, int GEOD>
PRR_DEV int phys_attempt(const FrameParams &fp, const Hot<T> &q, PhysRay<T> &R, int &result, V3<float> &colour,
                         T flag_r, int *hit_sphere = nullptr, EmisRay<T> *em = nullptr)
{
    using F = Fehlberg;
    if (phys_precheck<T>(R, result, colour) == STEP_DONE) return STEP_DONE;
    const T h = R.h;
    const V4<T> &x = R.x, &u = R.u;
#define PRR_ST2(c)                                                                                                 \
    zx.c = x.c + h * ((T)F::c2 * u.c);                                                                           \
    zu.c = u.c + (T)F::A21 * k1.c;
#define PRR_ST3(c)                                                                                                 \
    zx.c = x.c + h * ((T)F::c3 * u.c + (T)F::B31 * k1.c);                                                        \
    zu.c = u.c + (T)F::A31 * k1.c + (T)F::A32 * k2.c;
#define PRR_ST4(c)                                                                                                 \
    zx.c = x.c + h * ((T)F::c4 * u.c + (T)F::B41 * k1.c + (T)F::B42 * k2.c);                                     \
    zu.c = u.c + (T)F::A41 * k1.c + (T)F::A42 * k2.c + (T)F::A43 * k3.c;
#define PRR_ST5(c)                                                                                                 \
    zx.c = x.c + h * ((T)F::c5 * u.c + (T)F::B51 * k1.c + (T)F::B52 * k2.c + (T)F::B53 * k3.c);                 \
    zu.c = u.c + (T)F::A51 * k1.c + (T)F::A52 * k2.c + (T)F::A53 * k3.c + (T)F::A54 * k4.c;
#define PRR_ST6(c)                                                                                                 \
    zx.c = x.c + h * ((T)F::c6 * u.c + (T)F::B61 * k1.c + (T)F::B62 * k2.c + (T)F::B63 * k3.c + (T)F::B64 * k4.c); \
    zu.c = u.c + (T)F::A61 * k1.c + (T)F::A62 * k2.c + (T)F::A63 * k3.c + (T)F::A64 * k4.c + (T)F::A65 * k5.c;
    V4<T> k1, k2, k3, k4, k5, k6, zx, zu;
#ifdef PRR_STAGE_LOOP
    // one geodesic call site; the stage index is warp-uniform, so the
    // switch does not diverge, and every k stays in named registers
    zx = x; zu = u;
#pragma unroll 1
    for (int s = 0; s < 6; s++) {
        V4<T> g = v4scl(h, phys_geod<T, GEOD>(q, zx, zu));
        switch (s) {
        case 0: k1 = g; PRR_ST2(x) PRR_ST2(y) PRR_ST2(z) PRR_ST2(w) break;
        case 1: k2 = g; PRR_ST3(x) PRR_ST3(y) PRR_ST3(z) PRR_ST3(w) break;
        case 2: k3 = g; PRR_ST4(x) PRR_ST4(y) PRR_ST4(z) PRR_ST4(w) break;
        case 3: k4 = g; PRR_ST5(x) PRR_ST5(y) PRR_ST5(z) PRR_ST5(w) break;
        case 4: k5 = g; PRR_ST6(x) PRR_ST6(y) PRR_ST6(z) PRR_ST6(w) break;
        default: k6 = g; break;
        }
    }
#else
    k1 = v4scl(h, phys_geod<T, GEOD>(q, x, u));
    PRR_ST2(x) PRR_ST2(y) PRR_ST2(z) PRR_ST2(w)
    k2 = v4scl(h, phys_geod<T, GEOD>(q, zx, zu));
    PRR_ST3(x) PRR_ST3(y) PRR_ST3(z) PRR_ST3(w)
    k3 = v4scl(h, phys_geod<T, GEOD>(q, zx, zu));
    PRR_ST4(x) PRR_ST4(y) PRR_ST4(z) PRR_ST4(w)
    k4 = v4scl(h, phys_geod<T, GEOD>(q, zx, zu));
    PRR_ST5(x) PRR_ST5(y) PRR_ST5(z) PRR_ST5(w)
    k5 = v4scl(h, phys_geod<T, GEOD>(q, zx, zu));
    PRR_ST6(x) PRR_ST6(y) PRR_ST6(z) PRR_ST6(w)
    k6 = v4scl(h, phys_geod<T, GEOD>(q, zx, zu));
#endif
#undef PRR_ST2
#undef PRR_ST3
#undef PRR_ST4
#undef PRR_ST5
#undef PRR_ST6

    // increments, error estimate and scaled error norm
    T dxv[4], duv[4], err = 0;
#define PRR_FIN(c, j)                                                                                              \
    {                                                                                                              \
        T du = (T)F::K41 * k1.c + (T)F::K43 * k3.c + (T)F::K44 * k4.c + (T)F::K45 * k5.c;                      \
        T dx = h * (u.c + (T)F::b1 * k1.c + (T)F::b2 * k2.c + (T)F::b3 * k3.c + (T)F::b4 * k4.c);             \
        T eu = (T)F::E1 * k1.c + (T)F::E3 * k3.c + (T)F::E4 * k4.c + (T)F::E5 * k5.c + (T)F::E6 * k6.c;        \
        T ex = h * ((T)F::e1 * k1.c + (T)F::e2 * k2.c + (T)F::e3 * k3.c + (T)F::e4 * k4.c + (T)F::e5 * k5.c);  \
        T sx = q.atol + q.rtol * fmax(fabs(x.c), fabs(x.c + dx));                                                 \
        T su = q.atol + q.rtol * fmax(fabs(u.c), fabs(u.c + du));                                                 \
        err = fmax(err, fabs(ex) * frcp<T>(sx));                                                               \
        err = fmax(err, fabs(eu) * frcp<T>(su));                                                               \
        dxv[j] = dx; duv[j] = du;                                                                                  \
    }
    PRR_FIN(x, 0) PRR_FIN(y, 1) PRR_FIN(z, 2) PRR_FIN(w, 3)
#undef PRR_FIN
    T hn = (T)0.9 * h * fpow<T>(err, (T)-0.2);
    hn = fmin(fmax(hn, q.hmin), q.hmax);
    return phys_accept<T>(fp, q, R, dxv, duv, err, hn, result, colour, flag_r, hit_sphere, em);
}

template <class T>
PRR_DEV int phys_accept(const FrameParams &fp, const Hot<T> &q, PhysRay<T> &R, const T dxv[4], const T duv[4], T err,
                        T hn, int &result, V3<float> &colour, T flag_r, int *hit_sphere, EmisRay<T> *em)
{
    const T h = R.h;
    if (R.intersect && R.i > 10000) R.intersect = 0;
    if (R.i > 8 * q.max_steps) { result = PRR_RESULT_INFINITE_GEO; colour = {0, 0, 0}; return STEP_DONE; }
    if (err > (T)1 && h != q.hmin && !R.intersect) { R.h = hn; return STEP_CONTINUE; }

    // candidate new state
    V4<T> xn = R.x, un = R.u, cxn = R.cx, cun = R.cu;
    kahan_add(xn.x, cxn.x, dxv[0]); kahan_add(xn.y, cxn.y, dxv[1]); kahan_add(xn.z, cxn.z, dxv[2]); kahan_add(xn.w, cxn.w, dxv[3]);
    kahan_add(un.x, cun.x, duv[0]); kahan_add(un.y, cun.y, duv[1]); kahan_add(un.z, cun.z, duv[2]); kahan_add(un.w, cun.w, duv[3]);
    if (isnan(xn.x + xn.y + xn.z + xn.w + un.x + un.y + un.z + un.w)) {
        result = PRR_RESULT_MATH_ERROR; colour = {0, 0, 0}; return STEP_DONE;
    }

    // sphere geometry, shared by User_UPDATE (window h) and User_ENDLOOP
    // (window = next step, or the previous one in intersection mode)
    bool hitU = false;
    int candH = -1, candN = -1, candT = -1;
    T dH = (T)1e11, dN = (T)1e11, dT = (T)1e11;
    T vx = 0, vy = 0, vz = 0, v2 = 0;
    bool near = false;
    const T R2 = xn.x * xn.x + xn.y * xn.y + xn.z * xn.z;
    if (R2 >= (T)fp.sph_lo2 && R2 <= (T)fp.sph_hi2)
        for (int s = 0; s < q.nspheres; s++) near |= !sphere_far<T>(fp.sph[s], xn.x, xn.y, xn.z);
    if (near) {
        T k = frsqrt<T>(un.x * un.x + un.y * un.y + un.z * un.z);
        vx = un.x * k; vy = un.y * k; vz = un.z * k;
        v2 = vx * vx + vy * vy + vz * vz;
        for (int s = 0; s < q.nspheres; s++) {
            T d;
            if (!sphere_d<T>(fp.sph[s], xn.x, xn.y, xn.z, vx, vy, vz, v2, d)) continue;
            T dd = d * d;
            if (!(dd > v2 * h)) { hitU = true; if (d <= dH) { dH = d; candH = s; } }
            if (!(dd > v2 * hn) && d <= dN) { dN = d; candN = s; }
            if (!(dd > v2 * R.trace_h) && d <= dT) { dT = d; candT = s; }
        }
    }
    if (hitU && !R.intersect) {  // enter intersection mode; the step is retried at hmin
        R.intersect = 1; R.h = q.hmin;
        return STEP_CONTINUE;
    }
    R.x = xn; R.u = un; R.cx = cxn; R.cu = cun;
    R.accepted += 1;
    if (em) emis_step<T>(fp, q.M, q.a, xn, un, h, *em);
    int candE;
    T dE;
    if (!hitU) {
        if (!R.intersect) R.h = hn;
        R.trace_h = R.h;
        if (R.intersect) { candE = candH; dE = dH; } else { candE = candN; dE = dN; }
    } else {
        candE = candT; dE = dT;
    }
    // User_ENDLOOP, on the squared radius (one square root for Kerr, none otherwise)
    T r2 = R2;
    if (q.metric == PRR_METRIC_KERR) {
        T b = r2 - q.a * q.a;
        T S2 = b * b + (T)4 * q.a * q.a * xn.z * xn.z;
        r2 = (T)0.5 * (b + S2 * frsqrt<T>(S2));
    }
    const bool escaped = r2 >= q.rout * q.rout;
    if (escaped || (q.metric != PRR_METRIC_FLAT && r2 <= q.rstop * q.rstop)) {
        result = PRR_RESULT_SUCCESS;
        colour = escaped ? escape_colour<T>(fp, R.u) : V3<float>{0.0f, 0.0f, 0.0f};
        return STEP_DONE;
    }
    if (candE >= 0) {
        result = PRR_RESULT_INTERSECTION;
        colour = sphere_colour<T>(fp.sph[candE], xn.x, xn.y, xn.z, vx, vy, vz, dE);
        if (hit_sphere) *hit_sphere = candE;  // the caller keeps the final state
        else R.u = {(T)colour.x, (T)colour.y, (T)colour.z, (T)0};
        return STEP_DONE;
    }
    if (flag_r > (T)0 && r2 < flag_r * flag_r) return STEP_FLAG64;
    R.l += R.h;
    if (R.accepted >= q.max_steps) { result = PRR_RESULT_INFINITE_GEO; colour = {0, 0, 0}; return STEP_DONE; }
    return STEP_CONTINUE;
}

// Split precision: is the ray within `delta` of a photon orbit?  Uses the
// conserved E, L_z and Carter Q of the initial data: xi = L_z/E,
// eta = Q/E^2, and the Boyer-Lindquist radial potential
//   R(r) = (r^2 + a^2 - a xi)^2 - Delta (eta + (xi - a)^2).
// A photon orbit is a double root of R; for Schwarzschild
// min_r R/r^4 = 1 - (b/b_c)^2, so |min R/r^4| < 2 delta is |b - b_c|/b_c < delta
// to first order.  The minimum is searched on [r_+, 6M].
template <class T> PRR_DEV bool near_critical(const FrameParams &fp, const PhysRay<T> &R)
{
    if (fp.metric == PRR_METRIC_FLAT || fp.fp64_delta <= 0.0f) return false;
    double M = fp.M, a = fp.metric == PRR_METRIC_KERR ? fp.a : 0.0;
    double x = R.x.x, y = R.x.y, z = R.x.z;
    double g[16];
    metric_ks<double>(x, y, z, M, a, g);
    double uu[4] = {R.u.x, R.u.y, R.u.z, R.u.w};
    double p[4];
    for (int m = 0; m < 4; m++) p[m] = g[4 * m] * uu[0] + g[4 * m + 1] * uu[1] + g[4 * m + 2] * uu[2] + g[4 * m + 3] * uu[3];
    double E = -p[3];
    double Lz = x * p[1] - y * p[0];
    double r = ks_radius<double>(x, y, z, a);
    double ct = z / r, st2 = 1.0 - ct * ct;
    if (st2 < 1e-12 || E == 0.0) return false;
    double st = sqrt(st2);
    double pth = (ct / st) * (x * p[0] + y * p[1]) - r * st * p[2];
    double Q = pth * pth + ct * ct * (-a * a * E * E + Lz * Lz / st2);
    double xi = Lz / E, eta = Q / (E * E);
    double rp = kerr_r_plus<double>(M, a);
    double lo = rp * 1.0001, hi = 6.0 * M;
    const int N = 48;
    const double dr = (hi - lo) / N;
    auto pot = [&](double rr) {
        double A = rr * rr + a * a - a * xi;
        double D = rr * rr - 2.0 * M * rr + a * a;
        return (A * A - D * (eta + (xi - a) * (xi - a))) / (rr * rr * rr * rr);
    };
    double best = 1e300;
    int kb = 0;
    for (int k = 0; k <= N; k++) {
        double v = pot(lo + dr * k);
        if (v < best) { best = v; kb = k; }
    }
    if (kb > 0 && kb < N) {  // parabola through the three samples around the minimum
        double vm = pot(lo + dr * (kb - 1)), vp = pot(lo + dr * (kb + 1));
        double den = vm - 2.0 * best + vp;
        if (den > 0.0) best = best - 0.125 * (vp - vm) * (vp - vm) / den;
    }
    return fabs(best) < 2.0 * fp.fp64_delta;
}

}  // namespace prr
