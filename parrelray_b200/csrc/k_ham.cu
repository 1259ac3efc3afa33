// k_ham.cu - the FP32 renderer of PHYSICAL frames (one pixel in flight per
// thread) with the geodesic in Hamiltonian form; with SPLIT, the FP32 pass of a
// split-precision render; with EMIS, plasma emission along the rays.
//
// The geodesics of the Kerr-Schild metric g = eta + f l(x)l are integrated
// as the canonical system of H = 1/2 g^{ab} p_a p_b with the inverse metric
// g^{-1} = eta - f l l (l^a = eta^{ab} l_b, l^t = -1):
//     dx^i/dlambda = p_i - f Lam l_i,
//     dp_i/dlambda = 1/2 Lam^2 d_i f + f Lam d_i Lam,   Lam = l^a p_a,
// and p_t = -E is a constant of the motion (the metric does not depend on
// t), so the state is (x, y, z, p_x, p_y, p_z): six components instead of the
// eight of (x, u), no coordinate time, and no directional derivatives or
// raised contraction in the right-hand side (about 65 FP32 operations and 4
// SFU operations per evaluation, against about 110 for the contraction
// geod_ks evaluates for du/dlambda).  The velocity u = dx/dlambda, which the
// sphere test, the sky lookup and the per-ray outputs need, is formed from
// (x, p) where it is used.
//
// Everything else is the PHYSICAL mode of phys_stepper.cuh, unchanged:
// Fehlberg's RKF45 tableau with the 4th-order solution propagated, the mixed
// error test max_i |y5_i - y4_i| / (atol + rtol max(|y_i|, |y4_i|)) <= 1 over
// the state's components, the step update 0.9 h err^(-1/5) clamped to
// [hmin, hmax], Kahan-compensated FP32 updates, the reference's
// accept/reject, intersection-mode, sphere-window and termination rules
// (kernels/solver.cuh:142-219, metrics/schwarzschild.cuh:55-79,
// scene/sphere.h:34-64), l < 1000 and the max_steps caps.  Initial data are
// phys_init's null u, lowered once: p = g u.
//
// Scheduling is k_pair's (k_pair.cu): persistent CTAs, each lane owns one
// pixel and integrates its SSAA samples in order with the RMS combine in
// registers, one attempt per loop iteration, warp-aggregated refill of the
// lanes whose pixel is complete every compaction_interval attempts.  The
// three coordinate pairs (x, y), (p_x, p_y) and (z, p_z) share Blackwell's
// paired FP32 instructions in the stage combinations, and the x/y twins of
// the right-hand side (gradients, l, the gradient of Lam, the derivatives)
// share them too.
//
// SPLIT (split precision): per-sample colours go to sample_rgb (the per-pixel
// combine runs after the FP64 pass), and rays near a photon orbit
// (near_critical on the initial data) or that dip below fp64_rfac * r_+ are
// queued for k_fp64_requeue (k_persistent.cu), which integrates them again
// from the camera in FP64, as for k_pair's split pass.
//
// EMIS: the emission of emission.cuh at every accepted step, in its momentum
// form (emis_step_p: k.u_e = p_mu u_e^mu, no lowering needed).
#include "kernels.cuh"
#include "phys_pair.cuh"

namespace prr {

namespace {

using namespace pv;

constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ int find_frame_h(const long long *begin, int n, long long item)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (__ldg(begin + mid) <= item) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ void warp_sum_add_h(unsigned long long *p, unsigned long long v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(p, v);
}

__device__ __forceinline__ uint8_t q8h(float v) { return (uint8_t)roundf(255.0f * fminf(fmaxf(v, 0.0f), 1.0f)); }

// Per-ray constants of the right-hand side.
template <class T> struct HamConst {
    T M2, a, a2, nha2, pt;  // 2M, a, a^2, -a^2/2, p_t
};

// dy/dlambda at (P = (x, y), Q = (p_x, p_y), W = (z, p_z)); outputs dP, dQ, dW
// in the same pairing.  r is the Kerr-Schild radius, r^4 - (R^2 - a^2) r^2 -
// a^2 z^2 = 0; f = 2 M r^3 / (r^4 + a^2 z^2); l = ((r x + a y)/q, (r y - a
// x)/q, z/r) with q = r^2 + a^2 (l_t = 1).
template <class T>
PRR_DEV void ham_rhs(P2<T> P, P2<T> Q, P2<T> W, const HamConst<T> &c, P2<T> &dP, P2<T> &dQ, P2<T> &dW)
{
    using V = P2<T>;
    const T X = P.x, Y = P.y, z = W.x, pz = W.y;
    // with hb = (R^2 - a^2)/2 and Sh = S/2, S = sqrt((R^2 - a^2)^2 + 4 a^2 z^2):
    // r^2 = hb + Sh, grad r = (x, y, z q / r^2) r / S
    const T Z2 = mul_(z, z);
    const T R2 = fma_(X, X, fma_(Y, Y, Z2));
    const T hb = fma_(T(0.5), R2, c.nha2);
    const T a2Z2 = mul_(c.a2, Z2);
    const T S2h = fma_(hb, hb, a2Z2);
    const T iSh = rsq_(S2h);
    const T r2 = fma_(S2h, iSh, hb);
    const T ir = rsq_(r2);
    const T r = mul_(r2, ir);
    const T q = add_(r2, c.a2), iq = rcp_(q);
    const T Sig = fma_(r2, r2, a2Z2), iSig = rcp_(Sig);
    const V iq_ = sp(iq);
    // twice the gradient of r, and grad f / (2 f) (the 1/2 of 1/2 Lam^2 grad f folded in, and f taken out
    // into f Lam below): grad f = c1 grad r with c1 = f (3/r - 4 r^3/Sigma); c1/(4 f) = 3/(4r) - r^3/Sigma
    const V dr2 = mul_(P, sp(mul_(r, iSh)));
    const T drz2 = mul_(mul_(z, q), mul_(iSh, ir));
    const T r3 = mul_(r2, r);
    const T t = mul_(r3, iSig);
    const T f = mul_(c.M2, t);
    const T c1h = fma_(T(0.75), ir, neg_(t));
    const V dgh = mul_(sp(c1h), dr2);
    const T dgzh = fma_(c1h, drz2, mul_(iSig, mul_(neg_(c.a2), z)));
    // l and Lam = l.p - p_t
    const V l = mul_(fma_(sp(r), P, f2(mul_(c.a, Y), neg_(mul_(c.a, X)))), iq_);
    const T lz = mul_(z, ir);
    const T px = Q.x, py = Q.y;
    const T lpxy = fma_(px, l.x, mul_(py, l.y));
    const T Lam = fma_(lz, pz, add_(lpxy, neg_(c.pt)));
    // gradient of l.p at fixed p: grad r times Pp = ((x p_x + y p_y) - 2 r l.p_xy)/q - p_z l_z / r, taken
    // as (2 grad r) (Pp / 2)
    const T P0h = fma_(neg_(r), lpxy, mul_(T(0.5), fma_(px, X, mul_(py, Y))));
    const T Pph = fma_(P0h, iq, neg_(mul_(mul_(T(0.5), pz), mul_(lz, ir))));
    const V dL = fma_(dr2, sp(Pph), mul_(f2(fma_(r, px, neg_(mul_(c.a, py))), fma_(c.a, px, mul_(r, py))), iq_));
    const T dLz = fma_(drz2, Pph, mul_(pz, ir));
    // Hamilton's equations, dp = 1/2 Lam^2 grad f + f Lam grad Lam = f Lam (Lam grad f / (2 f) + grad Lam)
    const T fL = mul_(f, Lam);
    const V sfL = sp(fL);
    dQ = mul_(sfL, fma_(sp(Lam), dgh, dL));
    dP = fma_(neg_(sfL), l, Q);
    dW = f2(fma_(neg_(fL), lz, pz), mul_(fL, fma_(Lam, dgzh, dLz)));
}

// u = dx/dlambda (spatial) and u^t = -p_t + f Lam at (x, p), with IEEE
// square roots: used by the sphere test, the sky lookup and the outputs.
template <class T> PRR_DEV V4<T> ham_velocity(T x, T y, T z, T px, T py, T pz, const HamConst<T> &c)
{
    const T R2 = x * x + y * y + z * z;
    const T hb = T(0.5) * R2 + c.nha2;
    const T r2 = hb + sqrt(hb * hb + c.a2 * z * z);
    const T r = sqrt(r2);
    const T q = r2 + c.a2;
    const T f = c.M2 * r2 * r / (r2 * r2 + c.a2 * z * z);
    const T lx = (r * x + c.a * y) / q, ly = (r * y - c.a * x) / q, lz = z / r;
    const T Lam = lx * px + ly * py + lz * pz - c.pt;
    const T fL = f * Lam;
    return {px - fL * lx, py - fL * ly, pz - fL * lz, fL - c.pt};
}

template <class T> struct HamRay {
    P2<T> P, Q, W;     // (x, y), (p_x, p_y), (z, p_z)
    P2<T> cP, cQ, cW;  // Kahan compensation (FP32 only)
    T h, trace_h, l;
    T safe;  // FP32: distance to the nearest sphere's far radius at the last test, less the path since
    int i, accepted, intersect;
};

template <class T> struct HSlot {
    int frame, px, py, s, S;
    float acc0, acc1, acc2;
    bool busy, need;
    bool crit;      // split precision: the sample's initial data are near a photon orbit
    float flag_r;   // split precision: queue the ray for FP64 below this radius
    HamRay<T> R;
    HamConst<T> c;
    Hot<T> q;
    EmisRay<T> E;  // emission kernels only
};

// phys_init's null initial data, lowered: p_a = g_ab u^b.
template <class T, bool SPLIT, bool EMIS = false>
__device__ __forceinline__ void ham_init(const FrameParams &fp, HSlot<T> &sl, int s)
{
    PhysRay<T> U;
    phys_init<T>(fp, sl.px, sl.py, s, U);
    if constexpr (SPLIT) sl.crit = near_critical<T>(fp, U);
    const T M = fp.metric == PRR_METRIC_FLAT ? T(0) : (T)fp.M, a = fp.metric == PRR_METRIC_KERR ? (T)fp.a : T(0);
    T g[16];
    metric_ks<T>(U.x.x, U.x.y, U.x.z, M, a, g);
    const T u[4] = {U.u.x, U.u.y, U.u.z, U.u.w};
    T p[4];
#pragma unroll
    for (int m = 0; m < 4; m++) p[m] = g[4 * m] * u[0] + g[4 * m + 1] * u[1] + g[4 * m + 2] * u[2] + g[4 * m + 3] * u[3];
    HamRay<T> &R = sl.R;
    R.P = f2(U.x.x, U.x.y);
    R.Q = f2(p[0], p[1]);
    R.W = f2(U.x.z, p[2]);
    R.cP = R.cQ = R.cW = sp(T(0));
    R.h = (T)fp.h; R.trace_h = (T)fp.h; R.l = T(0);
    R.i = 0; R.accepted = 0; R.intersect = 0;
    R.safe = T(-1);
    sl.c = {T(2) * M, a, a * a, T(-0.5) * a * a, p[3]};
    if constexpr (EMIS) emis_init_p<T>(fp, U.x.x, U.x.y, U.x.z, p[3], sl.E);
}

template <class T> struct HamStep {
    P2<T> dP, dQ, dW;  // 4th-order increments
    T err, hn;
};

// The six Fehlberg stages on the pairs, the 4th-order increments, the scaled
// error norm and the next step (as pv::stages does for (x, u)).
template <class T> PRR_DEV HamStep<T> ham_stages(const HamRay<T> &R, const HamConst<T> &c, const Hot<T> &q)
{
    using F = Fehlberg;
    using V = P2<T>;
    const T h = R.h;
    const V H = sp(h);
    const V P = R.P, Q = R.Q, W = R.W;
#define PC(v) sp((T)(v))
#define RHS(kP, kQ, kW, zP, zQ, zW)                                                                                    \
    {                                                                                                                  \
        V dP_, dQ_, dW_;                                                                                               \
        ham_rhs<T>(zP, zQ, zW, c, dP_, dQ_, dW_);                                                                      \
        kP = mul_(H, dP_); kQ = mul_(H, dQ_); kW = mul_(H, dW_);                                                        \
    }
    V k1P, k1Q, k1W, k2P, k2Q, k2W, k3P, k3Q, k3W, k4P, k4Q, k4W, k5P, k5Q, k5W, k6P, k6Q, k6W;
    RHS(k1P, k1Q, k1W, P, Q, W)
#define ST2(Y) fma_(PC(F::A21), k1##Y, Y)
    RHS(k2P, k2Q, k2W, ST2(P), ST2(Q), ST2(W))
#undef ST2
#define ST3(Y) fma_(PC(F::A32), k2##Y, fma_(PC(F::A31), k1##Y, Y))
    RHS(k3P, k3Q, k3W, ST3(P), ST3(Q), ST3(W))
#undef ST3
#define ST4(Y) fma_(PC(F::A43), k3##Y, fma_(PC(F::A42), k2##Y, fma_(PC(F::A41), k1##Y, Y)))
    RHS(k4P, k4Q, k4W, ST4(P), ST4(Q), ST4(W))
#undef ST4
#define ST5(Y) fma_(PC(F::A54), k4##Y, fma_(PC(F::A53), k3##Y, fma_(PC(F::A52), k2##Y, fma_(PC(F::A51), k1##Y, Y))))
    RHS(k5P, k5Q, k5W, ST5(P), ST5(Q), ST5(W))
#undef ST5
#define ST6(Y)                                                                                                         \
    fma_(PC(F::A65), k5##Y, fma_(PC(F::A64), k4##Y, fma_(PC(F::A63), k3##Y, fma_(PC(F::A62), k2##Y,                \
                                                                              fma_(PC(F::A61), k1##Y, Y)))))
    RHS(k6P, k6Q, k6W, ST6(P), ST6(Q), ST6(W))
#undef ST6
#undef RHS
    HamStep<T> o;
    V err2 = sp(T(0));
    const V rtol = sp(q.rtol), atol = sp(q.atol);
#define FIN(Y, OUT)                                                                                                    \
    {                                                                                                                  \
        const V d = fma_(PC(F::K45), k5##Y, fma_(PC(F::K44), k4##Y, fma_(PC(F::K43), k3##Y, mul_(PC(F::K41), k1##Y)))); \
        const V e = fma_(PC(F::E6), k6##Y, fma_(PC(F::E5), k5##Y, fma_(PC(F::E4), k4##Y,                          \
                                                                          fma_(PC(F::E3), k3##Y, mul_(PC(F::E1), k1##Y))))); \
        const V sc = fma_(rtol, max_(abs_(Y), abs_(add_(Y, d))), atol);                                           \
        err2 = max_(err2, mul_(abs_(e), rcp_(sc)));                                                                    \
        OUT = d;                                                                                                       \
    }
    FIN(P, o.dP) FIN(Q, o.dQ) FIN(W, o.dW)
#undef FIN
#undef PC
    const T err = max_(err2.x, err2.y);
    o.err = err;
    const T hn = mul_(mul_(T(0.9), h), pow_(err, T(-0.2)));
    o.hn = min_(max_(hn, q.hmin), q.hmax);
    return o;
}

// state update: Kahan-compensated in FP32 (scalar adds: the paired form
// measured 2.5 ms slower on the 1080p frame), a plain sum in FP64 (whose
// roundoff over 10^4 steps stays far below the tolerances)
template <class V> PRR_DEV void upd2(V &s, V &c, V v)
{
    if constexpr (sizeof(s.x) == 4) {
        kahan_add(s.x, c.x, v.x);
        kahan_add(s.y, c.y, v.y);
    } else {
        s.x += v.x;
        s.y += v.y;
    }
}

// phys_accept (phys_stepper.cuh) on the Hamiltonian state.
template <class T, bool EMIS>
PRR_DEV int ham_accept(const FrameParams &fp, HSlot<T> &sl, HamRay<T> &R, const HamStep<T> &st, int &result,
                       V3<float> &colour, V4<T> &u_out)
{
    using V = P2<T>;
    const Hot<T> &q = sl.q;
    const T h = R.h, hn = st.hn;
    if (R.intersect && R.i > 10000) R.intersect = 0;
    if (R.i > 8 * q.max_steps) { result = PRR_RESULT_INFINITE_GEO; colour = {0, 0, 0}; return STEP_DONE; }
    if (st.err > T(1) && h != q.hmin && !R.intersect) { R.h = hn; return STEP_CONTINUE; }

    // candidate new state
    V Pn = R.P, Qn = R.Q, Wn = R.W, cPn = R.cP, cQn = R.cQ, cWn = R.cW;
    upd2(Pn, cPn, st.dP);
    upd2(Qn, cQn, st.dQ);
    upd2(Wn, cWn, st.dW);
    if (isnan(Pn.x + Pn.y + Wn.x + Qn.x + Qn.y + Wn.y)) {
        result = PRR_RESULT_MATH_ERROR; colour = {0, 0, 0};
        u_out = ham_velocity<T>(R.P.x, R.P.y, R.W.x, R.Q.x, R.Q.y, R.W.y, sl.c);
        return STEP_DONE;
    }
    const T xn = Pn.x, yn = Pn.y, zn = Wn.x;

    // sphere geometry, shared by User_UPDATE (window h) and User_ENDLOOP
    // (window = next step, or the previous one in intersection mode); the
    // velocity is formed only near a sphere
    bool hitU = false;
    int candH = -1, candN = -1, candT = -1;
    T dH = T(1e11), dN = T(1e11), dT = T(1e11);
    T vx = 0, vy = 0, vz = 0, v2 = 0;
    bool near = false;
    const T R2 = xn * xn + yn * yn + zn * zn;
    T safe = T(0);
    if constexpr (sizeof(T) == 4) {
        // The far tests run only when the path since the last test may have come within a sphere's far
        // radius: R.safe is the distance from the last tested point to the nearest far radius, less 1e-3,
        // and every accepted step takes its increment's L1 length (>= its Euclidean length) off it (the
        // compensated sums stay within rounding of the increments' sum). The length is summed rounding up
        // and subtracted rounding down, so the margin never drifts above the true distance, however many
        // small steps round against it. A point the margin covers is far from every sphere, so skipping
        // its tests changes nothing. One lane's test refreshes the margins of the warp's other active
        // lanes, which then run out together (a warp pays for the test once).
        safe = __fsub_rd(R.safe, __fadd_ru(__fadd_ru(fabsf(st.dP.x), fabsf(st.dP.y)), fabsf(st.dW.x)));
        if (__any_sync(__activemask(), !(safe > T(0)))) {
            T m = T(1e30);
            for (int s = 0; s < q.nspheres; s++) {
                const DevSphere &S = fp.sph[s];
                const T dx = xn - (T)S.cx, dy = yn - (T)S.cy, dz = zn - (T)S.cz;
                const T d2 = fmax(dx * dx + dy * dy + dz * dz, T(1e-30));
                near |= !(d2 > (T)S.far2);
                m = fmin(m, d2 * frsqrt<T>(d2) - (T)S.far);
            }
            safe = m - T(1e-3);
        }
    } else {  // FP64 keeps the shell test: with the margin, close cameras re-test often, each re-test pays
              // FP64 square roots, and the kernel spills more
        if (R2 >= (T)fp.sph_lo2 && R2 <= (T)fp.sph_hi2)
            for (int s = 0; s < q.nspheres; s++) near |= !sphere_far<T>(fp.sph[s], xn, yn, zn);
    }
    if (near) {
        const V4<T> un = ham_velocity<T>(xn, yn, zn, Qn.x, Qn.y, Wn.y, sl.c);
        const T k = frsqrt<T>(un.x * un.x + un.y * un.y + un.z * un.z);
        vx = un.x * k; vy = un.y * k; vz = un.z * k;
        v2 = vx * vx + vy * vy + vz * vz;
        for (int s = 0; s < q.nspheres; s++) {
            T d;
            if (!sphere_d<T>(fp.sph[s], xn, yn, zn, vx, vy, vz, v2, d)) continue;
            const T dd = d * d;
            if (!(dd > v2 * h)) { hitU = true; if (d <= dH) { dH = d; candH = s; } }
            if (!(dd > v2 * hn) && d <= dN) { dN = d; candN = s; }
            if (!(dd > v2 * R.trace_h) && d <= dT) { dT = d; candT = s; }
        }
    }
    if (hitU && !R.intersect) {  // enter intersection mode; the step is retried at hmin
        R.intersect = 1; R.h = q.hmin;
        return STEP_CONTINUE;
    }
    R.P = Pn; R.Q = Qn; R.W = Wn; R.cP = cPn; R.cQ = cQn; R.cW = cWn;
    R.safe = safe;
    R.accepted += 1;
    if constexpr (EMIS) emis_step_p<T>(fp, q.M, q.a, xn, yn, zn, Qn.x, Qn.y, Wn.y, sl.c.pt, h, sl.E);
    int candE;
    T dE;
    if (!hitU) {
        if (!R.intersect) R.h = hn;
        R.trace_h = R.h;
        if (R.intersect) { candE = candH; dE = dH; } else { candE = candN; dE = dN; }
    } else {
        candE = candT; dE = dT;
    }
    // User_ENDLOOP, on the squared radius
    T r2 = R2;
    if (q.metric == PRR_METRIC_KERR) {  // r^2 = hb + sqrt(hb^2 + a^2 z^2), hb = (R^2 - a^2)/2
        const T hb = fma_(T(0.5), R2, sl.c.nha2);
        const T S2h = fma_(hb, hb, mul_(sl.c.a2, mul_(zn, zn)));
        r2 = fma_(S2h, frsqrt<T>(S2h), hb);
    }
    const bool escaped = r2 >= q.rout * q.rout;
    if (escaped || (q.metric != PRR_METRIC_FLAT && r2 <= q.rstop * q.rstop)) {
        result = PRR_RESULT_SUCCESS;
        u_out = ham_velocity<T>(xn, yn, zn, Qn.x, Qn.y, Wn.y, sl.c);
        colour = escaped ? escape_colour<T>(fp, u_out) : V3<float>{0.0f, 0.0f, 0.0f};
        return STEP_DONE;
    }
    if (candE >= 0) {
        result = PRR_RESULT_INTERSECTION;
        colour = sphere_colour<T>(fp.sph[candE], xn, yn, zn, vx, vy, vz, dE);
        u_out = {(T)colour.x, (T)colour.y, (T)colour.z, T(0)};
        return STEP_DONE;
    }
    if (sl.flag_r > 0.0f && r2 < (T)sl.flag_r * (T)sl.flag_r) return STEP_FLAG64;
    R.l += R.h;
    if (R.accepted >= q.max_steps) {
        result = PRR_RESULT_INFINITE_GEO; colour = {0, 0, 0};
        u_out = ham_velocity<T>(xn, yn, zn, Qn.x, Qn.y, Wn.y, sl.c);
        return STEP_DONE;
    }
    return STEP_CONTINUE;
}

template <class O, class T>
__device__ __forceinline__ void ham_write_state(O *o, float uvx, float uvy, int result, T x, T y, T z, const V4<T> &u,
                                                int accepted)
{
    o[0] = (O)uvx; o[1] = (O)uvy; o[2] = (O)result;
    o[3] = (O)x; o[4] = (O)y; o[5] = (O)z; o[6] = (O)0;
    o[7] = (O)u.x; o[8] = (O)u.y; o[9] = (O)u.z; o[10] = (O)u.w;
    o[11] = (O)accepted;
}

struct HCounts {
    unsigned long long att = 0, acc = 0, rays = 0, esc = 0, cap = 0, hit = 0, inf = 0, nan = 0, f64 = 0;
};

// Split precision: a ray queued for the FP64 pass.  Its colour slot is zeroed
// here and overwritten by k_fp64_requeue, which counts it as a ray.  Returns
// true when the slot's pixel is complete.
__device__ __forceinline__ bool ham_flag(const PersistentArgs &a, HSlot<float> &sl, HCounts &c)
{
    const FrameParams &fp = a.frames[sl.frame];
    c.att += (unsigned)sl.R.i;
    c.acc += (unsigned)sl.R.accepted;
    c.f64++;
    const long long rid = ((long long)sl.py * fp.width + sl.px) * sl.S + sl.s;
    const unsigned long long slot = atomicAdd(&a.counters[C_FP64_QUEUED], 1ull);
    if ((long long)slot < a.fp64_capacity) a.fp64_queue[slot] = ((unsigned long long)sl.frame << 40) | (unsigned long long)rid;
    float *o = a.sample_rgb + 3 * (fp.ray_begin + rid);
    o[0] = o[1] = o[2] = 0.f;
    sl.s += 1;
    if (sl.s < sl.S) {
        ham_init<float, true>(fp, sl, sl.s);
        return false;
    }
    return true;
}

// A finished ray: counters, per-ray outputs, SSAA accumulation (split
// precision: the per-sample colour), next sample or pixel output.  Returns
// true when the slot's pixel is complete.
template <class T, bool SPLIT, bool EMIS>
__device__ __forceinline__ bool ham_finish(const PersistentArgs &a, HSlot<T> &sl, int result, V3<float> col,
                                           const V4<T> &u, HCounts &c)
{
    const FrameParams &fp = a.frames[sl.frame];
    if constexpr (EMIS) col = emis_colour<T>(fp, sl.E, col);
    c.att += (unsigned)sl.R.i;
    c.acc += (unsigned)sl.R.accepted;
    c.rays++;
    const T x = sl.R.P.x, y = sl.R.P.y, z = sl.R.W.x;
    if (!SPLIT && (a.ray_state || a.ray_state64 || a.sample_rgb || a.ray_steps)) {  // per-ray outputs (single-frame runs)
        const long long rid = ((long long)sl.py * fp.width + sl.px) * sl.S + sl.s;
        if (a.ray_steps) a.ray_steps[fp.ray_begin + rid] = sl.R.accepted;
        if (a.ray_state || a.ray_state64) {
            float uvx, uvy;
            ray_uv(fp, sl.px, sl.py, sl.s, uvx, uvy);
            // the coordinate time is not integrated: column 6 is 0
            if (a.ray_state) ham_write_state(a.ray_state + 12 * rid, uvx, uvy, result, x, y, z, u, sl.R.accepted);
            if (a.ray_state64) ham_write_state(a.ray_state64 + 12 * rid, uvx, uvy, result, x, y, z, u, sl.R.accepted);
        }
        if (a.sample_rgb) {
            float *o = a.sample_rgb + 3 * (fp.ray_begin + rid);
            o[0] = col.x; o[1] = col.y; o[2] = col.z;
        }
    }
    if (result == PRR_RESULT_SUCCESS) {
        if (metric_radius<T>(fp, x, y, z) >= sl.q.rout) c.esc++; else c.cap++;
    } else if (result == PRR_RESULT_INTERSECTION) c.hit++;
    else if (result == PRR_RESULT_INFINITE_GEO) c.inf++;
    else c.nan++;
    if constexpr (SPLIT) {
        const long long rid = ((long long)sl.py * fp.width + sl.px) * sl.S + sl.s;
        float *o = a.sample_rgb + 3 * (fp.ray_begin + rid);
        o[0] = col.x; o[1] = col.y; o[2] = col.z;
        sl.s += 1;
        if (sl.s < sl.S) {
            ham_init<T, true>(fp, sl, sl.s);
            return false;
        }
        return true;
    }
    if (sl.S == 1) {
        sl.acc0 = fminf(fmaxf(col.x, 0.f), 1.f); sl.acc1 = fminf(fmaxf(col.y, 0.f), 1.f); sl.acc2 = fminf(fmaxf(col.z, 0.f), 1.f);
    } else {
        sl.acc0 += fminf(fmaxf(col.x * col.x, 0.f), 1.f);
        sl.acc1 += fminf(fmaxf(col.y * col.y, 0.f), 1.f);
        sl.acc2 += fminf(fmaxf(col.z * col.z, 0.f), 1.f);
    }
    sl.s += 1;
    if (sl.s < sl.S) {
        ham_init<T, false, EMIS>(fp, sl, sl.s);
        return false;
    }
    float o0 = sl.acc0, o1 = sl.acc1, o2 = sl.acc2;
    if (sl.S > 1) { o0 = sqrtf(o0 / (float)sl.S); o1 = sqrtf(o1 / (float)sl.S); o2 = sqrtf(o2 / (float)sl.S); }
    const long long op = fp.pix_begin + (long long)sl.py * fp.width + sl.px;
    if (a.image) { a.image[3 * op] = o0; a.image[3 * op + 1] = o1; a.image[3 * op + 2] = o2; }
    if (a.rgb8 && !fp.fxaa) { a.rgb8[3 * op] = q8h(o0); a.rgb8[3 * op + 1] = q8h(o1); a.rgb8[3 * op + 2] = q8h(o2); }
    return true;
}

template <class T, bool SPLIT, bool EMIS>
__device__ __forceinline__ void ham_start(const PersistentArgs &a, HSlot<T> &sl, long long it)
{
    sl.frame = find_frame_h(a.frame_pix_begin, a.nframes, it);
    const FrameParams &fp = a.frames[sl.frame];
    const long long p = it - __ldg(a.frame_pix_begin + sl.frame);
    sl.px = (int)(p % fp.width);
    sl.py = (int)(p / fp.width);
    sl.S = fp.samples;
    sl.s = 0;
    sl.acc0 = sl.acc1 = sl.acc2 = 0.f;
    sl.q = make_hot<T>(fp);
    sl.flag_r = SPLIT ? (float)(fp.fp64_rfac * kerr_r_plus<T>(sl.q.M, sl.q.a)) : -1.0f;
    ham_init<T, SPLIT, EMIS>(fp, sl, 0);
    sl.busy = true;
}

}  // namespace

// Resident CTAs per SM the small-CTA (<= 64 threads) instantiations are
// built for: FP32 8 (128 registers, no spills); FP64 8 as well (128
// registers, 458 bytes of spills that stay in L1): the FP64 form is latency
// bound, and on the 1080p frame 8 CTAs measured 871 ms, 6 (168 registers)
// 922 ms, 4 (192 registers, no spills) 1100 ms.
#ifndef PRR_HAM_SMALL_MINB
#define PRR_HAM_SMALL_MINB 8
#endif
#ifndef PRR_HAM_SMALL_MINB_F64
#define PRR_HAM_SMALL_MINB_F64 8
#endif
template <class T> constexpr int ham_small_minb() { return sizeof(T) == 8 ? PRR_HAM_SMALL_MINB_F64 : PRR_HAM_SMALL_MINB; }

template <class T, int MAXT, int MINB, bool SPLIT, bool EMIS>
__global__ void __launch_bounds__(MAXT, MINB) k_ham(PersistentArgs a)
{
    static_assert(!(SPLIT && EMIS), "emission renders in FP32 or FP64, not split");
    static_assert(!SPLIT || sizeof(T) == 4, "the split pass is FP32");
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    HSlot<T> sl;
    HCounts cnt;
    sl.busy = false; sl.need = true; sl.crit = false; sl.flag_r = -1.0f;
    sl.frame = 0; sl.px = sl.py = sl.s = 0; sl.S = 1;
    sl.acc0 = sl.acc1 = sl.acc2 = 0.f;
    const long long t0 = clock64();
    unsigned iter = 0;
    const unsigned ci = a.compaction_interval > 1 ? (unsigned)a.compaction_interval : 1u;
    unsigned since = ci;
    while (true) {
        // ---- warp-aggregated refill of the lanes whose pixel is complete ----
        unsigned busy_mask = __ballot_sync(FULL, sl.busy);
        if (++since >= ci || busy_mask == 0) {
            since = 0;
            const unsigned m = __ballot_sync(FULL, sl.need);
            if (m) {
                const int leader = __ffs(m) - 1;
                unsigned long long base = 0;
                if (lane == leader) base = atomicAdd(&a.counters[C_WORK], (unsigned long long)__popc(m));
                base = __shfl_sync(FULL, base, leader);
                if (sl.need) {
                    const long long it = (long long)base + __popc(m & lt);
                    sl.need = false;
                    if (it < a.total_pixels) ham_start<T, SPLIT, EMIS>(a, sl, it);
                    else sl.busy = false;
                }
            }
            busy_mask = __ballot_sync(FULL, sl.busy);
        }
        if (busy_mask == 0) {
            if (__ballot_sync(FULL, sl.need) == 0) break;  // the queue is exhausted for every lane
            since = ci;
            continue;
        }
        if (a.watchdog_cycles > 0 && ((++iter) & 255u) == 0) {
            unsigned stop = 0;
            if (lane == 0) {
                if (clock64() - t0 > a.watchdog_cycles) atomicExch((unsigned long long *)&a.counters[C_TIMEOUT], 1ull);
                stop = (unsigned)*(volatile unsigned long long *)&a.counters[C_TIMEOUT];
            }
            if (__shfl_sync(FULL, stop, 0)) break;
        }
        if (!sl.busy) continue;
        // split precision: a ray near a photon orbit goes to the FP64 pass before its first attempt
        if constexpr (SPLIT) {
            if (sl.R.i == 0 && sl.crit) {
                if (ham_flag(a, sl, cnt)) { sl.busy = false; sl.need = true; }
                continue;
            }
        }
        // the loop bound of trace_RKF (l < 1000, solver.cuh:158) and the attempt counter
        if (!(sl.R.l < T(1000))) {
            const V4<T> u = ham_velocity<T>(sl.R.P.x, sl.R.P.y, sl.R.W.x, sl.R.Q.x, sl.R.Q.y, sl.R.W.y, sl.c);
            if (ham_finish<T, SPLIT, EMIS>(a, sl, PRR_RESULT_INFINITE_GEO, {0.f, 0.f, 0.f}, u, cnt)) { sl.busy = false; sl.need = true; }
            continue;
        }
        sl.R.i += 1;
        const HamStep<T> st = ham_stages<T>(sl.R, sl.c, sl.q);
        int result = 0;
        V3<float> col;
        V4<T> u;
        const int r = ham_accept<T, EMIS>(a.frames[sl.frame], sl, sl.R, st, result, col, u);
        if (r == STEP_CONTINUE) continue;
        bool done;
        if constexpr (SPLIT) done = r == STEP_FLAG64 ? ham_flag(a, sl, cnt) : ham_finish<T, SPLIT, EMIS>(a, sl, result, col, u, cnt);
        else done = ham_finish<T, SPLIT, EMIS>(a, sl, result, col, u, cnt);
        if (done) { sl.busy = false; sl.need = true; }
    }
    warp_sum_add_h(&a.counters[C_ATTEMPTS], cnt.att);
    warp_sum_add_h(&a.counters[C_ACCEPTED], cnt.acc);
    warp_sum_add_h(&a.counters[C_RAYS], cnt.rays);
    warp_sum_add_h(&a.counters[C_ESCAPED], cnt.esc);
    warp_sum_add_h(&a.counters[C_CAPTURED], cnt.cap);
    warp_sum_add_h(&a.counters[C_INTERSECTION], cnt.hit);
    warp_sum_add_h(&a.counters[C_INFINITE], cnt.inf);
    warp_sum_add_h(&a.counters[C_MATH_ERROR], cnt.nan);
    if (SPLIT) warp_sum_add_h(&a.counters[C_FP64], cnt.f64);
}

// FP64 re-integration, in Hamiltonian form, of the rays a split-precision
// FP32 pass queued (k_fp64_requeue's job for the (x, u) form): each queued
// ray is integrated again from the camera in FP64 and its per-sample colour
// overwritten; it is counted as a ray here.  64-thread CTAs built for the
// FP64 renderer's occupancy.
template <int MAXT, int MINB> __global__ void __launch_bounds__(MAXT, MINB) k_ham_requeue(PersistentArgs a)
{
    const int lane = threadIdx.x & 31;
    bool busy = false, need = true;
    HSlot<double> sl;
    sl.busy = false; sl.need = false; sl.crit = false; sl.flag_r = -1.0f;
    sl.frame = 0; sl.px = sl.py = sl.s = 0; sl.S = 1;
    sl.acc0 = sl.acc1 = sl.acc2 = 0.f;
    long long rid = 0;
    HCounts cnt;
    long long nq = (long long)*(volatile unsigned long long *)&a.counters[C_FP64_QUEUED];
    if (nq > a.fp64_capacity) nq = a.fp64_capacity;
    while (true) {
        const unsigned needmask = __ballot_sync(FULL, need);
        if (needmask) {
            const int leader = __ffs(needmask) - 1;
            unsigned long long base = 0;
            if (lane == leader) base = atomicAdd(&a.counters[C_WORK_FP64], (unsigned long long)__popc(needmask));
            base = __shfl_sync(FULL, base, leader);
            if (need) {
                const long long it = (long long)base + __popc(needmask & ((1u << lane) - 1));
                need = false;
                busy = false;
                if (it < nq) {
                    const unsigned long long e = a.fp64_queue[it];
                    sl.frame = (int)(e >> 40);
                    rid = (long long)(e & ((1ull << 40) - 1));
                    const FrameParams &fp = a.frames[sl.frame];
                    const long long pix = rid / fp.samples;
                    sl.s = (int)(rid - pix * fp.samples);
                    sl.px = (int)(pix % fp.width);
                    sl.py = (int)(pix / fp.width);
                    sl.S = fp.samples;
                    sl.q = make_hot<double>(fp);
                    ham_init<double, false, false>(fp, sl, sl.s);
                    busy = true;
                }
            }
        }
        if (__ballot_sync(FULL, busy) == 0) break;
        if (!busy) continue;
        const FrameParams &fp = a.frames[sl.frame];
        int result = 0;
        V3<float> col = {0.f, 0.f, 0.f};
        if (sl.R.l < 1000.0) {  // the loop bound of trace_RKF (solver.cuh:158)
            sl.R.i += 1;
            const HamStep<double> st = ham_stages<double>(sl.R, sl.c, sl.q);
            V4<double> u;
            if (ham_accept<double, false>(fp, sl, sl.R, st, result, col, u) == STEP_CONTINUE) continue;
        } else {
            result = PRR_RESULT_INFINITE_GEO;
        }
        cnt.att += (unsigned)sl.R.i;
        cnt.acc += (unsigned)sl.R.accepted;
        cnt.rays++;
        if (result == PRR_RESULT_SUCCESS) {
            if (metric_radius<double>(fp, sl.R.P.x, sl.R.P.y, sl.R.W.x) >= sl.q.rout) cnt.esc++; else cnt.cap++;
        } else if (result == PRR_RESULT_INTERSECTION) cnt.hit++;
        else if (result == PRR_RESULT_INFINITE_GEO) cnt.inf++;
        else cnt.nan++;
        float *o = a.sample_rgb + 3 * (fp.ray_begin + rid);
        o[0] = col.x; o[1] = col.y; o[2] = col.z;
        busy = false;
        need = true;
    }
    warp_sum_add_h(&a.counters[C_ATTEMPTS], cnt.att);
    warp_sum_add_h(&a.counters[C_ACCEPTED], cnt.acc);
    warp_sum_add_h(&a.counters[C_RAYS], cnt.rays);
    warp_sum_add_h(&a.counters[C_ESCAPED], cnt.esc);
    warp_sum_add_h(&a.counters[C_CAPTURED], cnt.cap);
    warp_sum_add_h(&a.counters[C_INTERSECTION], cnt.hit);
    warp_sum_add_h(&a.counters[C_INFINITE], cnt.inf);
    warp_sum_add_h(&a.counters[C_MATH_ERROR], cnt.nan);
}

cudaError_t launch_ham_requeue(const PersistentArgs &a, int nsm, cudaStream_t st)
{
    int bpsm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bpsm, k_ham_requeue<64, ham_small_minb<double>()>, 64, 0);
    if (e != cudaSuccess) return e;
    k_ham_requeue<64, ham_small_minb<double>()><<<nsm * (bpsm > 0 ? bpsm : 1), 64, 0, st>>>(a);
    return cudaGetLastError();
}

template <class T, bool SPLIT, bool EMIS> static cudaError_t ham_launch(const PersistentArgs &a, int block, int grid, cudaStream_t st)
{
    if (block <= 64) k_ham<T, 64, ham_small_minb<T>(), SPLIT, EMIS><<<grid, block, 0, st>>>(a);
    else k_ham<T, 256, 1, SPLIT, EMIS><<<grid, block, 0, st>>>(a);
    return cudaGetLastError();
}

template <class T, bool SPLIT, bool EMIS> static int ham_occ(int block)
{
    int n = 0;
    cudaError_t e = block <= 64
                        ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_ham<T, 64, ham_small_minb<T>(), SPLIT, EMIS>, block, 0)
                        : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_ham<T, 256, 1, SPLIT, EMIS>, block, 0);
    if (e != cudaSuccess) { cudaGetLastError(); return 0; }
    return n;
}

cudaError_t launch_ham(const PersistentArgs &a, int precision, bool split, int block, int blocks_per_sm, int nsm,
                       cudaStream_t st)
{
    if (block < 32 || block > 256 || block % 32) return cudaErrorInvalidValue;
    if (split && (precision != PRR_PREC_FP32 || !a.sample_rgb || !a.fp64_queue)) return cudaErrorInvalidValue;
    if (split && a.emission) return cudaErrorInvalidValue;
    int grid = nsm * blocks_per_sm;
    if (grid < 1) grid = 1;
    if (precision == PRR_PREC_FP64) {
        if (a.emission) return ham_launch<double, false, true>(a, block, grid, st);
        return ham_launch<double, false, false>(a, block, grid, st);
    }
    if (split) return ham_launch<float, true, false>(a, block, grid, st);
    if (a.emission) return ham_launch<float, false, true>(a, block, grid, st);
    return ham_launch<float, false, false>(a, block, grid, st);
}

int ham_occupancy(int precision, int block, bool split, bool emission)
{
    if (precision == PRR_PREC_FP64) return emission ? ham_occ<double, false, true>(block) : ham_occ<double, false, false>(block);
    if (split) return ham_occ<float, true, false>(block);
    if (emission) return ham_occ<float, false, true>(block);
    return ham_occ<float, false, false>(block);
}

}  // namespace prr
