// phys_pair.cuh - the FP32 RKF45 stages of one ray (V = float) or of two
// rays at once (V = float2: component x is one ray, y the other) with
// Blackwell's paired FP32 instructions (__ffma2_rn, __fadd2_rn, __fmul2_rn
// issue two FP32 results per instruction).  The tracing kernel is
// instruction-issue bound, and the six geodesic evaluations plus the stage
// combinations are two thirds of its instructions; pairing two lanes' worth
// of rays halves their issue cost.
//
// Every operation is written out (no compiler contraction) and the scalar and
// paired forms use the same operation sequence; the transcendental steps
// (reciprocal, reciprocal square root, power) run per component on the SFU
// through the same functions in both forms.  The paired instructions may
// treat subnormal intermediates differently, so the two forms agree to the
// last bits, not always bit for bit.
//
// Mathematics: as geod_ks (prr_device.cuh) and phys_attempt (phys_stepper.cuh).
#pragma once
#include "phys_stepper.cuh"

// One-ray stages (stages_xy) evaluate the geodesic with its x/y twins paired
// (geod_xy) unless built with PRR_GEOD_XY=0 (the all-scalar geod).
#ifndef PRR_GEOD_XY
#define PRR_GEOD_XY 1
#endif

namespace prr {
namespace pv {

// ---- lane-value operations ----
PRR_DEV float splat(float c, float) { return c; }
PRR_DEV float2 splat(float c, float2) { return make_float2(c, c); }
PRR_DEV float fma_(float a, float b, float c) { return __fmaf_rn(a, b, c); }
PRR_DEV float2 fma_(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
PRR_DEV float add_(float a, float b) { return __fadd_rn(a, b); }
PRR_DEV float2 add_(float2 a, float2 b) { return __fadd2_rn(a, b); }
PRR_DEV float mul_(float a, float b) { return __fmul_rn(a, b); }
PRR_DEV float2 mul_(float2 a, float2 b) { return __fmul2_rn(a, b); }
PRR_DEV float rsq_(float a) { return frsqrt<float>(a); }
PRR_DEV float2 rsq_(float2 a) { return make_float2(frsqrt<float>(a.x), frsqrt<float>(a.y)); }
PRR_DEV float rcp_(float a) { return frcp<float>(a); }
PRR_DEV float2 rcp_(float2 a) { return make_float2(frcp<float>(a.x), frcp<float>(a.y)); }
PRR_DEV float abs_(float a) { return fabsf(a); }
PRR_DEV float2 abs_(float2 a) { return make_float2(fabsf(a.x), fabsf(a.y)); }
PRR_DEV float max_(float a, float b) { return fmaxf(a, b); }
PRR_DEV float2 max_(float2 a, float2 b) { return make_float2(fmaxf(a.x, b.x), fmaxf(a.y, b.y)); }
PRR_DEV float min_(float a, float b) { return fminf(a, b); }
PRR_DEV float2 min_(float2 a, float2 b) { return make_float2(fminf(a.x, b.x), fminf(a.y, b.y)); }
PRR_DEV float pow_(float b, float e) { return fpow<float>(b, e); }
// negation is exact; in an operand of the next instruction it folds into a sign modifier
PRR_DEV float neg_(float a) { return -a; }
PRR_DEV float2 neg_(float2 a) { return make_float2(-a.x, -a.y); }
PRR_DEV float2 pow_(float2 b, float2 e) { return make_float2(fpow<float>(b.x, e.x), fpow<float>(b.y, e.y)); }

template <class V> struct Vec4 { V x, y, z, w; };

// Kerr-Schild geodesic acceleration du/dlambda = -Gamma u u (see geod_ks for
// the derivation); M = 0 gives flat space.  (Inlined at each stage: one
// out-of-line copy called six times measured 2 % slower.)
template <class V> PRR_DEV Vec4<V> geod(const Vec4<V> &p, const Vec4<V> &u, V Mass, V a)
{
    const V c05 = splat(0.5f, V{}), c2 = splat(2.0f, V{}), c3 = splat(3.0f, V{}), c4 = splat(4.0f, V{}),
            m1 = splat(-1.0f, V{}), m2 = splat(-2.0f, V{}), m4 = splat(-4.0f, V{});
    const V X = p.x, Y = p.y, Z = p.z;
    const V a2 = mul_(a, a), Z2 = mul_(Z, Z);
    const V R2 = fma_(X, X, fma_(Y, Y, Z2));
    const V b = fma_(m1, a2, R2);
    const V S2 = fma_(b, b, mul_(mul_(c4, a2), Z2));
    const V iS = rsq_(S2);
    const V S = mul_(S2, iS);
    const V r2 = mul_(c05, add_(b, S));
    const V ir = rsq_(r2);
    const V r = mul_(r2, ir);
    const V q = add_(r2, a2), iq = rcp_(q);
    const V Sig = fma_(r2, r2, mul_(a2, Z2)), iSig = rcp_(Sig);
    // radius gradient
    const V rS = mul_(r, iS);
    const V drx = mul_(X, rS), dry = mul_(Y, rS), drz = mul_(mul_(Z, q), mul_(iS, ir));
    // f and its gradient
    const V r3 = mul_(r2, r);
    const V f = mul_(mul_(mul_(c2, Mass), r3), iSig);
    const V c1 = mul_(f, fma_(mul_(m4, r3), iSig, mul_(c3, ir)));
    const V dfx = mul_(c1, drx), dfy = mul_(c1, dry);
    const V dfz = fma_(c1, drz, mul_(mul_(m2, f), mul_(a2, mul_(Z, iSig))));
    // null vector l (l_t = 1)
    const V lx = mul_(fma_(r, X, mul_(a, Y)), iq);
    const V ly = mul_(fma_(r, Y, neg_(mul_(a, X))), iq);
    const V lz = mul_(Z, ir);
    // directional derivatives along the spatial velocity
    const V ux = u.x, uy = u.y, uz = u.z, ut = u.w;
    const V Dr = fma_(ux, drx, fma_(uy, dry, mul_(uz, drz)));
    const V nDq = mul_(mul_(m2, r), Dr);
    const V Dlx = mul_(fma_(Dr, X, fma_(r, ux, fma_(a, uy, mul_(lx, nDq)))), iq);
    const V Dly = mul_(fma_(Dr, Y, fma_(r, uy, fma_(neg_(a), ux, mul_(ly, nDq)))), iq);
    const V Dlz = mul_(fma_(neg_(lz), Dr, uz), ir);
    const V Df = fma_(ux, dfx, fma_(uy, dfy, mul_(uz, dfz)));
    const V L = fma_(lx, ux, fma_(ly, uy, fma_(lz, uz, ut)));
    const V DL = fma_(ux, Dlx, fma_(uy, Dly, mul_(uz, Dlz)));
    // gradient of L at fixed u
    const V P0 = fma_(mul_(m2, r), fma_(ux, lx, mul_(uy, ly)), fma_(ux, X, mul_(uy, Y)));
    const V P = fma_(P0, iq, neg_(mul_(uz, mul_(lz, ir))));
    const V dLx = fma_(drx, P, mul_(fma_(r, ux, neg_(mul_(a, uy))), iq));
    const V dLy = fma_(dry, P, mul_(fma_(a, ux, mul_(r, uy)), iq));
    const V dLz = fma_(drz, P, mul_(uz, ir));
    // lowered contraction, then raise with g^{-1} = eta - f l l
    const V A = fma_(L, Df, mul_(f, DL));
    const V fL = mul_(f, L);
    const V nhL2 = mul_(mul_(splat(-0.5f, V{}), L), L);
    const V Gx = fma_(lx, A, fma_(fL, Dlx, fma_(nhL2, dfx, neg_(mul_(fL, dLx)))));
    const V Gy = fma_(ly, A, fma_(fL, Dly, fma_(nhL2, dfy, neg_(mul_(fL, dLy)))));
    const V Gz = fma_(lz, A, fma_(fL, Dlz, fma_(nhL2, dfz, neg_(mul_(fL, dLz)))));
    const V Lam = fma_(lx, Gx, fma_(ly, Gy, fma_(lz, Gz, neg_(A))));
    const V fLam = mul_(f, Lam);
    return {fma_(fLam, lx, neg_(Gx)), fma_(fLam, ly, neg_(Gy)), fma_(fLam, lz, neg_(Gz)), fma_(m1, fLam, A)};
}

PRR_DEV float2 f2(float a, float b) { return make_float2(a, b); }
PRR_DEV float2 sp(float a) { return make_float2(a, a); }

// FP64 lane values and pairs, so code written on (pair, scalar) values
// builds in both precisions (k_ham.cu); FP64 has no paired instructions, so
// a double2 operation is two scalar ones.
PRR_DEV double fma_(double a, double b, double c) { return __fma_rn(a, b, c); }
PRR_DEV double add_(double a, double b) { return __dadd_rn(a, b); }
PRR_DEV double mul_(double a, double b) { return __dmul_rn(a, b); }
PRR_DEV double rsq_(double a) { return frsqrt<double>(a); }
PRR_DEV double rcp_(double a) { return frcp<double>(a); }
PRR_DEV double abs_(double a) { return fabs(a); }
PRR_DEV double max_(double a, double b) { return fmax(a, b); }
PRR_DEV double min_(double a, double b) { return fmin(a, b); }
PRR_DEV double pow_(double b, double e) { return fpow<double>(b, e); }
PRR_DEV double neg_(double a) { return -a; }
PRR_DEV double2 f2(double a, double b) { return make_double2(a, b); }
PRR_DEV double2 sp(double a) { return make_double2(a, a); }
PRR_DEV double2 fma_(double2 a, double2 b, double2 c) { return make_double2(__fma_rn(a.x, b.x, c.x), __fma_rn(a.y, b.y, c.y)); }
PRR_DEV double2 add_(double2 a, double2 b) { return make_double2(__dadd_rn(a.x, b.x), __dadd_rn(a.y, b.y)); }
PRR_DEV double2 mul_(double2 a, double2 b) { return make_double2(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)); }
PRR_DEV double2 abs_(double2 a) { return make_double2(fabs(a.x), fabs(a.y)); }
PRR_DEV double2 max_(double2 a, double2 b) { return make_double2(fmax(a.x, b.x), fmax(a.y, b.y)); }
PRR_DEV double2 rcp_(double2 a) { return make_double2(frcp<double>(a.x), frcp<double>(a.y)); }
PRR_DEV double2 neg_(double2 a) { return make_double2(-a.x, -a.y); }

// the pair type of a lane type
template <class T> struct PairOf;
template <> struct PairOf<float> { using type = float2; };
template <> struct PairOf<double> { using type = double2; };
template <class T> using P2 = typename PairOf<T>::type;

// geod<float> with the x and y components of one ray paired: P = (X, Y) and
// U = (u^x, u^y) in, (du^x, du^y) in gxy and du^z, du^t in gz, gt out.  The
// operations are geod's, one for one and in its order; where geod applies
// the same operation to an x and a y quantity (gradients, l, D l, the
// lowered contraction, the raise) one paired instruction does both, and the
// rest (scalars and dot products) stays scalar.
PRR_DEV void geod_xy(float2 P, float Z, float2 U, float uz, float ut, float Mass, float a, float2 &gxy, float &gz,
                     float &gt)
{
    const float X = P.x, Y = P.y, ux = U.x, uy = U.y;
    const float a2 = mul_(a, a), Z2 = mul_(Z, Z);
    const float R2 = fma_(X, X, fma_(Y, Y, Z2));
    const float b = fma_(-1.0f, a2, R2);
    const float S2 = fma_(b, b, mul_(mul_(4.0f, a2), Z2));
    const float iS = rsq_(S2);
    const float S = mul_(S2, iS);
    const float r2 = mul_(0.5f, add_(b, S));
    const float ir = rsq_(r2);
    const float r = mul_(r2, ir);
    const float q = add_(r2, a2), iq = rcp_(q);
    const float Sig = fma_(r2, r2, mul_(a2, Z2)), iSig = rcp_(Sig);
    const float2 r_ = sp(r), iq_ = sp(iq);
    // radius gradient
    const float rS = mul_(r, iS);
    const float2 dr = mul_(P, sp(rS));
    const float drz = mul_(mul_(Z, q), mul_(iS, ir));
    // f and its gradient
    const float r3 = mul_(r2, r);
    const float f = mul_(mul_(mul_(2.0f, Mass), r3), iSig);
    const float c1 = mul_(f, fma_(mul_(-4.0f, r3), iSig, mul_(3.0f, ir)));
    const float2 df = mul_(sp(c1), dr);
    const float dfz = fma_(c1, drz, mul_(mul_(-2.0f, f), mul_(a2, mul_(Z, iSig))));
    // null vector l (l_t = 1)
    const float2 l = mul_(fma_(r_, P, f2(mul_(a, Y), neg_(mul_(a, X)))), iq_);
    const float lz = mul_(Z, ir);
    // directional derivatives along the spatial velocity
    const float Dr = fma_(ux, dr.x, fma_(uy, dr.y, mul_(uz, drz)));
    const float nDq = mul_(mul_(-2.0f, r), Dr);
    const float2 w = mul_(l, sp(nDq));
    const float2 Dl = mul_(fma_(sp(Dr), P, fma_(r_, U, f2(fma_(a, uy, w.x), fma_(neg_(a), ux, w.y)))), iq_);
    const float Dlz = mul_(fma_(neg_(lz), Dr, uz), ir);
    const float Df = fma_(ux, df.x, fma_(uy, df.y, mul_(uz, dfz)));
    const float L = fma_(l.x, ux, fma_(l.y, uy, fma_(lz, uz, ut)));
    const float DL = fma_(ux, Dl.x, fma_(uy, Dl.y, mul_(uz, Dlz)));
    // gradient of L at fixed u
    const float P0 = fma_(mul_(-2.0f, r), fma_(ux, l.x, mul_(uy, l.y)), fma_(ux, X, mul_(uy, Y)));
    const float Pp = fma_(P0, iq, neg_(mul_(uz, mul_(lz, ir))));
    const float2 dL = fma_(dr, sp(Pp), mul_(f2(fma_(r, ux, neg_(mul_(a, uy))), fma_(a, ux, mul_(r, uy))), iq_));
    const float dLz = fma_(drz, Pp, mul_(uz, ir));
    // lowered contraction, then raise with g^{-1} = eta - f l l
    const float A = fma_(L, Df, mul_(f, DL));
    const float fL = mul_(f, L);
    const float nhL2 = mul_(mul_(-0.5f, L), L);
    const float2 G = fma_(l, sp(A), fma_(sp(fL), Dl, fma_(sp(nhL2), df, neg_(mul_(sp(fL), dL)))));
    const float Gz = fma_(lz, A, fma_(fL, Dlz, fma_(nhL2, dfz, neg_(mul_(fL, dLz)))));
    const float Lam = fma_(l.x, G.x, fma_(l.y, G.y, fma_(lz, Gz, neg_(A))));
    const float fLam = mul_(f, Lam);
    gxy = fma_(sp(fLam), l, neg_(G));
    gz = fma_(fLam, lz, neg_(Gz));
    gt = fma_(-1.0f, fLam, A);
}

template <class V> PRR_DEV Vec4<V> scl(V h, const Vec4<V> &g) { return {mul_(h, g.x), mul_(h, g.y), mul_(h, g.z), mul_(h, g.w)}; }

// Per-ray inputs and outputs of the stage evaluation.
template <class V> struct StageIn {
    Vec4<V> x, u;
    V h, M, a, rtol, atol, hmin, hmax;
};
template <class V> struct StageOut {
    V dx[4], du[4], err, hn;
};

// The six Fehlberg stages, the 4th-order increments, the scaled error norm
// max_i |y5_i - y4_i| / (atol + rtol max(|y_i|, |y4_i|)) and the next step
// 0.9 h err^(-1/5) clamped to [hmin, hmax].  Position stages are linear in
// the velocity stages (phys_stepper.cuh); only the k's are kept.
template <class V> PRR_DEV StageOut<V> stages(const StageIn<V> &in)
{
    using F = Fehlberg;
    const V h = in.h;
    const Vec4<V> &x = in.x, &u = in.u;
#define PRR_C(v) splat((float)(v), V{})
#define PRR_EACH(OP) OP(x) OP(y) OP(z) OP(w)
    Vec4<V> zx, zu;
    const Vec4<V> k1 = scl(h, geod(x, u, in.M, in.a));
#define S2(c) zx.c = fma_(h, mul_(PRR_C(F::c2), u.c), x.c); zu.c = fma_(PRR_C(F::A21), k1.c, u.c);
    PRR_EACH(S2)
#undef S2
    const Vec4<V> k2 = scl(h, geod(zx, zu, in.M, in.a));
#define S3(c)                                                                                                      \
    zx.c = fma_(h, fma_(PRR_C(F::c3), u.c, mul_(PRR_C(F::B31), k1.c)), x.c);                                   \
    zu.c = fma_(PRR_C(F::A32), k2.c, fma_(PRR_C(F::A31), k1.c, u.c));
    PRR_EACH(S3)
#undef S3
    const Vec4<V> k3 = scl(h, geod(zx, zu, in.M, in.a));
#define S4(c)                                                                                                      \
    zx.c = fma_(h, fma_(PRR_C(F::c4), u.c, fma_(PRR_C(F::B42), k2.c, mul_(PRR_C(F::B41), k1.c))), x.c);       \
    zu.c = fma_(PRR_C(F::A43), k3.c, fma_(PRR_C(F::A42), k2.c, fma_(PRR_C(F::A41), k1.c, u.c)));
    PRR_EACH(S4)
#undef S4
    const Vec4<V> k4 = scl(h, geod(zx, zu, in.M, in.a));
#define S5(c)                                                                                                      \
    zx.c = fma_(h, fma_(PRR_C(F::c5), u.c, fma_(PRR_C(F::B53), k3.c, fma_(PRR_C(F::B52), k2.c,                 \
                                                                         mul_(PRR_C(F::B51), k1.c)))), x.c);      \
    zu.c = fma_(PRR_C(F::A54), k4.c, fma_(PRR_C(F::A53), k3.c, fma_(PRR_C(F::A52), k2.c, fma_(PRR_C(F::A51), k1.c, u.c))));
    PRR_EACH(S5)
#undef S5
    const Vec4<V> k5 = scl(h, geod(zx, zu, in.M, in.a));
#define S6(c)                                                                                                      \
    zx.c = fma_(h, fma_(PRR_C(F::c6), u.c, fma_(PRR_C(F::B64), k4.c, fma_(PRR_C(F::B63), k3.c,                 \
                fma_(PRR_C(F::B62), k2.c, mul_(PRR_C(F::B61), k1.c))))), x.c);                                    \
    zu.c = fma_(PRR_C(F::A65), k5.c, fma_(PRR_C(F::A64), k4.c, fma_(PRR_C(F::A63), k3.c,                         \
                fma_(PRR_C(F::A62), k2.c, fma_(PRR_C(F::A61), k1.c, u.c)))));
    PRR_EACH(S6)
#undef S6
    const Vec4<V> k6 = scl(h, geod(zx, zu, in.M, in.a));

    StageOut<V> o;
    V err = splat(0.0f, V{});
#define FIN(c, j)                                                                                                  \
    {                                                                                                              \
        const V du = fma_(PRR_C(F::K45), k5.c, fma_(PRR_C(F::K44), k4.c, fma_(PRR_C(F::K43), k3.c,               \
                                                                              mul_(PRR_C(F::K41), k1.c))));       \
        const V dx = mul_(h, fma_(PRR_C(F::b4), k4.c, fma_(PRR_C(F::b3), k3.c, fma_(PRR_C(F::b2), k2.c,          \
                                                                                fma_(PRR_C(F::b1), k1.c, u.c))))); \
        const V eu = fma_(PRR_C(F::E6), k6.c, fma_(PRR_C(F::E5), k5.c, fma_(PRR_C(F::E4), k4.c,                  \
                                                                            fma_(PRR_C(F::E3), k3.c, mul_(PRR_C(F::E1), k1.c))))); \
        const V ex = mul_(h, fma_(PRR_C(F::e5), k5.c, fma_(PRR_C(F::e4), k4.c, fma_(PRR_C(F::e3), k3.c,          \
                                                                                fma_(PRR_C(F::e2), k2.c, mul_(PRR_C(F::e1), k1.c)))))); \
        const V sx = fma_(in.rtol, max_(abs_(x.c), abs_(add_(x.c, dx))), in.atol);                               \
        const V su = fma_(in.rtol, max_(abs_(u.c), abs_(add_(u.c, du))), in.atol);                               \
        err = max_(err, max_(mul_(abs_(ex), rcp_(sx)), mul_(abs_(eu), rcp_(su))));                                \
        o.dx[j] = dx;                                                                                              \
        o.du[j] = du;                                                                                              \
    }
    FIN(x, 0) FIN(y, 1) FIN(z, 2) FIN(w, 3)
#undef FIN
#undef PRR_EACH
#undef PRR_C
    o.err = err;
    const V hn = mul_(mul_(splat(0.9f, V{}), h), pow_(err, splat(-0.2f, V{})));
    o.hn = min_(max_(hn, in.hmin), in.hmax);
    return o;
}

// One ray with its 4-vector components paired, (x, y) and (z, t), on the
// paired instructions: the stage combinations, the increments and the error
// estimate are component-wise, so half of their instructions go away; the
// geodesic stays scalar (its operands mix components).  Same mathematics as
// stages<float>; rounding differs in the last bits.

PRR_DEV StageOut<float> stages_xy(const StageIn<float> &in)
{
    using F = Fehlberg;
    const float h = in.h;
    const float2 H = sp(h);
    const float2 x01 = f2(in.x.x, in.x.y), x23 = f2(in.x.z, in.x.w);
    const float2 u01 = f2(in.u.x, in.u.y), u23 = f2(in.u.z, in.u.w);
#define PC(v) sp((float)(v))
    // k_i = h G(z_i), held as pairs
#if PRR_GEOD_XY
#define GEOD(Kp, Kq, zx01, zx23, zu01, zu23)                                                                           \
    {                                                                                                                  \
        float2 gxy;                                                                                                    \
        float gz, gt;                                                                                                  \
        geod_xy(zx01, zx23.x, zu01, zu23.x, zu23.y, in.M, in.a, gxy, gz, gt);                                          \
        Kp = mul_(H, gxy);                                                                                             \
        Kq = mul_(H, f2(gz, gt));                                                                                      \
    }
#else
#define GEOD(Kp, Kq, zx01, zx23, zu01, zu23)                                                                           \
    {                                                                                                                  \
        const Vec4<float> g = geod<float>({zx01.x, zx01.y, zx23.x, 0.0f}, {zu01.x, zu01.y, zu23.x, zu23.y}, in.M, in.a); \
        Kp = mul_(H, f2(g.x, g.y));                                                                                    \
        Kq = mul_(H, f2(g.z, g.w));                                                                                    \
    }
#endif
    float2 k1p, k1q, k2p, k2q, k3p, k3q, k4p, k4q, k5p, k5q, k6p, k6q;
    float2 zxp, zxq, zup, zuq;
    GEOD(k1p, k1q, x01, x23, u01, u23)
    zxp = fma_(H, mul_(PC(F::c2), u01), x01); zxq = fma_(H, mul_(PC(F::c2), u23), x23);
    zup = fma_(PC(F::A21), k1p, u01); zuq = fma_(PC(F::A21), k1q, u23);
    GEOD(k2p, k2q, zxp, zxq, zup, zuq)
    zxp = fma_(H, fma_(PC(F::c3), u01, mul_(PC(F::B31), k1p)), x01);
    zxq = fma_(H, fma_(PC(F::c3), u23, mul_(PC(F::B31), k1q)), x23);
    zup = fma_(PC(F::A32), k2p, fma_(PC(F::A31), k1p, u01));
    zuq = fma_(PC(F::A32), k2q, fma_(PC(F::A31), k1q, u23));
    GEOD(k3p, k3q, zxp, zxq, zup, zuq)
    zxp = fma_(H, fma_(PC(F::c4), u01, fma_(PC(F::B42), k2p, mul_(PC(F::B41), k1p))), x01);
    zxq = fma_(H, fma_(PC(F::c4), u23, fma_(PC(F::B42), k2q, mul_(PC(F::B41), k1q))), x23);
    zup = fma_(PC(F::A43), k3p, fma_(PC(F::A42), k2p, fma_(PC(F::A41), k1p, u01)));
    zuq = fma_(PC(F::A43), k3q, fma_(PC(F::A42), k2q, fma_(PC(F::A41), k1q, u23)));
    GEOD(k4p, k4q, zxp, zxq, zup, zuq)
    zxp = fma_(H, fma_(PC(F::c5), u01, fma_(PC(F::B53), k3p, fma_(PC(F::B52), k2p, mul_(PC(F::B51), k1p)))), x01);
    zxq = fma_(H, fma_(PC(F::c5), u23, fma_(PC(F::B53), k3q, fma_(PC(F::B52), k2q, mul_(PC(F::B51), k1q)))), x23);
    zup = fma_(PC(F::A54), k4p, fma_(PC(F::A53), k3p, fma_(PC(F::A52), k2p, fma_(PC(F::A51), k1p, u01))));
    zuq = fma_(PC(F::A54), k4q, fma_(PC(F::A53), k3q, fma_(PC(F::A52), k2q, fma_(PC(F::A51), k1q, u23))));
    GEOD(k5p, k5q, zxp, zxq, zup, zuq)
    zxp = fma_(H, fma_(PC(F::c6), u01, fma_(PC(F::B64), k4p, fma_(PC(F::B63), k3p, fma_(PC(F::B62), k2p,
                                                                                       mul_(PC(F::B61), k1p))))), x01);
    zxq = fma_(H, fma_(PC(F::c6), u23, fma_(PC(F::B64), k4q, fma_(PC(F::B63), k3q, fma_(PC(F::B62), k2q,
                                                                                       mul_(PC(F::B61), k1q))))), x23);
    zup = fma_(PC(F::A65), k5p, fma_(PC(F::A64), k4p, fma_(PC(F::A63), k3p, fma_(PC(F::A62), k2p,
                                                                                fma_(PC(F::A61), k1p, u01)))));
    zuq = fma_(PC(F::A65), k5q, fma_(PC(F::A64), k4q, fma_(PC(F::A63), k3q, fma_(PC(F::A62), k2q,
                                                                                fma_(PC(F::A61), k1q, u23)))));
    GEOD(k6p, k6q, zxp, zxq, zup, zuq)
#undef GEOD
    StageOut<float> o;
    float2 err2 = sp(0.0f);
    const float2 rtol = sp(in.rtol), atol = sp(in.atol);
#define FIN(kk, xx, uu, j0)                                                                                            {                                                                                                                      const float2 du = fma_(PC(F::K45), k5##kk, fma_(PC(F::K44), k4##kk, fma_(PC(F::K43), k3##kk,                                                                                               mul_(PC(F::K41), k1##kk))));            const float2 dx = mul_(H, fma_(PC(F::b4), k4##kk, fma_(PC(F::b3), k3##kk, fma_(PC(F::b2), k2##kk,                                                                                          fma_(PC(F::b1), k1##kk, uu)))));         const float2 eu = fma_(PC(F::E6), k6##kk, fma_(PC(F::E5), k5##kk, fma_(PC(F::E4), k4##kk,                                                                                                fma_(PC(F::E3), k3##kk, mul_(PC(F::E1), k1##kk)))));         const float2 ex = mul_(H, fma_(PC(F::e5), k5##kk, fma_(PC(F::e4), k4##kk, fma_(PC(F::e3), k3##kk,                                                                                          fma_(PC(F::e2), k2##kk, mul_(PC(F::e1), k1##kk))))));         const float2 sx = fma_(rtol, max_(abs_(xx), abs_(add_(xx, dx))), atol);                                            const float2 su = fma_(rtol, max_(abs_(uu), abs_(add_(uu, du))), atol);                                            err2 = max_(err2, max_(mul_(abs_(ex), rcp_(sx)), mul_(abs_(eu), rcp_(su))));                                       o.dx[j0] = dx.x; o.dx[j0 + 1] = dx.y;                                                                              o.du[j0] = du.x; o.du[j0 + 1] = du.y;                                                                          }
    FIN(p, x01, u01, 0)
    FIN(q, x23, u23, 2)
#undef FIN
#undef PC
    const float err = fmaxf(err2.x, err2.y);
    o.err = err;
    const float hn = mul_(mul_(0.9f, h), pow_(err, -0.2f));
    o.hn = min_(max_(hn, in.hmin), in.hmax);
    return o;
}

// Lane value of slot j (0 = x component, 1 = y) and back.
PRR_DEV float get(float v, int) { return v; }
PRR_DEV float get(float2 v, int j) { return j ? v.y : v.x; }

}  // namespace pv
}  // namespace prr
