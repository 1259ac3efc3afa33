// prr_oracle.cpp - CPU restatement of the ParRelRay hot path.
//
// TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
// bench's cpu_baseline leg may load this library; the product never does.
//
// Two integration modes, selected by prr_frame_desc::mode:
//  * PRR_MODE_REFERENCE: the reference algorithm restated in FP32 with the
//    reference's operation order and its quirks, so that it reproduces the
//    reference build (oracle/_ref) bit for bit on the same compiler flags.
//    Pinned by tests/test_oracle_golden.py (fixtures made by the reference
//    host build, and live runs of it where the reference tree is present).
//  * PRR_MODE_PHYSICAL: textbook RKF45 / Euler, null initial data, mixed
//    abs/rel error control, in FP32 or FP64.  The geodesic right-hand side is
//    the full Christoffel table of the Kerr-Schild metric (independent of the
//    GPU's restructured contraction).
//
// Reference correspondence (paths relative to the reference project):
//   ray placement        kernels/ssaa.cuh:36-48 (regular), 92-99 (none)
//   ray direction        main/Camera.h:39-42 (rayDir_Spherical)
//   initial momentum     kernels/solver.cuh:26-56 (initRays)
//   Euler                kernels/solver.cuh:68-116 (trace_Euler)
//   RKF45                kernels/solver.cuh:124-219 (tableau + trace_RKF)
//   Schwarzschild        metrics/schwarzschild.cuh:55-141 (hooks, getGeod, getMetric)
//   flat                 metrics/flat.cuh:55-99
//   colour               metrics/schwarzschild.cuh:151-183 (rayToRGB)
//   sphere hit / colour  scene/sphere.h:34-64, main/Spacetime.h:38-46
//   texture sampling     cudamaths/tex2d.cuh:112-131
//   background           main/base.h:119-162 (getColorDefault2), cudamaths/f3.cuh:101-103
//   SSAA combine / FXAA  kernels/ssaa.cuh:109-131, 141-181
//   plasma emission      the model of prr_emission (include/prr.h) for the
//                        fields main/Spacetime.h:50-51 and Ray::I
//                        (main/base.h:175), which the reference declares
//                        and never uses; restated here with the full 4x4
//                        metric
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <type_traits>
#include <vector>

#include "prr.h"

namespace {

// Unqualified math calls: float/double resolve to the std overloads (float
// stays float, as in the reference's host build); the dual numbers of the
// gradient path resolve to their own overloads.
using std::acos;
using std::atan2;
using std::fabs;
using std::floor;
using std::fmax;
using std::fmin;
using std::isnan;
using std::pow;
using std::sqrt;
using std::sin;
using std::cos;

// Forward-mode dual number v + sum_k d[k] e_k for the FP64 host gradient.
// Comparisons use the value, so every branch (accept/reject, termination,
// hit) is decided by the primal run; pow() carries no derivative, so the
// step sizes the controller picks are frozen.
template <int N> struct HD {
    double v = 0.0;
    double d[N] = {};
    HD() = default;
    HD(double x) : v(x) {}
    static HD var(double x, int k) { HD r(x); r.d[k] = 1.0; return r; }
    explicit operator double() const { return v; }
    explicit operator float() const { return (float)v; }
    explicit operator int() const { return (int)v; }
};
template <int N> HD<N> operator+(const HD<N> &a, const HD<N> &b) { HD<N> r(a.v + b.v); for (int k = 0; k < N; k++) r.d[k] = a.d[k] + b.d[k]; return r; }
template <int N> HD<N> operator-(const HD<N> &a, const HD<N> &b) { HD<N> r(a.v - b.v); for (int k = 0; k < N; k++) r.d[k] = a.d[k] - b.d[k]; return r; }
template <int N> HD<N> operator*(const HD<N> &a, const HD<N> &b) { HD<N> r(a.v * b.v); for (int k = 0; k < N; k++) r.d[k] = a.d[k] * b.v + a.v * b.d[k]; return r; }
template <int N> HD<N> operator/(const HD<N> &a, const HD<N> &b) { HD<N> r(a.v / b.v); for (int k = 0; k < N; k++) r.d[k] = (a.d[k] - r.v * b.d[k]) / b.v; return r; }
template <int N> HD<N> operator-(const HD<N> &a) { HD<N> r(-a.v); for (int k = 0; k < N; k++) r.d[k] = -a.d[k]; return r; }
template <int N> HD<N> &operator+=(HD<N> &a, const HD<N> &b) { return a = a + b; }
template <int N> HD<N> &operator-=(HD<N> &a, const HD<N> &b) { return a = a - b; }
template <int N> HD<N> &operator*=(HD<N> &a, const HD<N> &b) { return a = a * b; }
template <int N> HD<N> operator+(const HD<N> &a, double b) { return a + HD<N>(b); }
template <int N> HD<N> operator-(const HD<N> &a, double b) { return a - HD<N>(b); }
template <int N> HD<N> operator*(const HD<N> &a, double b) { return a * HD<N>(b); }
template <int N> HD<N> operator/(const HD<N> &a, double b) { return a / HD<N>(b); }
template <int N> HD<N> operator+(double a, const HD<N> &b) { return HD<N>(a) + b; }
template <int N> HD<N> operator-(double a, const HD<N> &b) { return HD<N>(a) - b; }
template <int N> HD<N> operator*(double a, const HD<N> &b) { return HD<N>(a) * b; }
template <int N> HD<N> operator/(double a, const HD<N> &b) { return HD<N>(a) / b; }
#define PRR_HD_CMP(OP)                                                                              \
    template <int N> bool operator OP(const HD<N> &a, const HD<N> &b) { return a.v OP b.v; }      \
    template <int N> bool operator OP(const HD<N> &a, double b) { return a.v OP b; }               \
    template <int N> bool operator OP(double a, const HD<N> &b) { return a OP b.v; }
PRR_HD_CMP(<) PRR_HD_CMP(>) PRR_HD_CMP(<=) PRR_HD_CMP(>=) PRR_HD_CMP(==) PRR_HD_CMP(!=)
#undef PRR_HD_CMP
template <int N> HD<N> hd_chain(const HD<N> &a, double f, double df) { HD<N> r(f); for (int k = 0; k < N; k++) r.d[k] = df * a.d[k]; return r; }
template <int N> HD<N> sqrt(const HD<N> &a) { double s = std::sqrt(a.v); return hd_chain(a, s, s > 0 ? 0.5 / s : 0.0); }
template <int N> HD<N> sin(const HD<N> &a) { return hd_chain(a, std::sin(a.v), std::cos(a.v)); }
template <int N> HD<N> cos(const HD<N> &a) { return hd_chain(a, std::cos(a.v), -std::sin(a.v)); }
template <int N> HD<N> acos(const HD<N> &a) { double s = 1 - a.v * a.v; return hd_chain(a, std::acos(a.v), s > 0 ? -1 / std::sqrt(s) : 0.0); }
template <int N> HD<N> atan2(const HD<N> &y, const HD<N> &x)
{
    HD<N> r(std::atan2(y.v, x.v));
    double den = x.v * x.v + y.v * y.v;
    for (int k = 0; k < N; k++) r.d[k] = den > 0 ? (x.v * y.d[k] - y.v * x.d[k]) / den : 0.0;
    return r;
}
template <int N> HD<N> fabs(const HD<N> &a) { return a.v < 0 ? -a : a; }
template <int N> HD<N> fmax(const HD<N> &a, const HD<N> &b) { return a.v >= b.v ? a : b; }
template <int N> HD<N> fmin(const HD<N> &a, const HD<N> &b) { return a.v <= b.v ? a : b; }
template <int N> HD<N> floor(const HD<N> &a) { return HD<N>(std::floor(a.v)); }
template <int N> HD<N> pow(const HD<N> &a, const HD<N> &b) { return HD<N>(std::pow(a.v, b.v)); }
template <int N> bool isnan(const HD<N> &a) { return std::isnan(a.v); }
template <int N> HD<N> add_d(HD<N> x, double c) { return x + c; }
template <int N> HD<N> div_d(HD<N> x, double c) { return x / c; }

const double PI_BASE = 3.14159265358979323846;  // main/base.h:20
const double PI_SPHERE = 3.14159265359;          // scene/sphere.h:16 (redefines PI)

struct Tex {
    const uint8_t *p = nullptr;
    int w = 0, h = 0;
};

template <class T> struct V3 { T x, y, z; };
template <class T> struct V4 { T x, y, z, w; };

template <class T> inline T texel(const Tex &t, int i, int j, int c) { return (T)t.p[4 * ((size_t)j * t.w + i) + c] / (T)255; }

template <class T> inline V3<T> texel3(const Tex &t, int i, int j)
{
    return {texel<T>(t, i, j, 0), texel<T>(t, i, j, 1), texel<T>(t, i, j, 2)};
}

// tex2d::operator[](i2): clamp to [0, res-1] (cudamaths/tex2d.cuh:130)
template <class T> inline V3<T> tex_at(const Tex &t, int i, int j)
{
    i = i < 0 ? 0 : (i > t.w - 1 ? t.w - 1 : i);
    j = j < 0 ? 0 : (j > t.h - 1 ? t.h - 1 : j);
    return texel3<T>(t, i, j);
}

// tex2d::operator[](f2): bilinear; the cell index is clamped to [0, res-2]
// AFTER the fraction is taken, so uv outside the interior extrapolates
// (cudamaths/tex2d.cuh:112-119).
// Texel cells read by the last colour lookup of this thread (hashed), part of
// the per-pixel event signature of prr_oracle_grad.
thread_local unsigned long long g_cells = 0;

template <class T> inline V3<T> tex_bilinear(const Tex &t, T u, T v)
{
    T ux = u * (T)t.w, uy = v * (T)t.h;
    int ix = (int)floor(ux), iy = (int)floor(uy);
    g_cells = g_cells * 1315423911ULL + (unsigned long long)(ix * 8191 + iy);
    T px = ux - (T)ix, py = uy - (T)iy;
    ix = ix < 0 ? 0 : (ix > t.w - 2 ? t.w - 2 : ix);
    iy = iy < 0 ? 0 : (iy > t.h - 2 ? t.h - 2 : iy);
    V3<T> a = texel3<T>(t, ix, iy), b = texel3<T>(t, ix + 1, iy);
    V3<T> c = texel3<T>(t, ix, iy + 1), d = texel3<T>(t, ix + 1, iy + 1);
    T one = 1;
    V3<T> r;
    r.x = a.x * (one - px) * (one - py) + b.x * px * (one - py) + c.x * (one - px) * py + d.x * px * py;
    r.y = a.y * (one - px) * (one - py) + b.y * px * (one - py) + c.y * (one - px) * py + d.y * px * py;
    r.z = a.z * (one - px) * (one - py) + b.z * px * (one - py) + c.z * (one - px) * py + d.z * px * py;
    return r;
}

template <class T> inline T fmaxT(T a, T b) { return fmax(a, b); }
template <class T> inline T fminT(T a, T b) { return fmin(a, b); }

// Host copy of a plasma grid (prr_oracle_set_plasma).
struct Plasma {
    bool present = false;
    int nx = 0, ny = 0, nz = 0;
    float lo[3] = {0, 0, 0}, inv[3] = {0, 0, 0};  // inv = (n - 1) / (hi - lo), in float as the library computes it
    std::vector<float> n, theta, vel;             // theta, vel empty when absent
};
Plasma g_plasma;

struct Scene {
    const prr_frame_desc *d;
    Tex tex[PRR_MAX_TEXTURES];
    const Plasma *plasma = nullptr;
};

// ---------------------------------------------------------------- metrics

// Kerr-Schild radius and outer horizon.
template <class T> inline T ks_r(T x, T y, T z, T a)
{
    T R2 = x * x + y * y + z * z;
    T b = R2 - a * a;
    T S = sqrt(b * b + (T)4 * a * a * z * z);
    return sqrt((T)0.5 * (b + S));
}

template <class T> inline T r_plus(T M, T a)
{
    T d = M * M - a * a;
    return M + sqrt(d > 0 ? d : (T)0);
}

// f, l_mu and spatial derivatives (index order x, y, z, t).
template <class T> void ks_fields(T x, T y, T z, T M, T a, T &f, T l[4], T df[3], T dl[4][3])
{
    T R2 = x * x + y * y + z * z, a2 = a * a, b = R2 - a2;
    T S = sqrt(b * b + (T)4 * a2 * z * z);
    T r2 = (T)0.5 * (b + S), r = sqrt(r2);
    T dr[3] = {x * r / S, y * r / S, z * (r2 + a2) / (r * S)};
    T q = r2 + a2, Sig = r2 * r2 + a2 * z * z;
    f = (T)2 * M * r2 * r / Sig;
    for (int k = 0; k < 3; k++) {
        T dSig = (T)4 * r2 * r * dr[k] + (k == 2 ? (T)2 * a2 * z : (T)0);
        df[k] = (T)2 * M * ((T)3 * r2 * dr[k] * Sig - r2 * r * dSig) / (Sig * Sig);
    }
    T nx = r * x + a * y, ny = r * y - a * x;
    l[0] = nx / q; l[1] = ny / q; l[2] = z / r; l[3] = 1;
    for (int k = 0; k < 3; k++) {
        T dq = (T)2 * r * dr[k];
        T dnx = dr[k] * x + (k == 0 ? r : (T)0) + (k == 1 ? a : (T)0);
        T dny = dr[k] * y + (k == 1 ? r : (T)0) - (k == 0 ? a : (T)0);
        dl[0][k] = (dnx * q - nx * dq) / (q * q);
        dl[1][k] = (dny * q - ny * dq) / (q * q);
        dl[2][k] = (k == 2 ? (T)1 / r : (T)0) - z * dr[k] / r2;
        dl[3][k] = 0;
    }
}

// du/dlambda = -Gamma^k_mn u^m u^n from the full Christoffel table.
template <class T> V4<T> geod_table(const V4<T> &p, const V4<T> &u, T M, T a)
{
    if (M == 0) return {0, 0, 0, 0};
    T f, l[4], df[3], dl[4][3];
    ks_fields<T>(p.x, p.y, p.z, M, a, f, l, df, dl);
    const T eta[4] = {1, 1, 1, -1};
    T dg[4][4][4];
    for (int m = 0; m < 4; m++)
        for (int n = 0; n < 4; n++) {
            for (int k = 0; k < 3; k++) dg[m][n][k] = df[k] * l[m] * l[n] + f * (dl[m][k] * l[n] + l[m] * dl[n][k]);
            dg[m][n][3] = 0;
        }
    T lu[4] = {l[0], l[1], l[2], -l[3]};
    T uu[4] = {u.x, u.y, u.z, u.w};
    T acc[4];
    for (int k = 0; k < 4; k++) {
        T s = 0;
        for (int m = 0; m < 4; m++)
            for (int n = 0; n < 4; n++) {
                T G = 0;
                for (int q = 0; q < 4; q++) {
                    T gi = (k == q ? eta[k] : (T)0) - f * lu[k] * lu[q];
                    G += gi * (T)0.5 * (dg[q][n][m] + dg[q][m][n] - dg[m][n][q]);
                }
                s += G * uu[m] * uu[n];
            }
        acc[k] = -s;
    }
    return {acc[0], acc[1], acc[2], acc[3]};
}

// metrics/schwarzschild.cuh:90-119 in the reference's FP32 operation order.
inline V4<float> geod_schw_ref(const V4<float> &p, const V4<float> &u, float rs)
{
    V4<float> du;
    float r = sqrt(p.x * p.x + p.y * p.y + p.z * p.z);
    float x2 = p.x * p.x, y2 = p.y * p.y, z2 = p.z * p.z;
    float Phi = (r * (x2 - 2.0f * y2 - 2.0f * z2) + rs * x2) * u.x * u.x
              + (r * (-2.0f * x2 + y2 - 2.0f * z2) + rs * y2) * u.y * u.y
              + (r * (-2.0f * x2 - 2.0f * y2 + z2) + rs * z2) * u.z * u.z
              + 2.0f * (3.0f * r + rs) * (p.x * p.y * u.x * u.y + p.x * p.z * u.x * u.z + p.y * p.z * u.y * u.z)
              + r * r * (rs - r) * u.w * u.w + 2.0f * r * rs * u.w * (p.x * u.x + p.y * u.y + p.z * u.z);
    Phi *= rs / (2.0f * powf(r, 6));
    du.x = p.x * Phi;
    du.y = p.y * Phi;
    du.z = p.z * Phi;
    du.w = (2.0f * r * (-x2 + y2 + z2) - rs * x2) * u.x * u.x
         + (2.0f * r * (x2 - y2 + z2) - rs * y2) * u.y * u.y
         + (2.0f * r * (x2 + y2 - z2) - rs * z2) * u.z * u.z
         - 2.0f * (4.0f * r + rs) * (p.x * p.y * u.x * u.y + p.x * p.z * u.x * u.z + p.y * p.z * u.y * u.z)
         - r * r * rs * u.w * u.w - 2.0f * r * (r + rs) * u.w * (p.x * u.x + p.y * u.y + p.z * u.z);
    du.w *= rs / (2.0f * powf(r, 5));
    return du;
}

// Kerr-Schild metric, (x,y,z,t) order: g = eta + f l l.
template <class T> void metric_ks(const V4<T> &p, T M, T a, T g[16])
{
    const T eta[4] = {1, 1, 1, -1};
    T f = 0, l[4] = {0, 0, 0, 1};
    if (M != 0) {
        T r = ks_r<T>(p.x, p.y, p.z, a), r2 = r * r, q = r2 + a * a;
        f = (T)2 * M * r2 * r / (r2 * r2 + a * a * p.z * p.z);
        l[0] = (r * p.x + a * p.y) / q; l[1] = (r * p.y - a * p.x) / q; l[2] = p.z / r;
    }
    for (int m = 0; m < 4; m++)
        for (int n = 0; n < 4; n++) g[m * 4 + n] = (m == n ? eta[m] : (T)0) + f * l[m] * l[n];
}

// metrics/schwarzschild.cuh:123-141 in FP32 order.
inline void metric_schw_ref(const V4<float> &p, float rs, float g[16])
{
    float ir = 1.0f / sqrt(p.x * p.x + p.y * p.y + p.z * p.z);
    float ir2 = ir * ir, ir3 = ir2 * ir;
    g[0] = 1.0f + rs * p.x * p.x * ir3; g[1] = rs * p.x * p.y * ir3; g[2] = rs * p.x * p.z * ir3; g[3] = rs * p.x * ir2;
    g[4] = g[1]; g[5] = 1.0f + rs * p.y * p.y * ir3; g[6] = rs * p.y * p.z * ir3; g[7] = rs * p.y * ir2;
    g[8] = g[2]; g[9] = g[6]; g[10] = 1 + rs * p.z * p.z * ir3; g[11] = rs * p.z * ir2;
    g[12] = g[3]; g[13] = g[7]; g[14] = g[11]; g[15] = -1 + rs * ir;
}

template <class T> struct Metric {
    int kind;
    T M, a, rs;
    V4<T> geod(const V4<T> &p, const V4<T> &u, bool refmode) const;
    void metric(const V4<T> &p, T g[16], bool refmode) const;
    T radius(const V4<T> &p) const { return kind == PRR_METRIC_KERR ? ks_r<T>(p.x, p.y, p.z, a) : sqrt(p.x * p.x + p.y * p.y + p.z * p.z); }
    T horizon() const { return kind == PRR_METRIC_SCHWARZSCHILD ? rs : (kind == PRR_METRIC_KERR ? r_plus<T>(M, a) : (T)0); }
};

template <> V4<float> Metric<float>::geod(const V4<float> &p, const V4<float> &u, bool refmode) const
{
    if (kind == PRR_METRIC_FLAT) return {0, 0, 0, 0};
    if (kind == PRR_METRIC_SCHWARZSCHILD && refmode) return geod_schw_ref(p, u, rs);
    return geod_table<float>(p, u, M, kind == PRR_METRIC_KERR ? a : 0.0f);
}
template <> V4<double> Metric<double>::geod(const V4<double> &p, const V4<double> &u, bool) const
{
    if (kind == PRR_METRIC_FLAT) return {0, 0, 0, 0};
    return geod_table<double>(p, u, M, kind == PRR_METRIC_KERR ? a : 0.0);
}
template <> void Metric<float>::metric(const V4<float> &p, float g[16], bool refmode) const
{
    if (kind == PRR_METRIC_SCHWARZSCHILD && refmode) { metric_schw_ref(p, rs, g); return; }
    metric_ks<float>(p, kind == PRR_METRIC_FLAT ? 0.0f : M, kind == PRR_METRIC_KERR ? a : 0.0f, g);
}
template <> void Metric<double>::metric(const V4<double> &p, double g[16], bool) const
{
    metric_ks<double>(p, kind == PRR_METRIC_FLAT ? 0.0 : M, kind == PRR_METRIC_KERR ? a : 0.0, g);
}
// any other T (the dual numbers of the gradient path)
template <class T> V4<T> Metric<T>::geod(const V4<T> &p, const V4<T> &u, bool) const
{
    if (kind == PRR_METRIC_FLAT) return {T(0.0), T(0.0), T(0.0), T(0.0)};
    return geod_table<T>(p, u, M, kind == PRR_METRIC_KERR ? a : T(0.0));
}
template <class T> void Metric<T>::metric(const V4<T> &p, T g[16], bool) const
{
    metric_ks<T>(p, kind == PRR_METRIC_FLAT ? T(0.0) : M, kind == PRR_METRIC_KERR ? a : T(0.0), g);
}

// ---------------------------------------------------------------- scene

template <class T> struct Hit { bool hit; V3<T> c; };

// `x + c` and `x / c` with a double constant, as the reference writes them
// (float + double -> double, stored to float).  Dual numbers keep their
// derivatives.
template <class T> inline T add_d(T x, double c) { return (T)((double)x + c); }
template <class T> inline T div_d(T x, double c) { return (T)((double)x / c); }

// Orbit camera and sphere-phase parameters of the gradient path (T-valued so
// that dual numbers carry d/dparameter through the initial data and the
// hit point).
template <class T> struct Orbit {
    T cam_r, incl;     // camera at (r sin i, 0, r cos i), yaw pi, pitch i - pi/2
    int sphere;        // index of the sphere on the orbit (-1: none)
    T sph_R, sph_phase, sph_z;
};

// Sphere::intersects + Sphere::getColor (scene/sphere.h:34-64) and the
// closest-hit loop of Spacetime::IntersectsScene (main/Spacetime.h:38-46).
// The sphere geometry and texture arithmetic is done in T.
template <class T> Hit<T> intersect_scene(const Scene &sc, const V3<T> &p, V3<T> v, T h, const Orbit<T> *orb = nullptr)
{
    T best_d = (T)100000000000.0, cx = -1, cy = -1, cz = -1;
    bool any = false;
    const prr_frame_desc *d = sc.d;
    // v.normalize(): k = 1/|v|; v *= k
    T k = (T)1 / sqrt(v.x * v.x + v.y * v.y + v.z * v.z);
    v.x *= k; v.y *= k; v.z *= k;
    for (int s = 0; s < d->nspheres; s++) {
        const prr_sphere &S = d->spheres[s];
        V3<T> c = {(T)S.center[0], (T)S.center[1], (T)S.center[2]};
        if (orb && orb->sphere == s)
            c = {orb->sph_R * cos(orb->sph_phase), orb->sph_R * sin(orb->sph_phase), orb->sph_z};
        T rad = (T)S.radius;
        T v2 = v.x * v.x + v.y * v.y + v.z * v.z;
        V3<T> pc = {p.x - c.x, p.y - c.y, p.z - c.z};
        T dvp = v.x * pc.x + v.y * pc.y + v.z * pc.z;
        T disc = dvp * dvp - v2 * ((pc.x * pc.x + pc.y * pc.y + pc.z * pc.z) - rad * rad);
        if (disc < 0) continue;
        T dd = ((T)(-2.0f) * dvp - sqrt(disc)) / v2;
        if (dd * dd > v2 * h) continue;
        if (dd < 0) continue;
        // getColor((p + v*d) - c)
        V3<T> in = {(p.x + v.x * dd) - c.x, (p.y + v.y * dd) - c.y, (p.z + v.z * dd) - c.z};
        T theta = acos(in.z / rad);
        T phi = add_d(atan2(in.y, in.x), PI_SPHERE);
        T uu = div_d(phi, 2.0 * PI_SPHERE), vv = div_d(theta, PI_SPHERE);
        const T uvmax = (T)0.999999999f;
        uu = fminT<T>(fmaxT<T>(uu, (T)0), uvmax);
        vv = fminT<T>(fmaxT<T>(vv, (T)0), uvmax);
        V3<T> col = {(T)0.5, (T)0.5, (T)0.5};
        if (S.texture_id >= 0 && S.texture_id < PRR_MAX_TEXTURES && sc.tex[S.texture_id].p) col = tex_bilinear<T>(sc.tex[S.texture_id], uu, vv);
        T shade = fmaxT<T>((T)0, fminT<T>((T)0.5 + (T)0.5 * in.z / rad, (T)1));
        col.x *= shade; col.y *= shade; col.z *= shade;
        if (col.x >= 0 && dd <= best_d) {
            best_d = dd; cx = col.x; cy = col.y; cz = col.z; any = true;
        }
    }
    Hit<T> r;
    r.hit = any && cx >= 0;
    r.c = {cx, cy, cz};
    return r;
}

// OutSphere::getColorDefault2 (main/base.h:119-162): RMS of the 2x2 texel
// block at floor(uv); a single texel on the last row/column.
template <class T> V3<T> background_rms(const Tex &t, const V4<T> &u)
{
    T k = (T)1 / sqrt(u.x * u.x + u.y * u.y + u.z * u.z);
    V3<T> n = {u.x * k, u.y * k, u.z * k};
    T theta = acos(n.z);
    T phi = atan2(n.y, n.x);
    phi = (phi >= 0 ? phi : (T)((double)phi + 2.0 * PI_BASE));
    if ((double)phi > 2.0 * PI_BASE || phi < 0) return {(T)0.5, (T)0.5, (T)0};
    if (theta < 0 || (double)theta > PI_BASE) return {(T)0, (T)0.5, (T)0.8};
    T ux = (T)((double)phi / (2.0 * PI_BASE) * t.w), uy = (T)((double)theta / PI_BASE * t.h);
    int px = (int)floor(ux), py = (int)floor(uy);
    if (px == t.w) px -= 1;
    if (py == t.h) py -= 1;
    if (px < 0 || px >= t.w || py < 0 || py >= t.h) return {(T)0, (T)0.5, (T)0};
    if (px == t.w - 1 || py == t.h - 1) return tex_at<T>(t, px, py);
    V3<T> a = tex_at<T>(t, px, py), b = tex_at<T>(t, px, py + 1), c = tex_at<T>(t, px + 1, py), d = tex_at<T>(t, px + 1, py + 1);
    const T q = (T)0.25;
    return {sqrt(q * (a.x * a.x + b.x * b.x + c.x * c.x + d.x * d.x)),
            sqrt(q * (a.y * a.y + b.y * b.y + c.y * c.y + d.y * d.y)),
            sqrt(q * (a.z * a.z + b.z * b.z + c.z * c.z + d.z * d.z))};
}

// Continuous lookup (PRR_BG_BILINEAR): bilinear over texel centres, wrap in
// longitude, clamp in latitude.
template <class T> V3<T> background_bilinear(const Tex &t, const V4<T> &u)
{
    T k = (T)1 / sqrt(u.x * u.x + u.y * u.y + u.z * u.z);
    T nz = u.z * k;
    nz = nz > 1 ? 1 : (nz < -1 ? -1 : nz);
    T theta = acos(nz);
    T phi = atan2(u.y, u.x);
    if (phi < 0) phi += (T)(2.0 * PI_BASE);
    T fx = phi / (T)(2.0 * PI_BASE) * t.w - (T)0.5, fy = theta / (T)PI_BASE * t.h - (T)0.5;
    T flx = floor(fx), fly = floor(fy);
    T wx = fx - flx, wy = fy - fly;
    int x0 = (int)flx, y0 = (int)fly;
    g_cells = g_cells * 1315423911ULL + (unsigned long long)(x0 * 8191 + y0);
    int x1 = x0 + 1, y1 = y0 + 1;
    x0 = ((x0 % t.w) + t.w) % t.w; x1 = ((x1 % t.w) + t.w) % t.w;
    y0 = y0 < 0 ? 0 : (y0 > t.h - 1 ? t.h - 1 : y0);
    y1 = y1 < 0 ? 0 : (y1 > t.h - 1 ? t.h - 1 : y1);
    V3<T> a = texel3<T>(t, x0, y0), b = texel3<T>(t, x1, y0), c = texel3<T>(t, x0, y1), d = texel3<T>(t, x1, y1);
    T w00 = (1 - wx) * (1 - wy), w10 = wx * (1 - wy), w01 = (1 - wx) * wy, w11 = wx * wy;
    return {a.x * w00 + b.x * w10 + c.x * w01 + d.x * w11, a.y * w00 + b.y * w10 + c.y * w01 + d.y * w11,
            a.z * w00 + b.z * w10 + c.z * w01 + d.z * w11};
}

// ---------------------------------------------------------------- ray

template <class T> struct RayState {
    T uvx, uvy;
    int result;
    V4<T> r, u;
    long long accepted = 0, attempts = 0;
    V3<float> rgb;
    V3<T> rgbT;  // the same colour in T (gradient path)
    unsigned long long cells = 0;  // texel cells read for the colour (finite-difference tests)
    T I = T(0.0), trans = T(1.0), nu_cam = T(0.0);  // plasma emission (intensity, transmittance, camera frequency)
};

// The stochastic placements' hash: the PCG output permutation of an LCG
// step ("pcg_hash", Jarzynski & Olano, JCGT 2020), two 24-bit uniforms per
// (seed, pixel, sample).
inline uint32_t pcg_hash(uint32_t v)
{
    uint32_t state = v * 747796405u + 2891336453u;
    uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
    return (word >> 22u) ^ word;
}

inline void sample_offsets(uint32_t seed, long long p, int s, float &r0, float &r1)
{
    uint32_t h = pcg_hash(seed ^ pcg_hash((uint32_t)p ^ pcg_hash((uint32_t)(p >> 32) + 0x9e3779b9u * (uint32_t)(s + 1))));
    uint32_t g = pcg_hash(h);
    r0 = (float)(h >> 8) * (1.0f / 16777216.0f);
    r1 = (float)(g >> 8) * (1.0f / 16777216.0f);
}

// createRays_none / createRays_regular (kernels/ssaa.cuh:92-99, 36-48); RANDOM
// (uniform in the pixel) and JITTERED (uniform in each cell of an n x n grid).
inline void ray_uv(const prr_frame_desc *d, long long rid, float &uvx, float &uvy)
{
    int S = d->samples;
    long long pix = rid / S;
    int s = (int)(rid % S);
    int x = (int)(pix % d->width), y = (int)(pix / d->width);
    if (d->ssaa == PRR_SSAA_NONE) {
        uvx = (float)x / d->width + (1.0f / d->width) * 0.5f;
        uvy = (float)y / d->height + (1.0f / d->height) * 0.5f;
    } else if (d->ssaa == PRR_SSAA_REGULAR) {
        int n = (int)roundf(sqrtf((float)S));
        float dux = (1.0f / d->width) / (n + 1.0f), duy = (1.0f / d->height) / (n + 1.0f);
        int i = s % n, j = s / n;
        uvx = (float)x / d->width + (float)(i + 1) * dux;
        uvy = (float)y / d->height + (float)(j + 1) * duy;
    } else {
        float r0, r1;
        sample_offsets(d->ssaa_seed, pix, s, r0, r1);
        if (d->ssaa == PRR_SSAA_JITTERED) {
            const int n = (int)roundf(sqrtf((float)S));
            r0 = ((float)(s % n) + r0) / (float)n;
            r1 = ((float)(s / n) + r1) / (float)n;
        }
        uvx = ((float)x + r0) / (float)d->width;
        uvy = ((float)y + r1) / (float)d->height;
    }
}

// Camera::computeVectors (main/Camera.cpp:19-28) in FP32.
inline void camera_basis(float a, float b, float fwd[3], float right[3], float up[3])
{
    auto nrm = [](float v[3]) {
        float k = 1.0f / sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        v[0] = k * v[0]; v[1] = k * v[1]; v[2] = k * v[2];
    };
    fwd[0] = cosf(b) * cosf(a); fwd[1] = cosf(b) * sinf(a); fwd[2] = -sinf(b);
    nrm(fwd);
    up[0] = cosf(a) * sinf(b); up[1] = sinf(a) * sinf(b); up[2] = cosf(b);
    nrm(up);
    right[0] = fwd[1] * up[2] - fwd[2] * up[1];
    right[1] = fwd[2] * up[0] - fwd[0] * up[2];
    right[2] = fwd[0] * up[1] - fwd[1] * up[0];
    nrm(right);
}

// Camera::rayDir_Spherical (main/Camera.h:39-42) in FP32, rayDir_PinHole
// (30-33) and the equirectangular panorama (34-37), the last two on the
// basis oriented like the spherical model (see prr_camera).
inline V3<float> ray_dir(const prr_frame_desc *d, float uvx, float uvy)
{
    V3<float> v;
    if (d->camera == PRR_CAMERA_SPHERICAL) {
        float nu = (0.5f - uvy) * d->vfov;
        float mu = (0.5f - uvx) * (float)d->width / (float)d->height * d->vfov;
        float cb = cosf(d->cam_beta + nu);
        v = {cb * cosf(d->cam_alpha + mu), cb * sinf(d->cam_alpha + mu), sinf(d->cam_beta + nu)};
    } else {
        float f[3], r[3], u[3];
        camera_basis(d->cam_alpha, -d->cam_beta, f, r, u);  // pitch sign: see the renderer's basis
        float a, b, c;
        if (d->camera == PRR_CAMERA_PINHOLE) {
            const float t = tanf(d->vfov / 2.0f);
            a = 1.0f;
            b = (2.0f * uvx - 1.0f) * t * (float)d->width / (float)d->height;
            c = (1.0f - 2.0f * uvy) * t;
        } else {
            const float mu = (0.5f - uvy) * d->vfov;
            const float nu = (uvx - 0.5f) * (float)d->width / (float)d->height * d->vfov;
            const float cm = cosf(mu);
            a = cm * cosf(nu); b = cm * sinf(nu); c = sinf(mu);
        }
        v = {a * f[0] + b * r[0] + c * u[0], a * f[1] + b * r[1] + c * u[1], a * f[2] + b * r[2] + c * u[2]};
    }
    float k = 1.0f / sqrtf(v.x * v.x + v.y * v.y + v.z * v.z);
    return {v.x * k, v.y * k, v.z * k};
}

// (float) of the reference's double-literal tableau (solver.cuh:125-131).
struct Tableau {
    double A21 = 1.0 / 4.0, A31 = 3.0 / 32.0, A32 = 9.0 / 32.0, A41 = 1932.0 / 2197.0, A42 = -7200.0 / 2197.0,
           A43 = 7296.0 / 2197.0, A51 = 439.0 / 216.0, A52 = -8.0, A53 = 3680.0 / 513.0, A54 = -845.0 / 4104.0,
           A61 = -8.0 / 27.0, A62 = 2.0, A63 = -3544.0 / 2565.0, A64 = 1859.0 / 4104.0, A65 = -11.0 / 40.0,
           K41 = 25.0 / 216.0, K42 = 0.0, K43 = 1408.0 / 2565.0, K44 = 2197.0 / 4104.0, K45 = -1.0 / 5.0, K46 = 0.0,
           K51 = 16.0 / 135.0, K52 = 0.0, K53 = 6656.0 / 12825.0, K54 = 28561.0 / 56430.0, K55 = -9.0 / 50.0,
           K56 = 2.0 / 55.0;
};

template <class T> inline V4<T> add(const V4<T> &a, const V4<T> &b) { return {a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }
template <class T> inline V4<T> scl(T s, const V4<T> &a) { return {a.x * s, a.y * s, a.z * s, a.w * s}; }
template <class T> inline bool isnan4(const V4<T> &a) { return isnan(a.x) || isnan(a.y) || isnan(a.z) || isnan(a.w); }
template <class T> inline T max4abs(const V4<T> &a, const V4<T> &b)
{
    return fmaxT<T>(fmaxT<T>(fmaxT<T>(fabs(a.x - b.x), fabs(a.y - b.y)), fabs(a.z - b.z)), fabs(a.w - b.w));
}

// ---------------------------------------------------------------- emission

template <class T> inline T gdot(const T g[16], const T A[4], const T B[4])
{
    T s = 0;
    for (int m = 0; m < 4; m++)
        for (int n = 0; n < 4; n++) s += g[4 * m + n] * A[m] * B[n];
    return s;
}

// Trilinear interpolation of the grid's nodes around (x, y, z); false
// outside the box.
template <class T> bool plasma_at(const Plasma &P, T x, T y, T z, T &n, T &theta, T v[3])
{
    const T p[3] = {x, y, z};
    const int dim[3] = {P.nx, P.ny, P.nz};
    int i[3];
    T t[3];
    for (int k = 0; k < 3; k++) {
        T s = (p[k] - (T)P.lo[k]) * (T)P.inv[k];
        if (!(s >= (T)0 && s <= (T)(dim[k] - 1))) return false;
        i[k] = std::min((int)s, dim[k] - 2);
        t[k] = s - (T)i[k];
    }
    n = 0; theta = P.theta.empty() ? (T)1 : (T)0;
    v[0] = v[1] = v[2] = 0;
    for (int c = 0; c < 8; c++) {
        const int bx = c & 1, by = (c >> 1) & 1, bz = c >> 2;
        const T w = (bx ? t[0] : (T)1 - t[0]) * (by ? t[1] : (T)1 - t[1]) * (bz ? t[2] : (T)1 - t[2]);
        const size_t id = (size_t)(i[0] + bx) + (size_t)P.nx * ((size_t)(i[1] + by) + (size_t)P.ny * (size_t)(i[2] + bz));
        n += w * (T)P.n[id];
        if (!P.theta.empty()) theta += w * (T)P.theta[id];
        if (!P.vel.empty())
            for (int k = 0; k < 3; k++) v[k] += w * (T)P.vel[3 * id + k];
    }
    return true;
}

template <class T> class Tracer {
public:
    Tracer(const Scene &sc) : sc_(sc), d_(sc.d)
    {
        mt_.kind = d_->metric;
        mt_.M = (T)d_->mass;
        mt_.a = (T)d_->spin;
        mt_.rs = (T)(2.0f * d_->mass);
        ref_ = d_->mode == PRR_MODE_REFERENCE;
        rstop_ = ref_ && d_->metric == PRR_METRIC_SCHWARZSCHILD ? (T)(2.0f * d_->mass + d_->horizon_eps)
                                                                : mt_.horizon() + (T)d_->horizon_eps;
    }

    // Gradient path: mass and spin as given (dual numbers), camera and one
    // sphere from `orb`.
    Tracer(const Scene &sc, T M, T a, const Orbit<T> *orb) : Tracer(sc)
    {
        mt_.M = M;
        mt_.a = a;
        mt_.rs = (T)2 * M;
        rstop_ = T((double)(mt_.horizon() + (T)d_->horizon_eps));  // the stop radius is an event threshold
        orb_ = orb;
    }

    RayState<T> run(long long rid) const
    {
        RayState<T> R;
        float ux, uy;
        ray_uv(d_, rid, ux, uy);
        R.uvx = ux; R.uvy = uy;
        R.result = PRR_RESULT_SUCCESS;
        init(R);
        if (d_->solver == PRR_SOLVER_EULER) euler(R);
        else rkf(R);
        g_cells = 0;
        colour(R);
        R.cells = g_cells;
        return R;
    }

private:
    const Scene &sc_;
    const prr_frame_desc *d_;
    Metric<T> mt_;
    bool ref_;
    T rstop_;
    const Orbit<T> *orb_ = nullptr;

    // initRays (kernels/solver.cuh:26-56)
    void init(RayState<T> &R) const
    {
        V4<T> u;
        if (orb_) {
            // Camera::rayDir_Spherical with a = pi, b = i - pi/2, evaluated in T
            const double PI = 3.14159265358979323846;
            T beta = orb_->incl - (T)(0.5 * PI);
            double nu = (0.5 - (double)R.uvy) * (double)d_->vfov;
            double mu = (0.5 - (double)R.uvx) * (double)d_->width / (double)d_->height * (double)d_->vfov;
            T cb = cos(beta + (T)nu);
            T dx = cb * (T)std::cos(PI + mu), dy = cb * (T)std::sin(PI + mu), dz = sin(beta + (T)nu);
            T k = (T)1 / sqrt(dx * dx + dy * dy + dz * dz);
            R.r = {orb_->cam_r * sin(orb_->incl), (T)0, orb_->cam_r * cos(orb_->incl), (T)0};
            u = {dx * k, dy * k, dz * k, (T)1};
        } else {
            V3<float> dir = ray_dir(d_, (float)R.uvx, (float)R.uvy);
            R.r = {(T)d_->cam_pos[0], (T)d_->cam_pos[1], (T)d_->cam_pos[2], (T)0};
            u = {(T)dir.x, (T)dir.y, (T)dir.z, (T)1};
        }
        T g[16];
        mt_.metric(R.r, g, ref_);
        T a = g[15];
        T b = (T)2 * (g[12] * u.x + g[13] * u.y + g[14] * u.z);
        T c = g[0] * u.x * u.x + g[5] * u.y * u.y + g[10] * u.z * u.z + (T)2 * (g[1] * u.x * u.y + g[2] * u.x * u.z + g[6] * u.y * u.z);
        T rt = sqrt(b * b - (T)4 * a * c);
        T u0 = fmaxT<T>((-b + rt) / ((T)2 * a), (-b - rt) / ((T)2 * a));
        if (u0 < 0) u0 = 1;
        if (ref_) u = scl(u0, u);  // whole 4-vector scaled (solver.cuh:54)
        else u.w = u0;            // null: u^t solves g(u,u) = 0
        R.u = u;
        if constexpr (std::is_floating_point<T>::value) emis_init(R);
    }

    // Frequency of the ray measured by a static observer at the camera:
    // nu_cam = -k_t / sqrt(-g_tt).
    void emis_init(RayState<T> &R) const
    {
        if (d_->emission == PRR_EMISSION_NONE) return;
        T g[16];
        mt_.metric(R.r, g, false);
        const T k[4] = {R.u.x, R.u.y, R.u.z, R.u.w};
        const T kt = g[12] * k[0] + g[13] * k[1] + g[14] * k[2] + g[15] * k[3];
        R.nu_cam = -kt / sqrt(-g[15]);
        R.I = 0;
        R.trans = 1;
    }

    // Emission of one accepted step of affine length h ending at (R.r, R.u).
    void emis_step(RayState<T> &R, T h) const
    {
        if (d_->emission == PRR_EMISSION_NONE) return;
        const prr_emission_desc &e = d_->emis;
        const T M = d_->metric == PRR_METRIC_FLAT ? (T)0 : mt_.M, a = d_->metric == PRR_METRIC_KERR ? mt_.a : (T)0;
        const T r = ks_r<T>(R.r.x, R.r.y, R.r.z, a);
        if (!(r >= (T)e.r_in && r <= (T)e.r_out)) return;
        T n, theta = 1, v[3];
        bool flow = false;
        if (d_->emission == PRR_EMISSION_DISK) {
            const T c = R.r.z / r;
            n = pow(r / (T)e.r_in, -(T)e.index) * std::exp(-c * c / ((T)2 * (T)e.height * (T)e.height));
        } else {
            if (!sc_.plasma || !plasma_at<T>(*sc_.plasma, R.r.x, R.r.y, R.r.z, n, theta, v)) return;
            flow = !sc_.plasma->vel.empty();
        }
        if (!(n > (T)0)) return;
        if (!flow) {  // equatorial Keplerian angular velocity at r, about the z axis
            const T s = (T)e.sense, om = s * sqrt(M) / (r * sqrt(r) + s * a * sqrt(M));
            v[0] = -om * R.r.y; v[1] = om * R.r.x; v[2] = 0;
        }
        T g[16];
        mt_.metric(R.r, g, false);
        const T xi[4] = {v[0], v[1], v[2], (T)1}, k[4] = {R.u.x, R.u.y, R.u.z, R.u.w};
        const T N = gdot<T>(g, xi, xi);
        if (!(N < (T)0)) return;
        const T nu_e = -gdot<T>(g, k, xi) / sqrt(-N);
        if (!(nu_e > (T)0)) return;
        const T gr = R.nu_cam / nu_e, dl = R.nu_cam * h;
        T j = n;
        if (d_->emission == PRR_EMISSION_GRID && e.temp_power != 0.0f) j *= pow(theta, (T)e.temp_power);
        const T w = e.spectral_index == 0.0f ? gr * gr : pow(gr, (T)2 + (T)e.spectral_index);
        R.I += R.trans * w * j * dl;
        if (e.absorb > 0.0f) R.trans *= std::exp(-(T)e.absorb * n * dl / gr);
    }

    bool user_update(RayState<T> &R, T h) const
    {
        Hit<T> c = intersect_scene<T>(sc_, {R.r.x, R.r.y, R.r.z}, {R.u.x, R.u.y, R.u.z}, h, orb_);
        if (c.hit) { R.result = PRR_RESULT_INTERSECTION; return false; }
        return true;
    }

    bool user_endloop(RayState<T> &R, T th) const
    {
        T r = mt_.radius(R.r);
        bool horizon = d_->metric != PRR_METRIC_FLAT && r <= rstop_;
        if (r >= (T)d_->rout || horizon) { R.result = PRR_RESULT_SUCCESS; return false; }
        Hit<T> c = intersect_scene<T>(sc_, {R.r.x, R.r.y, R.r.z}, {R.u.x, R.u.y, R.u.z}, th, orb_);
        if (c.hit) {
            R.u = {c.c.x, c.c.y, c.c.z, (T)0};
            R.result = PRR_RESULT_INTERSECTION;
            return false;
        }
        return true;
    }

    // trace_Euler (kernels/solver.cuh:68-116)
    void euler(RayState<T> &R) const
    {
        bool intersect = false;
        T h = (T)d_->h;
        long long steps = 0;
        const T lmax = (T)5000;
        for (T l = 0; l < lmax; l += h) {
            if (!ref_ && steps >= d_->max_steps) break;
            V4<T> du = mt_.geod(R.r, R.u, ref_);
            R.attempts++;
            if (isnan4(du)) { R.result = PRR_RESULT_MATH_ERROR; return; }
            R.r = add(R.r, scl(h, R.u));
            R.u = add(R.u, scl(h, du));
            steps++;
            R.accepted = steps;
            if (!user_update(R, h)) {
                if (R.result == PRR_RESULT_INTERSECTION && !intersect) { intersect = true; h = (T)d_->hmin; continue; }
            }
            if (!user_endloop(R, (T)d_->h)) return;
        }
        R.result = PRR_RESULT_INFINITE_GEO;
    }

    V4<T> G(const V4<T> &x, const V4<T> &u) const { return mt_.geod(x, u, ref_); }

    // trace_RKF (kernels/solver.cuh:142-219)
    void rkf(RayState<T> &R) const
    {
        const Tableau tb;
        // REFERENCE mode: the reference stores the tableau as float
        // (solver.cuh:125-131); PHYSICAL mode rounds the exact fractions to T.
        auto c = [&](double v) { return ref_ ? (T)(float)v : (T)v; };
        const T A21 = c(tb.A21), A31 = c(tb.A31), A32 = c(tb.A32), A41 = c(tb.A41), A42 = c(tb.A42), A43 = c(tb.A43),
                A51 = c(tb.A51), A52 = c(tb.A52), A53 = c(tb.A53), A54 = c(tb.A54), A61 = c(tb.A61), A62 = c(tb.A62),
                A63 = c(tb.A63), A64 = c(tb.A64), A65 = c(tb.A65);
        const T K41 = c(tb.K41), K42 = c(tb.K42), K43 = c(tb.K43), K44 = c(tb.K44), K45 = c(tb.K45), K46 = c(tb.K46),
                K51 = c(tb.K51), K52 = c(tb.K52), K53 = c(tb.K53), K54 = c(tb.K54), K55 = c(tb.K55), K56 = c(tb.K56);
        T h = (T)d_->h, hmin = (T)d_->hmin, hmax = (T)d_->hmax, _h = h;
        T eps = (T)d_->eps, rtol = (T)d_->rtol, atol = (T)d_->atol;
        T trace_h = (T)d_->h;
        V4<T> x = R.r, u = R.u, _x = x, _u = u, __x, __u;
        bool intersect = false;
        long long i = 0, accepted = 0;
        const long long max_att = ref_ ? 1000000 : 8LL * d_->max_steps;
        for (T l = 0; l < (T)1000;) {
            i += 1;
            R.attempts = i;
            V4<T> kx1 = scl(h, u);
            V4<T> ku1 = scl(h, G(x, u));
            V4<T> z2x = add(x, scl(A21, kx1));
            V4<T> z2u = ref_ ? add(u, scl(A21, kx1)) : add(u, scl(A21, ku1));
            V4<T> kx2 = scl(h, z2u), ku2 = scl(h, G(z2x, z2u));
            V4<T> z3x = add(add(x, scl(A31, kx1)), scl(A32, kx2));
            V4<T> z3u = add(add(u, scl(A31, ref_ ? kx1 : ku1)), scl(A32, ku2));
            V4<T> kx3 = scl(h, z3u), ku3 = scl(h, G(z3x, z3u));
            V4<T> z4x = add(add(add(x, scl(A41, kx1)), scl(A42, kx2)), scl(A43, kx3));
            V4<T> z4u = add(add(add(u, scl(A41, ref_ ? kx1 : ku1)), scl(A42, ku2)), scl(A43, ku3));
            V4<T> kx4 = scl(h, z4u), ku4 = scl(h, G(z4x, z4u));
            V4<T> z5x = add(add(add(add(x, scl(A51, kx1)), scl(A52, kx2)), scl(A53, kx3)), scl(A54, kx4));
            V4<T> z5u = add(add(add(add(u, scl(A51, ref_ ? kx1 : ku1)), scl(A52, ku2)), scl(A53, ku3)), scl(A54, ku4));
            V4<T> kx5 = scl(h, z5u), ku5 = scl(h, G(z5x, z5u));
            V4<T> z6x = add(add(add(add(add(x, scl(A61, kx1)), scl(A62, kx2)), scl(A63, kx3)), scl(A64, kx4)), scl(A65, kx5));
            V4<T> z6u = add(add(add(add(add(u, scl(A61, ref_ ? kx1 : ku1)), scl(A62, ku2)), scl(A63, ku3)), scl(A64, ku4)), scl(A65, ku5));
            V4<T> kx6 = scl(h, z6u), ku6 = scl(h, G(z6x, z6u));

            _x = add(add(add(add(add(add(x, scl(K41, kx1)), scl(K42, kx2)), scl(K43, kx3)), scl(K44, kx4)), scl(K45, kx5)), scl(K46, kx6));
            _u = add(add(add(add(add(add(u, scl(K41, ku1)), scl(K42, ku2)), scl(K43, ku3)), scl(K44, ku4)), scl(K45, ku5)), scl(K46, ku6));
            __x = add(add(add(add(add(add(x, scl(K51, kx1)), scl(K52, kx2)), scl(K53, kx3)), scl(K54, kx4)), scl(K55, kx5)), scl(K56, kx6));
            __u = add(add(add(add(add(add(u, scl(K51, ku1)), scl(K52, ku2)), scl(K53, ku3)), scl(K54, ku4)), scl(K55, ku5)), scl(K56, ku6));

            T maxerr;
            if (ref_) {
                maxerr = fmaxT<T>(max4abs(__x, _x), max4abs(__u, _u));
                _h = (T)0.9f * h * (T)pow((T)(eps / maxerr), (T)0.2f);
            } else {
                // mixed error norm: max_i |y5_i - y4_i| / (atol + rtol*max(|y_i|, |y4_i|))
                const T *a0 = &x.x, *a1 = &_x.x, *a2 = &__x.x, *b0 = &u.x, *b1 = &_u.x, *b2 = &__u.x;
                maxerr = 0;
                for (int c = 0; c < 4; c++) {
                    T sx = atol + rtol * fmaxT<T>(fabs(a0[c]), fabs(a1[c]));
                    T su = atol + rtol * fmaxT<T>(fabs(b0[c]), fabs(b1[c]));
                    maxerr = fmaxT<T>(maxerr, fabs(a2[c] - a1[c]) / sx);
                    maxerr = fmaxT<T>(maxerr, fabs(b2[c] - b1[c]) / su);
                }
                _h = (T)0.9 * h * pow((T)1 / maxerr, (T)0.2);
            }
            _h = fminT<T>(fmaxT<T>(_h, hmin), hmax);

            if (intersect && i > 10000) intersect = false;
            if (i > max_att) break;
            T tol = ref_ ? eps : (T)1;
            if (maxerr > tol && h != hmin && !intersect) { h = _h; continue; }
            if (isnan4(x) || isnan4(u)) { R.result = PRR_RESULT_MATH_ERROR; R.accepted = accepted; return; }

            R.r = _x; R.u = _u;
            accepted++;
            R.accepted = accepted;
            const T h_step = h;
            if (user_update(R, h)) {
                if (!intersect) h = _h;
                x = _x; u = _u; R.r = x; R.u = u; trace_h = h;
            } else if (R.result == PRR_RESULT_INTERSECTION && !intersect) {
                intersect = true; h = hmin; continue;
            }
            if constexpr (std::is_floating_point<T>::value) emis_step(R, h_step);
            if (!user_endloop(R, trace_h)) return;
            x = R.r; u = R.u;
            l += h;
            if (!ref_ && accepted >= d_->max_steps) break;
        }
        R.result = PRR_RESULT_INFINITE_GEO;
    }

    // rayToRGB (metrics/schwarzschild.cuh:151-183, metrics/flat.cuh:104-131)
    void colour(RayState<T> &R) const
    {
        T r = mt_.radius(R.r);
        V3<T> c = {R.u.x, R.u.y, R.u.z};
        const T black[3] = {0, 0, 0};
        bool set_black = false;
        if (R.result == PRR_RESULT_SUCCESS) {
            bool captured = d_->metric != PRR_METRIC_FLAT &&
                            (ref_ ? r <= (d_->metric == PRR_METRIC_SCHWARZSCHILD ? (T)(2.0f * d_->mass) * (T)1.01f : mt_.horizon() * (T)1.01f)
                                  : r < (T)d_->rout);
            if (captured) set_black = true;
            else if (r >= (T)d_->rout) {
                int bid = d_->background_id;
                if (bid >= 0 && bid < PRR_MAX_TEXTURES && sc_.tex[bid].p)
                    c = d_->bg_filter == PRR_BG_BILINEAR ? background_bilinear<T>(sc_.tex[bid], R.u) : background_rms<T>(sc_.tex[bid], R.u);
                else set_black = true;
            }
        } else if (R.result == PRR_RESULT_INTERSECTION) {
        } else set_black = true;
        if (set_black) c = {black[0], black[1], black[2]};
        R.rgb = {(float)c.x, (float)c.y, (float)c.z};
        R.rgbT = c;
        if (d_->emission != PRR_EMISSION_NONE) {  // trans * colour + map(gain * I)
            const float x = (float)((T)d_->emis.gain * R.I), tr = (float)R.trans;
            auto cl = [](float v) { return std::fmin(std::fmax(v, 0.0f), 1.0f); };
            float m[3];
            if (d_->emis.colormap == PRR_CMAP_GREY) m[0] = m[1] = m[2] = cl(x);
            else { m[0] = cl(2.0f * x); m[1] = cl(2.0f * x - 0.5f); m[2] = cl(2.0f * x - 1.0f); }
            R.rgb = {tr * R.rgb.x + m[0], tr * R.rgb.y + m[1], tr * R.rgb.z + m[2]};
        }
    }
};

inline float luma_ref(float r, float g, float b)
{
    // kernels/ssaa.cuh:141-143: the weights are double literals, so the sum
    // is formed in double and returned as float.
    return (float)(r * 0.299 * (1.0f / 255.0f) + g * 0.587 * (1.0f / 255.0f) + b * 0.114 * (1.0f / 255.0f));
}

struct Img {
    const float *p;
    int w, h;
    void at(int i, int j, float c[3]) const
    {
        i = i < 0 ? 0 : (i > w - 1 ? w - 1 : i);
        j = j < 0 ? 0 : (j > h - 1 ? h - 1 : j);
        const float *q = p + 3 * ((size_t)j * w + i);
        c[0] = q[0]; c[1] = q[1]; c[2] = q[2];
    }
    void bilinear(float ux, float uy, float c[3]) const
    {
        ux = ux * (float)w; uy = uy * (float)h;
        int ix = (int)floorf(ux), iy = (int)floorf(uy);
        float px = ux - (float)ix, py = uy - (float)iy;
        ix = ix < 0 ? 0 : (ix > w - 2 ? w - 2 : ix);
        iy = iy < 0 ? 0 : (iy > h - 2 ? h - 2 : iy);
        const float *a = p + 3 * ((size_t)iy * w + ix), *b = a + 3, *cc = a + 3 * (size_t)w, *d = cc + 3;
        for (int k = 0; k < 3; k++) c[k] = a[k] * (1 - px) * (1 - py) + b[k] * px * (1 - py) + cc[k] * (1 - px) * py + d[k] * px * py;
    }
};

// kernels/ssaa.cuh:150-181.  Pixels the reference kernel never writes
// (border rows/columns: it clamps the index to [1, res-2] and writes there)
// are returned unfiltered.
void fxaa_ref(const float *in, float *out, int w, int h)
{
    memcpy(out, in, sizeof(float) * 3 * (size_t)w * h);
    if (w < 3 || h < 3) return;
    Img im{in, w, h};
    const float SPAN_MAX = 8.0f, REDUCE_MUL = 1.0f / 8.0f, REDUCE_MIN = 1.0f / 128.0f;
    for (int y = 1; y < h - 1; y++)
        for (int x = 1; x < w - 1; x++) {
            float cNW[3], cNE[3], cSW[3], cSE[3], cM[3];
            im.at(x - 1, y - 1, cNW); im.at(x + 1, y - 1, cNE); im.at(x - 1, y + 1, cSW); im.at(x + 1, y + 1, cSE); im.at(x, y, cM);
            float lNW = luma_ref(cNW[0], cNW[1], cNW[2]), lNE = luma_ref(cNE[0], cNE[1], cNE[2]);
            float lSW = luma_ref(cSW[0], cSW[1], cSW[2]), lSE = luma_ref(cSE[0], cSE[1], cSE[2]);
            float lM = luma_ref(cM[0], cM[1], cM[2]);
            float lMin = fminf(lM, fminf(fminf(lNW, lNE), fminf(lSW, lSE)));
            float lMax = fmaxf(lM, fmaxf(fmaxf(lNW, lNE), fmaxf(lSW, lSE)));
            float dx = -((lNW + lNE) - (lSW + lSE)), dy = ((lNW + lSW) - (lNE + lSE));
            float dirReduce = fmaxf((lNW + lNE + lSW + lSE) * (0.25f * REDUCE_MUL), REDUCE_MIN);
            float rcp = 1.0f / (fminf(fabsf(dx), fabsf(dy)) + dirReduce);
            dx = fminf(fmaxf(dx * rcp, -SPAN_MAX), SPAN_MAX);
            dy = fminf(fmaxf(dy * rcp, -SPAN_MAX), SPAN_MAX);
            float t1[3], t2[3], t3[3], t4[3];
            const float k1 = 1.0f / 3.0f - 0.5f, k2 = 2.0f / 3.0f - 0.5f;
            im.bilinear((x + dx * k1) / w, (y + dy * k1) / h, t1);
            im.bilinear((x + dx * k2) / w, (y + dy * k2) / h, t2);
            im.bilinear((x + dx * (-0.5f)) / w, (y + dy * (-0.5f)) / h, t3);
            im.bilinear((x + dx * 0.5f) / w, (y + dy * 0.5f) / h, t4);
            float A[3], B[3];
            for (int k = 0; k < 3; k++) {
                A[k] = t1[k] * 0.5f + t2[k] * 0.5f;
                B[k] = 0.5f * A[k] + (t3[k] * 0.25f + t4[k] * 0.25f);
            }
            float lB = luma_ref(B[0], B[1], B[2]);
            float *o = out + 3 * ((size_t)y * w + x);
            const float *src = (lB < lMin || lB > lMax) ? A : B;
            o[0] = src[0]; o[1] = src[1]; o[2] = src[2];
        }
}

// combineSamples (kernels/ssaa.cuh:109-131)
void combine(const float *rgb, int S, size_t npix, float *image)
{
    for (size_t p = 0; p < npix; p++) {
        float c[3] = {0, 0, 0};
        if (S == 1) {
            for (int k = 0; k < 3; k++) c[k] = fminf(fmaxf(rgb[3 * p + k], 0.0f), 1.0f);
        } else {
            for (int s = 0; s < S; s++)
                for (int k = 0; k < 3; k++) {
                    float v = rgb[3 * (p * S + s) + k];
                    c[k] += fminf(fmaxf(v * v, 0.0f), 1.0f);
                }
            for (int k = 0; k < 3; k++) c[k] = sqrtf(c[k] / (float)S);
        }
        for (int k = 0; k < 3; k++) image[3 * p + k] = c[k];
    }
}

Scene make_scene(const prr_frame_desc *d, const uint8_t *const *tex, const int *tw, const int *th)
{
    Scene sc;
    sc.d = d;
    for (int i = 0; i < PRR_MAX_TEXTURES; i++) {
        if (tex && tex[i]) { sc.tex[i].p = tex[i]; sc.tex[i].w = tw[i]; sc.tex[i].h = th[i]; }
    }
    if (g_plasma.present) sc.plasma = &g_plasma;
    return sc;
}

template <class T>
void trace_list(const Scene &sc, const long long *ids, long long n, int nthreads, double *state, float *rgb,
                double *emis = nullptr)
{
    Tracer<T> tr(sc);
#pragma omp parallel for schedule(dynamic, 16) num_threads(nthreads > 0 ? nthreads : 1)
    for (long long k = 0; k < n; k++) {
        RayState<T> R = tr.run(ids ? ids[k] : k);
        if (state) {
            double *s = state + 13 * k;
            s[0] = R.uvx; s[1] = R.uvy; s[2] = R.result;
            s[3] = R.r.x; s[4] = R.r.y; s[5] = R.r.z; s[6] = R.r.w;
            s[7] = R.u.x; s[8] = R.u.y; s[9] = R.u.z; s[10] = R.u.w;
            s[11] = (double)R.accepted; s[12] = (double)R.attempts;
        }
        if (rgb) { rgb[3 * k] = R.rgb.x; rgb[3 * k + 1] = R.rgb.y; rgb[3 * k + 2] = R.rgb.z; }
        if (emis) { emis[3 * k] = (double)R.I; emis[3 * k + 1] = (double)R.trans; emis[3 * k + 2] = (double)R.nu_cam; }
    }
}

}  // namespace

extern "C" {

// Traces the rays `ids[0..n)` (ray index = (y*width + x)*samples + sample;
// ids == NULL means 0..n-1) of frame `d`.  precision: 0 = FP32, 1 = FP64
// (PHYSICAL mode only).  tex/tw/th: PRR_MAX_TEXTURES RGBA8 textures by id
// (NULL entries absent).  Outputs per ray (may be NULL):
//   state[13]: uv.x uv.y result r.x r.y r.z r.w u.x u.y u.z u.w accepted attempts
//   rgb[3]:    per-sample colour (rayToRGB)
int prr_oracle_trace(const prr_frame_desc *d, const uint8_t *const *tex, const int *tw, const int *th,
                     int precision, const long long *ids, long long n, int nthreads, double *state, float *rgb)
{
    if (!d || n < 0) return 1;
    if (d->ssaa == PRR_SSAA_REGULAR || d->ssaa == PRR_SSAA_JITTERED) {
        int q = (int)roundf(sqrtf((float)d->samples));
        if (q * q != d->samples) return 1;
    }
    if (d->mode == PRR_MODE_REFERENCE && precision != 0) return 1;
    Scene sc = make_scene(d, tex, tw, th);
    if (precision == 1) trace_list<double>(sc, ids, n, nthreads, state, rgb);
    else trace_list<float>(sc, ids, n, nthreads, state, rgb);
    return 0;
}

// Plasma emission per ray: emis[3] = I, transmittance, nu_cam (the camera
// frequency); otherwise as prr_oracle_trace.
int prr_oracle_trace_emission(const prr_frame_desc *d, const uint8_t *const *tex, const int *tw, const int *th,
                              int precision, const long long *ids, long long n, int nthreads, double *emis)
{
    if (!d || n < 0 || d->mode != PRR_MODE_PHYSICAL) return 1;
    Scene sc = make_scene(d, tex, tw, th);
    if (precision == 1) trace_list<double>(sc, ids, n, nthreads, nullptr, nullptr, emis);
    else trace_list<float>(sc, ids, n, nthreads, nullptr, nullptr, emis);
    return 0;
}

// The plasma grid of GRID emission (as prr_upload_plasma takes it); NULL
// clears it.  Returns 1 on a bad descriptor.
int prr_oracle_set_plasma(const prr_plasma_desc *p)
{
    g_plasma = Plasma();
    if (!p) return 0;
    if (!p->density || p->nx < 2 || p->ny < 2 || p->nz < 2) return 1;
    const size_t nn = (size_t)p->nx * p->ny * p->nz;
    g_plasma.nx = p->nx; g_plasma.ny = p->ny; g_plasma.nz = p->nz;
    const int dim[3] = {p->nx, p->ny, p->nz};
    for (int k = 0; k < 3; k++) {
        if (!(p->hi[k] > p->lo[k])) return 1;
        g_plasma.lo[k] = p->lo[k];
        g_plasma.inv[k] = (float)(dim[k] - 1) / (p->hi[k] - p->lo[k]);
    }
    g_plasma.n.assign(p->density, p->density + nn);
    if (p->temperature) g_plasma.theta.assign(p->temperature, p->temperature + nn);
    if (p->velocity) g_plasma.vel.assign(p->velocity, p->velocity + 3 * nn);
    g_plasma.present = true;
    return 0;
}

// SSAA combine and optional FXAA of per-sample colours (rgb: W*H*S*3).
// FP64 host gradient of sum(dL_dimage * image) with respect to (spin, mass,
// camera inclination, camera distance, orbital phase of sphere
// `sphere_index`), by forward-mode dual numbers through the PHYSICAL-mode
// trace with the step sizes and discrete events of the primal run frozen -
// the same discrete map the GPU adjoint differentiates in reverse.  The frame
// must use an orbit camera (position (r sin i, 0, r cos i)).  image_out
// (optional, W*H*3) receives the combined image of the primal run.
// params (optional) overrides the parameter values taken from the frame:
// (spin, mass, inclination, camera distance, sphere phase), in FP64 - the
// finite-difference tests perturb them below float resolution.
// loss_out (optional) receives sum(dL_dimage * image) in FP64; sig_out
// (optional, one per pixel) a signature of the pixel's discrete events (each
// sample's result and accepted-step count) for finite-difference tests.
int prr_oracle_grad(const prr_frame_desc *d, const uint8_t *const *tex, const int *tw, const int *th,
                    const float *dL_dimage, int sphere_index, int nthreads, double grads[5], double *image_out,
                    const double *params, double *loss_out, long long *sig_out)
{
    typedef HD<5> D;
    if (!d || !dL_dimage || !grads || d->mode != PRR_MODE_PHYSICAL || d->fxaa || d->emission != PRR_EMISSION_NONE) return 1;
    Scene sc = make_scene(d, tex, tw, th);
    double px = d->cam_pos[0], py = d->cam_pos[1], pz = d->cam_pos[2];
    double r = std::sqrt(px * px + py * py + pz * pz);
    double pv[5] = {d->metric == PRR_METRIC_KERR ? (double)d->spin : 0.0, (double)d->mass, std::acos(pz / r), r, 0.0};
    Orbit<D> orb;
    orb.sphere = sphere_index;
    if (sphere_index >= 0 && sphere_index < d->nspheres) {
        const prr_sphere &S = d->spheres[sphere_index];
        orb.sph_R = D(std::hypot((double)S.center[0], (double)S.center[1]));
        pv[4] = std::atan2((double)S.center[1], (double)S.center[0]);
        orb.sph_z = D((double)S.center[2]);
    } else orb.sphere = -1;
    if (params)
        for (int k = 0; k < 5; k++) pv[k] = params[k];
    orb.incl = D::var(pv[2], 2);
    orb.cam_r = D::var(pv[3], 3);
    orb.sph_phase = D::var(pv[4], 4);
    D M = D::var(pv[1], 1), a = D::var(pv[0], 0);
    Tracer<D> tr(sc, M, a, &orb);
    const long long npx = (long long)d->width * d->height;
    const int S = d->samples;
    double acc[5] = {0, 0, 0, 0, 0}, loss = 0.0;
#pragma omp parallel num_threads(nthreads > 0 ? nthreads : 1)
    {
        double loc[5] = {0, 0, 0, 0, 0}, loc_loss = 0.0;
#pragma omp for schedule(dynamic, 8)
        for (long long p = 0; p < npx; p++) {
            D I[3];
            long long sig = 0;
            if (S == 1) {
                RayState<D> R = tr.run(p);
                sig = R.result * 1000003LL + R.accepted + (long long)(R.cells * 7919ULL);
                const D c[3] = {R.rgbT.x, R.rgbT.y, R.rgbT.z};
                for (int k = 0; k < 3; k++) I[k] = c[k].v <= 0 ? D(0.0) : (c[k].v >= 1 ? D(1.0) : c[k]);
            } else {
                D sum[3] = {D(0.0), D(0.0), D(0.0)};
                for (int s = 0; s < S; s++) {
                    RayState<D> R = tr.run(p * S + s);
                    sig = sig * 31 + R.result * 1000003LL + R.accepted + (long long)(R.cells * 7919ULL);
                    const D c[3] = {R.rgbT.x, R.rgbT.y, R.rgbT.z};
                    for (int k = 0; k < 3; k++) {
                        D c2 = c[k] * c[k];
                        sum[k] += c2.v <= 0 ? D(0.0) : (c2.v >= 1 ? D(1.0) : c2);
                    }
                }
                for (int k = 0; k < 3; k++) I[k] = sqrt(sum[k] / (double)S);
            }
            for (int k = 0; k < 3; k++) {
                double g = dL_dimage[3 * p + k];
                for (int j = 0; j < 5; j++) loc[j] += g * I[k].d[j];
                loc_loss += g * I[k].v;
                if (image_out) image_out[3 * p + k] = I[k].v;
            }
            if (sig_out) sig_out[p] = sig;
        }
#pragma omp critical
        {
            for (int j = 0; j < 5; j++) acc[j] += loc[j];
            loss += loc_loss;
        }
    }
    for (int j = 0; j < 5; j++) grads[j] = acc[j];
    if (loss_out) *loss_out = loss;
    return 0;
}

int prr_oracle_post(const float *rgb, int w, int h, int samples, int do_fxaa, float *image)
{
    size_t npix = (size_t)w * h;
    std::vector<float> tmp(3 * npix);
    combine(rgb, samples, npix, do_fxaa ? tmp.data() : image);
    if (do_fxaa) fxaa_ref(tmp.data(), image, w, h);
    return 0;
}

// Whole frame: trace every ray, combine, FXAA if d->fxaa.
int prr_oracle_render(const prr_frame_desc *d, const uint8_t *const *tex, const int *tw, const int *th,
                      int precision, int nthreads, double *state, float *rgb_out, float *image)
{
    long long n = (long long)d->width * d->height * d->samples;
    std::vector<float> rgb(3 * (size_t)n);
    int rc = prr_oracle_trace(d, tex, tw, th, precision, nullptr, n, nthreads, state, rgb.data());
    if (rc) return rc;
    if (rgb_out) memcpy(rgb_out, rgb.data(), sizeof(float) * rgb.size());
    if (image) prr_oracle_post(rgb.data(), d->width, d->height, d->samples, d->fxaa, image);
    return 0;
}

// Geodesic right-hand side (for known-answer tests): du/dlambda at (p, u).
// refmode selects the reference's FP32 Schwarzschild formula.
void prr_oracle_geod(int metric, double M, double a, const double p[4], const double u[4], int refmode, double out[4])
{
    if (refmode) {
        Metric<float> mt;
        mt.kind = metric; mt.M = (float)M; mt.a = (float)a; mt.rs = (float)(2.0f * (float)M);
        V4<float> r = mt.geod({(float)p[0], (float)p[1], (float)p[2], (float)p[3]}, {(float)u[0], (float)u[1], (float)u[2], (float)u[3]}, true);
        out[0] = r.x; out[1] = r.y; out[2] = r.z; out[3] = r.w;
        return;
    }
    Metric<double> mt;
    mt.kind = metric; mt.M = M; mt.a = a; mt.rs = 2 * M;
    V4<double> r = mt.geod({p[0], p[1], p[2], p[3]}, {u[0], u[1], u[2], u[3]}, false);
    out[0] = r.x; out[1] = r.y; out[2] = r.z; out[3] = r.w;
}

void prr_oracle_metric(int metric, double M, double a, const double p[4], double g[16])
{
    metric_ks<double>({p[0], p[1], p[2], p[3]}, metric == PRR_METRIC_FLAT ? 0.0 : M, metric == PRR_METRIC_KERR ? a : 0.0, g);
}

}  // extern "C"
