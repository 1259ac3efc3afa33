// emission.cuh - plasma emission integrated along a ray (the luminosity
// Ray::I of main/base.h:175 and the plasma fields of main/Spacetime.h:50-51,
// which the reference declares and never uses).  The model and its
// conventions are stated with prr_emission in include/prr.h; in short, at
// every accepted step of affine length h:
//     g      = nu_cam / nu_e,  nu = -k.u  (k the ray's 4-momentum)
//     I     += trans * g^(2 + spectral) * j * nu_cam * h
//     trans *= exp(-absorb * n * nu_cam * h / g)
// and the pixel colour is trans * colour + map(gain * I).
//
// Kerr-Schild form g_mn = eta_mn + f l_m l_n, (x, y, z, t) order, l_t = 1:
// every inner product is eta(A, B) + f (l.A)(l.B), so no 4x4 metric is built.
#pragma once
#include "prr_device.cuh"

namespace prr {

// a / b and a^e: in FP32 a multiplication by the SFU reciprocal and the SFU
// power (the renderer's FP32 convention, prr_device.cuh:frcp/fpow) unless
// built with PRR_EMIS_FAST=0; in FP64 the IEEE division and pow
#ifndef PRR_EMIS_FAST
#define PRR_EMIS_FAST 1
#endif
template <class T> PRR_DEV T ediv(T a, T b) { return a / b; }
template <class T> PRR_DEV T epow(T b, T e) { return pow(b, e); }
#if PRR_EMIS_FAST
template <> PRR_DEV float ediv<float>(float a, float b) { return a * frcp<float>(b); }
template <> PRR_DEV float epow<float>(float b, float e) { return fpow<float>(b, e); }
#endif

template <class T> struct EmisRay {
    T I;       // accumulated intensity
    T trans;   // transmittance from the camera to the current point
    T nu_cam;  // -k.u_cam at the camera
};

// f and l_x, l_y, l_z of the Kerr-Schild metric at (x, y, z), and the
// Kerr-Schild r; flat (M = 0): f = 0.
template <class T> PRR_DEV void ks_fl_at(T x, T y, T z, T M, T a, T r, T &f, T l[3])
{
    f = 0; l[0] = l[1] = l[2] = 0;
    if (M != (T)0) {
        const T r2 = r * r, q = r2 + a * a;
        f = ediv<T>((T)2 * M * r2 * r, r2 * r2 + a * a * z * z);
        l[0] = ediv<T>(r * x + a * y, q); l[1] = ediv<T>(r * y - a * x, q); l[2] = ediv<T>(z, r);
    }
}
template <class T> PRR_DEV void ks_fl(T x, T y, T z, T M, T a, T &r, T &f, T l[3])
{
    r = ks_radius<T>(x, y, z, a);
    ks_fl_at<T>(x, y, z, M, a, r, f, l);
}

// nu_cam of a static observer at the camera: -k_t / sqrt(-g_tt).  The camera
// is outside the ergoregion (f < 1; checked when the frame is validated).
template <class T> PRR_DEV void emis_init(const FrameParams &fp, const V4<T> &x, const V4<T> &k, EmisRay<T> &E)
{
    const T M = fp.metric == PRR_METRIC_FLAT ? (T)0 : (T)fp.M;
    const T a = fp.metric == PRR_METRIC_KERR ? (T)fp.a : (T)0;
    T r, f, l[3];
    ks_fl<T>(x.x, x.y, x.z, M, a, r, f, l);
    const T lk = l[0] * k.x + l[1] * k.y + l[2] * k.z + k.w;
    E.nu_cam = (k.w - f * lk) / sqrt((T)1 - f);
    E.I = 0;
    E.trans = 1;
}

// Trilinear sample of the grid at (x, y, z); false outside the box.
template <class T>
PRR_DEV bool plasma_sample(const DevPlasma &G, T x, T y, T z, T &n, T &theta, T v[3])
{
    const T fx = (x - (T)G.lo[0]) * (T)G.inv[0], fy = (y - (T)G.lo[1]) * (T)G.inv[1], fz = (z - (T)G.lo[2]) * (T)G.inv[2];
    if (!(fx >= (T)0 && fx <= (T)(G.nx - 1) && fy >= (T)0 && fy <= (T)(G.ny - 1) && fz >= (T)0 && fz <= (T)(G.nz - 1)))
        return false;
    const int i = min((int)fx, G.nx - 2), j = min((int)fy, G.ny - 2), k = min((int)fz, G.nz - 2);
    const T tx = fx - (T)i, ty = fy - (T)j, tz = fz - (T)k;
    const long long sy = G.nx, sz = (long long)G.nx * G.ny;
    const long long c = i + sy * j + sz * k;
    const long long o[8] = {c, c + 1, c + sy, c + sy + 1, c + sz, c + sz + 1, c + sz + sy, c + sz + sy + 1};
    const T w[8] = {((T)1 - tx) * ((T)1 - ty) * ((T)1 - tz), tx * ((T)1 - ty) * ((T)1 - tz),
                    ((T)1 - tx) * ty * ((T)1 - tz),         tx * ty * ((T)1 - tz),
                    ((T)1 - tx) * ((T)1 - ty) * tz,         tx * ((T)1 - ty) * tz,
                    ((T)1 - tx) * ty * tz,                  tx * ty * tz};
    n = 0; theta = G.theta ? (T)0 : (T)1;
    v[0] = v[1] = v[2] = 0;
#pragma unroll
    for (int m = 0; m < 8; m++) {
        n += w[m] * (T)__ldg(G.n + o[m]);
        if (G.theta) theta += w[m] * (T)__ldg(G.theta + o[m]);
        if (G.vel) {
            const float4 q = __ldg(G.vel + o[m]);
            v[0] += w[m] * (T)q.x; v[1] += w[m] * (T)q.y; v[2] += w[m] * (T)q.z;
        }
    }
    return true;
}

// One accepted step ending at x with momentum k, of affine length h.
template <class T>
PRR_DEV void emis_step(const FrameParams &fp, T M, T a, const V4<T> &x, const V4<T> &k, T h, EmisRay<T> &E)
{
    const EmisParams &e = fp.em;
    if (e.kind == PRR_EMISSION_NONE) return;  // a frame without plasma in a batch with some
    const T r = ks_radius<T>(x.x, x.y, x.z, a);
    if (!(r >= (T)e.r_in && r <= (T)e.r_out)) return;  // outside the emitting shell: f and l are not needed
    T f, l[3];
    ks_fl_at<T>(x.x, x.y, x.z, M, a, r, f, l);
    T n, theta = 1, v[3];
    bool flow = false;
    if (e.kind == PRR_EMISSION_DISK) {
        const T c = ediv<T>(x.z, r), hh = (T)e.height;
        n = epow<T>(ediv<T>(r, (T)e.r_in), -(T)e.index) * exp(ediv<T>(-c * c, (T)2 * hh * hh));
    } else {
        if (!plasma_sample<T>(e.grid, x.x, x.y, x.z, n, theta, v)) return;
        flow = e.grid.vel != nullptr;
    }
    if (!(n > (T)0)) return;
    if (!flow) {  // circular orbits at the equatorial Keplerian angular velocity of r
        const T sm = sqrt(M), s = (T)e.sense;
        const T om = ediv<T>(s * sm, r * sqrt(r) + s * a * sm);
        v[0] = -om * x.y; v[1] = om * x.x; v[2] = 0;
    }
    const T lv = l[0] * v[0] + l[1] * v[1] + l[2] * v[2] + (T)1;
    const T N = v[0] * v[0] + v[1] * v[1] + v[2] * v[2] - (T)1 + f * lv * lv;  // g(xi, xi), xi = (v, 1)
    if (!(N < (T)0)) return;
    const T ut = ediv<T>((T)1, sqrt(-N));
    const T lk = l[0] * k.x + l[1] * k.y + l[2] * k.z + k.w;
    const T nu_e = -ut * (k.x * v[0] + k.y * v[1] + k.z * v[2] - k.w + f * lk * lv);
    if (!(nu_e > (T)0)) return;
    const T g = ediv<T>(E.nu_cam, nu_e);
    const T dl = E.nu_cam * h;
    T j = n;
    if (e.kind == PRR_EMISSION_GRID && e.temp_power != 0.0f) j *= pow(theta, (T)e.temp_power);
    const T w = e.spectral == 0.0f ? g * g : pow(g, (T)2 + (T)e.spectral);
    E.I += E.trans * w * j * dl;
    if (e.absorb > 0.0f) E.trans *= exp(ediv<T>(-(T)e.absorb * n * dl, g));
}

// The same step for a ray carried by its covariant momentum p_mu (the
// Hamiltonian form of the FP32 renderer): k.u_e = p_mu u_e^mu needs no
// lowering, so nu_e = -u_e^t (p_i v^i + p_t); p_t is the constant of the
// motion.  Same model, same arithmetic otherwise.
template <class T>
PRR_DEV void emis_step_p(const FrameParams &fp, T M, T a, T x, T y, T z, T px, T py, T pz, T pt, T h, EmisRay<T> &E)
{
    const EmisParams &e = fp.em;
    if (e.kind == PRR_EMISSION_NONE) return;
    const T r = ks_radius<T>(x, y, z, a);
    if (!(r >= (T)e.r_in && r <= (T)e.r_out)) return;  // outside the emitting shell: f and l are not needed
    T f, l[3];
    ks_fl_at<T>(x, y, z, M, a, r, f, l);
    T n, theta = 1, v[3];
    bool flow = false;
    if (e.kind == PRR_EMISSION_DISK) {
        const T c = ediv<T>(z, r), hh = (T)e.height;
        n = epow<T>(ediv<T>(r, (T)e.r_in), -(T)e.index) * exp(ediv<T>(-c * c, (T)2 * hh * hh));
    } else {
        if (!plasma_sample<T>(e.grid, x, y, z, n, theta, v)) return;
        flow = e.grid.vel != nullptr;
    }
    if (!(n > (T)0)) return;
    if (!flow) {
        const T sm = sqrt(M), s = (T)e.sense;
        const T om = ediv<T>(s * sm, r * sqrt(r) + s * a * sm);
        v[0] = -om * y; v[1] = om * x; v[2] = 0;
    }
    const T lv = l[0] * v[0] + l[1] * v[1] + l[2] * v[2] + (T)1;
    const T N = v[0] * v[0] + v[1] * v[1] + v[2] * v[2] - (T)1 + f * lv * lv;  // g(xi, xi), xi = (v, 1)
    if (!(N < (T)0)) return;
    const T ut = ediv<T>((T)1, sqrt(-N));
    const T nu_e = -ut * (px * v[0] + py * v[1] + pz * v[2] + pt);
    if (!(nu_e > (T)0)) return;
    const T g = ediv<T>(E.nu_cam, nu_e);
    const T dl = E.nu_cam * h;
    T j = n;
    if (e.kind == PRR_EMISSION_GRID && e.temp_power != 0.0f) j *= pow(theta, (T)e.temp_power);
    const T w = e.spectral == 0.0f ? g * g : pow(g, (T)2 + (T)e.spectral);
    E.I += E.trans * w * j * dl;
    if (e.absorb > 0.0f) E.trans *= exp(ediv<T>(-(T)e.absorb * n * dl, g));
}

// emis_init for the momentum form: nu_cam = -p_t / sqrt(1 - f) at the camera.
template <class T> PRR_DEV void emis_init_p(const FrameParams &fp, T x, T y, T z, T pt, EmisRay<T> &E)
{
    const T M = fp.metric == PRR_METRIC_FLAT ? (T)0 : (T)fp.M;
    const T a = fp.metric == PRR_METRIC_KERR ? (T)fp.a : (T)0;
    T r, f, l[3];
    ks_fl<T>(x, y, z, M, a, r, f, l);
    E.nu_cam = -pt / sqrt((T)1 - f);
    E.I = 0;
    E.trans = 1;
}

// The pixel colour of a finished ray: trans * colour + map(gain * I).
template <class T> PRR_DEV V3<float> emis_colour(const FrameParams &fp, const EmisRay<T> &E, V3<float> c)
{
    if (fp.em.kind == PRR_EMISSION_NONE) return c;
    const float x = (float)((T)fp.em.gain * E.I), tr = (float)E.trans;
    auto cl = [](float v) { return fminf(fmaxf(v, 0.0f), 1.0f); };
    V3<float> m;
    if (fp.em.cmap == PRR_CMAP_GREY) m = {cl(x), cl(x), cl(x)};
    else m = {cl(2.0f * x), cl(2.0f * x - 0.5f), cl(2.0f * x - 1.0f)};
    return {tr * c.x + m.x, tr * c.y + m.y, tr * c.z + m.z};
}

}  // namespace prr
