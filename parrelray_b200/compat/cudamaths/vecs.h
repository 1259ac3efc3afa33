#pragma once
// Compatibility vector types for ParRelRay metric plug-in headers.
//
// A metric header written for the reference (metrics/*.cuh) includes
// "../cudamaths/mats.h" and uses the small vector classes of the reference's
// cudamaths/ directory (f2/f3/f4, i2/i3/i4: cudamaths/f2.cuh .. i4.cuh,
// cudamaths/if_interop.cuh).  This header provides the same class names,
// members, constructors and free functions so such a header compiles
// unchanged against prr-b200.  Component-wise arithmetic is spelled out in
// component order (x, y, z, w) in FP32, as the reference evaluates it, so a
// plug-in compiled here computes what it computes in the reference.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cuda_runtime.h>

#define PRR_VHD __host__ __device__ inline

PRR_VHD float sq(float x) { return x * x; }

// ---------------------------------------------------------------- floats
class f2 {
public:
    float x, y;
    PRR_VHD f2() : x(0), y(0) {}
    PRR_VHD f2(float k) : x(k), y(k) {}
    PRR_VHD f2(float a, float b) : x(a), y(b) {}
    PRR_VHD const f2 &operator+() const { return *this; }
    PRR_VHD f2 operator-() const { return f2(-x, -y); }
    PRR_VHD float norm() { return sqrtf(x * x + y * y); }
    PRR_VHD float norm2() { return x * x + y * y; }
    PRR_VHD void normalize() { float k = 1.0f / norm(); x *= k; y *= k; }
    PRR_VHD void cinv() { x = 1.0f / x; y = 1.0f / y; }
};

class f3 {
public:
    float x, y, z;
    PRR_VHD f3() : x(0), y(0), z(0) {}
    PRR_VHD f3(float k) : x(k), y(k), z(k) {}
    PRR_VHD f3(float a, float b, float c) : x(a), y(b), z(c) {}
    PRR_VHD const f3 &operator+() const { return *this; }
    PRR_VHD f3 operator-() const { return f3(-x, -y, -z); }
    PRR_VHD f2 xy() { return f2(x, y); }
    PRR_VHD f2 xz() { return f2(x, z); }
    PRR_VHD f2 yz() { return f2(y, z); }
    PRR_VHD float norm() { return sqrtf(x * x + y * y + z * z); }
    PRR_VHD float norm2() { return x * x + y * y + z * z; }
    PRR_VHD void normalize() { float k = 1.0f / norm(); x *= k; y *= k; z *= k; }
    PRR_VHD void cinv() { x = 1.0f / x; y = 1.0f / y; z = 1.0f / z; }
};

class f4 {
public:
    float x, y, z, w;
    PRR_VHD f4() : x(0), y(0), z(0), w(0) {}
    PRR_VHD f4(float k) : x(k), y(k), z(k), w(k) {}
    PRR_VHD f4(float a, float b, float c, float d) : x(a), y(b), z(c), w(d) {}
    PRR_VHD f4(const f3 &v, float d) : x(v.x), y(v.y), z(v.z), w(d) {}
    PRR_VHD const f4 &operator+() const { return *this; }
    PRR_VHD f4 operator-() const { return f4(-x, -y, -z, -w); }
    PRR_VHD f3 xyz() { return f3(x, y, z); }
    PRR_VHD float norm() { return sqrtf(x * x + y * y + z * z + w * w); }
    PRR_VHD float norm2() { return x * x + y * y + z * z + w * w; }
    PRR_VHD void normalize() { float k = 1.0f / norm(); x *= k; y *= k; z *= k; w *= k; }
    PRR_VHD void cinv() { x = 1.0f / x; y = 1.0f / y; z = 1.0f / z; w = 1.0f / w; }
};

// ---------------------------------------------------------------- ints
class i2 {
public:
    int x, y;
    PRR_VHD i2() : x(0), y(0) {}
    PRR_VHD i2(int k) : x(k), y(k) {}
    PRR_VHD i2(int a, int b) : x(a), y(b) {}
    PRR_VHD const i2 &operator+() const { return *this; }
    PRR_VHD i2 operator-() const { return i2(-x, -y); }
    PRR_VHD float norm() { return sqrtf((float)(x * x + y * y)); }
    PRR_VHD int norm2() { return x * x + y * y; }
};

class i3 {
public:
    int x, y, z;
    PRR_VHD i3() : x(0), y(0), z(0) {}
    PRR_VHD i3(int k) : x(k), y(k), z(k) {}
    PRR_VHD i3(int a, int b, int c) : x(a), y(b), z(c) {}
    PRR_VHD const i3 &operator+() const { return *this; }
    PRR_VHD i3 operator-() const { return i3(-x, -y, -z); }
    PRR_VHD float norm() { return sqrtf((float)(x * x + y * y + z * z)); }
    PRR_VHD int norm2() { return x * x + y * y + z * z; }
};

class i4 {
public:
    int x, y, z, w;
    PRR_VHD i4() : x(0), y(0), z(0), w(0) {}
    PRR_VHD i4(int k) : x(k), y(k), z(k), w(k) {}
    PRR_VHD i4(int a, int b, int c, int d) : x(a), y(b), z(c), w(d) {}
    PRR_VHD const i4 &operator+() const { return *this; }
    PRR_VHD i4 operator-() const { return i4(-x, -y, -z, -w); }
    PRR_VHD float norm() { return sqrtf((float)(x * x + y * y + z * z + w * w)); }
    PRR_VHD int norm2() { return x * x + y * y + z * z + w * w; }
};

// Component-wise helpers: apply OP to each component, in component order.
#define PRR_EW2(R, a, b, OP) R((a).x OP (b).x, (a).y OP (b).y)
#define PRR_EW3(R, a, b, OP) R((a).x OP (b).x, (a).y OP (b).y, (a).z OP (b).z)
#define PRR_EW4(R, a, b, OP) R((a).x OP (b).x, (a).y OP (b).y, (a).z OP (b).z, (a).w OP (b).w)
#define PRR_ES2(R, a, t, OP) R((a).x OP (t), (a).y OP (t))
#define PRR_ES3(R, a, t, OP) R((a).x OP (t), (a).y OP (t), (a).z OP (t))
#define PRR_ES4(R, a, t, OP) R((a).x OP (t), (a).y OP (t), (a).z OP (t), (a).w OP (t))

// vector (op) vector, vector * scalar, scalar * vector, vector / scalar, and
// the compound assignments, for one float class V of N components.
#define PRR_FLOAT_OPS(V, N)                                                                             \
    PRR_VHD V operator+(const V &a, const V &b) { return PRR_EW##N(V, a, b, +); }                   \
    PRR_VHD V operator-(const V &a, const V &b) { return PRR_EW##N(V, a, b, -); }                   \
    PRR_VHD V operator*(const V &a, const V &b) { return PRR_EW##N(V, a, b, *); }                   \
    PRR_VHD V operator/(const V &a, const V &b) { return PRR_EW##N(V, a, b, /); }                   \
    PRR_VHD V operator*(float t, const V &a) { return PRR_ES##N(V, a, t, *); }                      \
    PRR_VHD V operator*(const V &a, float t) { return PRR_ES##N(V, a, t, *); }                      \
    PRR_VHD V operator/(const V &a, float t) { return PRR_ES##N(V, a, t, /); }                      \
    PRR_VHD V &operator+=(V &a, const V &b) { a = a + b; return a; }                                \
    PRR_VHD V &operator-=(V &a, const V &b) { a = a - b; return a; }                                \
    PRR_VHD V &operator*=(V &a, const V &b) { a = a * b; return a; }                                \
    PRR_VHD V &operator/=(V &a, const V &b) { a = a / b; return a; }                                \
    PRR_VHD V &operator*=(V &a, float t) { a = a * t; return a; }                                   \
    PRR_VHD V &operator/=(V &a, float t) { a = a / t; return a; }

#define PRR_INT_OPS(V, N)                                                                               \
    PRR_VHD V operator+(const V &a, const V &b) { return PRR_EW##N(V, a, b, +); }                   \
    PRR_VHD V operator-(const V &a, const V &b) { return PRR_EW##N(V, a, b, -); }                   \
    PRR_VHD V operator*(const V &a, const V &b) { return PRR_EW##N(V, a, b, *); }                   \
    PRR_VHD V operator*(int t, const V &a) { return PRR_ES##N(V, a, t, *); }                        \
    PRR_VHD V operator*(const V &a, int t) { return PRR_ES##N(V, a, t, *); }                        \
    PRR_VHD V &operator+=(V &a, const V &b) { a = a + b; return a; }                                \
    PRR_VHD V &operator-=(V &a, const V &b) { a = a - b; return a; }                                \
    PRR_VHD V &operator*=(V &a, const V &b) { a = a * b; return a; }                                \
    PRR_VHD V &operator*=(V &a, int t) { a = a * t; return a; }

PRR_FLOAT_OPS(f2, 2)
PRR_FLOAT_OPS(f3, 3)
PRR_FLOAT_OPS(f4, 4)
PRR_INT_OPS(i2, 2)
PRR_INT_OPS(i3, 3)
PRR_INT_OPS(i4, 4)

// mixed int/float (cudamaths/if_interop.cuh): the result is a float vector
#define PRR_MIXED_OPS(F, I, N)                                                                          \
    PRR_VHD F operator+(const F &a, const I &b) { return PRR_EW##N(F, a, b, +); }                   \
    PRR_VHD F operator-(const F &a, const I &b) { return PRR_EW##N(F, a, b, -); }                   \
    PRR_VHD F operator*(const F &a, const I &b) { return PRR_EW##N(F, a, b, *); }                   \
    PRR_VHD F operator/(const F &a, const I &b) { return PRR_EW##N(F, a, b, /); }                   \
    PRR_VHD F operator+(const I &a, const F &b) { return PRR_EW##N(F, a, b, +); }                   \
    PRR_VHD F operator-(const I &a, const F &b) { return PRR_EW##N(F, a, b, -); }                   \
    PRR_VHD F operator*(const I &a, const F &b) { return PRR_EW##N(F, a, b, *); }                   \
    PRR_VHD F operator/(const I &a, const F &b) { return PRR_EW##N(F, a, b, /); }                   \
    PRR_VHD F operator*(float t, const I &a) { return PRR_ES##N(F, a, t, *); }                      \
    PRR_VHD F operator*(const I &a, float t) { return PRR_ES##N(F, a, t, *); }                      \
    PRR_VHD F operator/(const I &a, float t) { return PRR_ES##N(F, a, t, /); }

PRR_MIXED_OPS(f2, i2, 2)
PRR_MIXED_OPS(f3, i3, 3)
PRR_MIXED_OPS(f4, i4, 4)
PRR_VHD f2 operator/(const i2 &a, const i2 &b) { return f2((float)a.x / b.x, (float)a.y / b.y); }
PRR_VHD f3 operator/(const i3 &a, const i3 &b) { return f3((float)a.x / b.x, (float)a.y / b.y, (float)a.z / b.z); }
PRR_VHD f4 operator/(const i4 &a, const i4 &b) { return f4((float)a.x / b.x, (float)a.y / b.y, (float)a.z / b.z, (float)a.w / b.w); }

// ---------------------------------------------------------------- functions
PRR_VHD float dot(const f2 &a, const f2 &b) { return a.x * b.x + a.y * b.y; }
PRR_VHD float dot(const f3 &a, const f3 &b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
PRR_VHD float dot(const f4 &a, const f4 &b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
PRR_VHD int dot(const i2 &a, const i2 &b) { return a.x * b.x + a.y * b.y; }
PRR_VHD f3 cross(const f3 &a, const f3 &b) { return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
PRR_VHD float norm2(const f2 &a) { return a.x * a.x + a.y * a.y; }
PRR_VHD float norm2(const f3 &a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
PRR_VHD float norm2(const f4 &a) { return a.x * a.x + a.y * a.y + a.z * a.z + a.w * a.w; }
PRR_VHD float norm(const f2 &a) { return sqrtf(a.x * a.x + a.y * a.y); }
PRR_VHD float norm(const f3 &a) { return sqrtf(a.x * a.x + a.y * a.y + a.z * a.z); }
PRR_VHD float norm(const f4 &a) { return sqrtf(a.x * a.x + a.y * a.y + a.z * a.z + a.w * a.w); }
PRR_VHD int norm2(const i2 &a) { return a.x * a.x + a.y * a.y; }
PRR_VHD float norm(const i2 &a) { return sqrtf((float)(a.x * a.x + a.y * a.y)); }
PRR_VHD float norm(const i3 &a) { return sqrtf((float)(a.x * a.x + a.y * a.y + a.z * a.z)); }
PRR_VHD float norm(const i4 &a) { return sqrtf((float)(a.x * a.x + a.y * a.y + a.z * a.z + a.w * a.w)); }
PRR_VHD f2 normalize(const f2 &a) { float k = 1.0f / norm(a); return k * a; }
PRR_VHD f3 normalize(const f3 &a) { float k = 1.0f / norm(a); return k * a; }
PRR_VHD f4 normalize(const f4 &a) { float k = 1.0f / norm(a); return k * a; }
PRR_VHD f2 normalize(const i2 &a) { float k = 1.0f / norm(a); return k * a; }
PRR_VHD f3 normalize(const i3 &a) { float k = 1.0f / norm(a); return k * a; }
PRR_VHD f4 normalize(const i4 &a) { float k = 1.0f / norm(a); return k * a; }
PRR_VHD f2 cinv(const f2 &a) { return f2(1.0f / a.x, 1.0f / a.y); }
PRR_VHD f3 cinv(const f3 &a) { return f3(1.0f / a.x, 1.0f / a.y, 1.0f / a.z); }
PRR_VHD f4 cinv(const f4 &a) { return f4(1.0f / a.x, 1.0f / a.y, 1.0f / a.z, 1.0f / a.w); }
PRR_VHD f2 cinv(const i2 &a) { return f2(1.0f / a.x, 1.0f / a.y); }
PRR_VHD f3 cinv(const i3 &a) { return f3(1.0f / a.x, 1.0f / a.y, 1.0f / a.z); }
PRR_VHD f4 cinv(const i4 &a) { return f4(1.0f / a.x, 1.0f / a.y, 1.0f / a.z, 1.0f / a.w); }
PRR_VHD f2 abs(const f2 &a) { return f2(fabsf(a.x), fabsf(a.y)); }
PRR_VHD f3 abs(const f3 &a) { return f3(fabsf(a.x), fabsf(a.y), fabsf(a.z)); }
PRR_VHD f4 abs(const f4 &a) { return f4(fabsf(a.x), fabsf(a.y), fabsf(a.z), fabsf(a.w)); }
PRR_VHD f2 cmin(const f2 &a, const f2 &b) { return f2(fminf(a.x, b.x), fminf(a.y, b.y)); }
PRR_VHD f3 cmin(const f3 &a, const f3 &b) { return f3(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)); }
PRR_VHD f4 cmin(const f4 &a, const f4 &b) { return f4(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z), fminf(a.w, b.w)); }
PRR_VHD f2 cmax(const f2 &a, const f2 &b) { return f2(fmaxf(a.x, b.x), fmaxf(a.y, b.y)); }
PRR_VHD f3 cmax(const f3 &a, const f3 &b) { return f3(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)); }
PRR_VHD f4 cmax(const f4 &a, const f4 &b) { return f4(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z), fmaxf(a.w, b.w)); }
PRR_VHD i2 cmin(const i2 &a, const i2 &b) { return i2(a.x < b.x ? a.x : b.x, a.y < b.y ? a.y : b.y); }
PRR_VHD i2 cmax(const i2 &a, const i2 &b) { return i2(a.x > b.x ? a.x : b.x, a.y > b.y ? a.y : b.y); }
PRR_VHD f2 clamp(const f2 &v, const f2 &lo, const f2 &hi) { return cmin(cmax(v, lo), hi); }
PRR_VHD f3 clamp(const f3 &v, const f3 &lo, const f3 &hi) { return cmin(cmax(v, lo), hi); }
PRR_VHD f4 clamp(const f4 &v, const f4 &lo, const f4 &hi) { return cmin(cmax(v, lo), hi); }
PRR_VHD i2 clamp(const i2 &v, const i2 &lo, const i2 &hi) { return cmin(cmax(v, lo), hi); }
PRR_VHD f3 nmin(const f3 &a, const f3 &b) { return norm2(a) < norm2(b) ? a : b; }
PRR_VHD f3 nmax(const f3 &a, const f3 &b) { return norm2(a) > norm2(b) ? a : b; }
PRR_VHD float min(const f4 &a) { return fminf(fminf(fminf(a.x, a.y), a.z), a.w); }
PRR_VHD float max(const f4 &a) { return fmaxf(fmaxf(fmaxf(a.x, a.y), a.z), a.w); }
PRR_VHD f3 sqrt(const f3 &a) { return f3(sqrtf(a.x), sqrtf(a.y), sqrtf(a.z)); }
PRR_VHD f3 sq(const f3 &a) { return f3(a.x * a.x, a.y * a.y, a.z * a.z); }
PRR_VHD bool isnan(const f2 &a) { return isnan(a.x) || isnan(a.y); }
PRR_VHD bool isnan(const f3 &a) { return isnan(a.x) || isnan(a.y) || isnan(a.z); }
PRR_VHD bool isnan(const f4 &a) { return isnan(a.x) || isnan(a.y) || isnan(a.z) || isnan(a.w); }
PRR_VHD f3 avg(const f3 &a, const f3 &b) { return f3(0.5f * (a.x + b.x), 0.5f * (a.y + b.y), 0.5f * (a.z + b.z)); }
PRR_VHD f3 avg(const f3 &a, const f3 &b, const f3 &c, const f3 &d)
{
    return f3(0.25f * (a.x + b.x + c.x + d.x), 0.25f * (a.y + b.y + c.y + d.y), 0.25f * (a.z + b.z + c.z + d.z));
}
// root mean square of four colours, per channel (the background filter of
// main/base.h:119-162)
PRR_VHD f3 sqavg(const f3 &a, const f3 &b, const f3 &c, const f3 &d)
{
    return f3(sqrtf(0.25f * (a.x * a.x + b.x * b.x + c.x * c.x + d.x * d.x)),
              sqrtf(0.25f * (a.y * a.y + b.y * b.y + c.y * c.y + d.y * d.y)),
              sqrtf(0.25f * (a.z * a.z + b.z * b.z + c.z * c.z + d.z * d.z)));
}
PRR_VHD i2 floor(const f2 &a) { return i2((int)floorf(a.x), (int)floorf(a.y)); }
PRR_VHD i3 floor(const f3 &a) { return i3((int)floorf(a.x), (int)floorf(a.y), (int)floorf(a.z)); }
PRR_VHD i2 ceil(const f2 &a) { return i2((int)ceilf(a.x), (int)ceilf(a.y)); }
PRR_VHD i2 round(const f2 &a) { return i2((int)roundf(a.x), (int)roundf(a.y)); }
PRR_VHD f2 f2_zero() { return f2(0, 0); }
PRR_VHD f3 f3_zero() { return f3(0, 0, 0); }
PRR_VHD f4 f4_zero() { return f4(0, 0, 0, 0); }
PRR_VHD f3 f3_id() { return f3(1, 1, 1); }
PRR_VHD f4 f4_id() { return f4(1, 1, 1, 1); }
PRR_VHD i2 i2_zero() { return i2(0, 0); }

// Cartesian <-> spherical conversions (the reference's vecs.h includes them)
#include "transform.cuh"
