#pragma once
// Compatibility base types for ParRelRay metric plug-in headers (the shapes of
// main/base.h of the reference): the enums SOLVER, RESULT and SSAA_DISTR with
// the reference's values, BlackHole, the sky sphere OutSphere, the integrator
// parameters Tracer and the per-ray record Ray, plus the lowercase aliases
// `ray` and `tracer` that the reference's metric headers and solver use
// (metrics/schwarzschild.cuh:15,66; kernels/solver.cuh:26,68).  A metric
// header includes "../main/base.h", "../main/Camera.h", "../main/Spacetime.h"
// and "../cudamaths/mats.h"; placed in this tree's metrics/ directory it
// compiles against these files unchanged.
#include <cstdio>
#include <map>
#include <string>

#include "../cudamaths/mats.h"
#include "../cudamaths/tex2d.cuh"

#ifndef PI
#define PI 3.14159265358979323846
#endif
#define RAYPAR 1

typedef std::map<std::string, std::map<std::string, std::string>> map2d;

enum class SOLVER { EULER = 0, RUNGE_KUTTA = 1, RUNGE_KUTTA_FEHLBERG = 2, ADAMS = 3, GRAGG = 4, DORMAND = 5, TAYLOR = 6 };
enum class RESULT { SUCCESS = 0, MATH_ERROR = 1, IO_ERROR = 2, INFINITE_GEO = 3, INTERSECTION = 4 };
enum class SSAA_DISTR { NONE = 0, REGULAR = 1, RANDOM = 2, POISSON = 3, JITTERED = 4, ROTATED = 5 };

struct BlackHole {
    float M, rs, a, q, p[16];
};

// The sky: a texture on the sphere r = rout.
struct OutSphere {
    tex2d tex;
    float rout;

    // RMS of the 2x2 texel block at the direction (theta, phi), with the
    // reference's guards (main/base.h:119-162)
    __device__ f3 cell_rms(float theta, float phi)
    {
        if (phi > 2.0f * PI || phi < 0.0f) return f3(0.5f, 0.5f, 0.0f);
        if (theta < 0.0f || theta > PI) return f3(0.0f, 0.5f, 0.8f);
        f2 uv = f2(phi / (2.0f * PI) * tex.res.x, theta / PI * tex.res.y);
        i2 pi = floor(uv);
        if (pi.x == tex.res.x) pi.x -= 1;
        if (pi.y == tex.res.y) pi.y -= 1;
        if (pi.x < 0 || pi.x >= tex.res.x || pi.y < 0 || pi.y >= tex.res.y) return f3(0.0f, 0.5f, 0.0f);
        if (pi.x == tex.res.x - 1 || pi.y == tex.res.y - 1) return tex[pi];
        return sqavg(tex[pi], tex[pi + i2(0, 1)], tex[pi + i2(1, 0)], tex[pi + i2(1, 1)]);
    }

    // background at the POSITION p (main/base.h:68-117); with SPHERICAL, p
    // is (r, theta, phi, t) and the sky is mirrored in phi (base.h:76-83)
    __device__ f3 getColorDefault(f4 p)
    {
        if (!tex.dt.p) return f3(0.0f, 0.0f, 0.0f);
#ifdef SPHERICAL
        float theta = p.y, phi = p.z;
        phi = -phi;
        phi += 2.0f * PI;  // in double, as the reference's PI is a double literal
        if (phi == 2.0f * PI) phi = 0;
        if (theta == PI) theta = 0;
#else
        float theta = acosf(p.z / p.xyz().norm()), phi = atan2f(p.y, p.x);
        phi = (phi >= 0 ? phi : phi + 2.0f * PI);
#endif
        return cell_rms(theta, phi);
    }

    // background in the DIRECTION u (main/base.h:119-162); the library's
    // own lookup, which reproduces the reference's arithmetic.  With
    // SPHERICAL the reference has no direction lookup and returns green
    // (base.h:121-124; its diagnostic printf is not repeated here).
    __device__ f3 getColorDefault2(f4 u)
    {
#ifdef SPHERICAL
        return f3(0.0f, 1.0f, 0.0f);
#endif
        if (!tex.dt.p) return f3(0.0f, 0.0f, 0.0f);
        prr::V3<float> c = prr::background_rms<float>(tex.dt, u.x, u.y, u.z);
        return f3(c.x, c.y, c.z);
    }
};

struct Tracer {
    float h, hmin, hmax, eps;
    OutSphere sph1, sph2;
    SOLVER solver;
};

// 48 bytes, the reference's layout (main/base.h:172-176)
struct Ray {
    f2 uv;
    RESULT result;
    f4 r, u;
    float I = 0.0f;
};

typedef Ray ray;
typedef Tracer tracer;
