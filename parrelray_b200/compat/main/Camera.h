#pragma once
// Compatibility Camera for ParRelRay metric plug-in headers: the members and
// methods of the reference's Camera (main/Camera.h:17-52, main/Camera.cpp)
// that device code reaches - resolution, SSAA settings, pose (pos, a, b) and
// the three ray-direction models.  The plug-in kernels build one per frame
// from the frame descriptor.
#include "base.h"

class Camera {
public:
    PRR_VHD Camera() : AAsamples(1), ssaa(SSAA_DISTR::NONE), vfov(1.0471975512f) {}
    PRR_VHD Camera(float vertFov, i2 resolution, SSAA_DISTR distr, int samples)
        : vfov(vertFov), res(resolution), ssaa(distr), AAsamples(samples) {}
    PRR_VHD Camera(f3 position, float alpha, float beta, float vertFov, i2 resolution, SSAA_DISTR distr, int samples)
        : a(alpha), b(beta), pos(position), vfov(vertFov), res(resolution), ssaa(distr), AAsamples(samples) {}
    PRR_VHD i2 getRes() { return res; }
    PRR_VHD int getAAsamples() { return AAsamples; }
    PRR_VHD SSAA_DISTR getSSAADistr() { return ssaa; }
    PRR_VHD float getVfov() { return vfov; }

    // forward/up/right from the yaw a and pitch b (main/Camera.cpp:19-28)
    PRR_VHD void computeVectors()
    {
        forward = normalize(f3(cosf(b) * cosf(a), cosf(b) * sinf(a), -sinf(b)));
        up = normalize(f3(cosf(a) * sinf(b), sinf(a) * sinf(b), cosf(b)));
        right = normalize(cross(forward, up));
    }
    __device__ inline f3 rayDir_PinHole(f2 uv)
    {
        return normalize(forward + (2.0f * uv.x - 1) * tanf(vfov / 2.0f) * res.x / res.y * right +
                         (1.0f - 2.0f * uv.y) * tanf(vfov / 2.0f) * up);
    }
    __device__ inline f3 rayDir_Panorama(f2 uv)
    {
        float mu = (0.5f - uv.y) * vfov;
        float nu = (0.5f - uv.x) * res.x / res.y * vfov;
        return normalize(cosf(mu) * cosf(nu) * forward + cosf(mu) * sinf(nu) * right + sinf(mu) * mu * up);
    }
    // the model the reference's initRays uses (kernels/solver.cuh:40)
    __device__ inline f3 rayDir_Spherical(f2 uv)
    {
        float nu = (0.5f - uv.y) * vfov;
        float mu = (0.5f - uv.x) * res.x / res.y * vfov;
        return normalize(f3(cosf(b + nu) * cosf(a + mu), cosf(b + nu) * sinf(a + mu), sinf(b + nu)));
    }

    float a = 0.0f, b = 0.0f;
    f3 pos, spos;

private:
    f3 forward, right, up;
    float vfov = 1.0471975512f;
    i2 res;
    SSAA_DISTR ssaa;
    int AAsamples;
};
