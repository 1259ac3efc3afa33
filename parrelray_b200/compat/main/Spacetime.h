#pragma once
// Compatibility Spacetime for ParRelRay metric plug-in headers: the black-hole
// getters and the scene query of the reference's Spacetime
// (main/Spacetime.h:16-53).  IntersectsScene runs the library's sphere test,
// which reproduces Sphere::intersects / Sphere::getColor (scene/sphere.h:34-64)
// and the closest-hit rule of Spacetime.h:38-46, on the frame's spheres.
#include "base.h"

class Spacetime {
public:
    PRR_VHD Spacetime() : fp(nullptr), hasBlackhole(true) { bh.M = bh.rs = bh.a = bh.q = 0.0f; for (int i = 0; i < 16; i++) bh.p[i] = 0.0f; }
    PRR_VHD BlackHole &getBlackHole() { return bh; }
    PRR_VHD bool hasBh() { return hasBlackhole; }
    PRR_VHD void setHasBh(bool) { hasBlackhole = true; }
    PRR_VHD float getBhMass() { return bh.M; }
    PRR_VHD float getBhRs() { return bh.rs; }
    PRR_VHD void setBhMass(float mass) { bh.M = mass; bh.rs = 2.0f * mass; }
    PRR_VHD float getBhSpin() { return bh.a; }
    PRR_VHD void setBhSpin(float spin) { bh.a = spin; }
    PRR_VHD float getBhCharge() { return bh.q; }
    PRR_VHD void setBhCharge(float charge) { bh.q = charge; }
    PRR_VHD float getBhP(int i) { return i >= 16 ? 0.0f : bh.p[i]; }
    PRR_VHD void setBhP(int i, float p) { if (i < 16) bh.p[i] = p; }

    // colour of the closest sphere hit within the step window h, else (-1, -1, -1)
    __device__ f3 IntersectsScene(f3 p, f3 u, float h)
    {
        if (!fp) return f3(-1.0f, -1.0f, -1.0f);
        prr::Hit c = prr::intersect_scene<float>(*fp, p.x, p.y, p.z, u.x, u.y, u.z, h);
        return f3(c.r, c.g, c.b);
    }

    const prr::FrameParams *fp;  // the frame (device memory): its spheres

private:
    BlackHole bh;
    bool hasBlackhole;
};
