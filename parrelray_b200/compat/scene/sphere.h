#pragma once
// Compatibility Sphere (the shape of scene/sphere.h:19-65 of the reference):
// centre c and radius r.  Scene spheres live in the frame descriptor and are
// tested through Spacetime::IntersectsScene.
#include "../main/base.h"

struct Sphere {
    f3 c;
    float r;
    PRR_VHD Sphere() : c(), r(0.0f) {}
    PRR_VHD Sphere(f3 position, float radius) : c(position), r(radius) {}
    PRR_VHD void update(f3 position, float radius) { c = position; r = radius; }
};
