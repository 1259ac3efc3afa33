#pragma once
// Compatibility Cartesian <-> spherical conversions for ParRelRay metric
// plug-in headers (the functions of the reference's cudamaths/transform.cuh,
// which its cudamaths/vecs.h includes).  Spherical triples are (r, theta,
// phi) with theta from +z and phi = atan2(y, x); velocities are the
// coordinate rates (dr, dtheta, dphi) of a Cartesian velocity at a point.
// The reference's solver uses them when SPHERICAL is defined
// (kernels/solver.cuh:34-37, prr.cpp:250-252).
#include "vecs.h"

PRR_VHD f3 pos_cartTOspher(f3 p)
{
    const float r = p.norm();
    return f3(r, acosf(p.z / r), atan2f(p.y, p.x));
}

PRR_VHD f3 pos_spherTOcart(f3 s)
{
    return f3(s.x * cosf(s.z) * sinf(s.y), s.x * sinf(s.z) * sinf(s.y), s.x * cosf(s.y));
}

// (dr, dtheta, dphi) of the Cartesian velocity v at p:
//   dr = p.v / r,  dtheta = (z (x vx + y vy) - rho^2 vz) / (r^2 rho),
//   dphi = (vx y - x vy) / rho^2,  rho^2 = x^2 + y^2
// (the sign of dphi is the reference's, transform.cuh:25-31)
PRR_VHD f3 vel_cartTOspher(f3 p, f3 v)
{
    const float rho2 = p.xy().norm2();
    const float r2 = rho2 + p.z * p.z;
    f3 s;
    s.x = dot(p, v) / sqrtf(r2);
    s.y = (p.z * (p.x * v.x + p.y * v.y) - rho2 * v.z) / (r2 * sqrtf(rho2));
    s.z = (v.x * p.y - p.x * v.y) / rho2;
    return s;
}
