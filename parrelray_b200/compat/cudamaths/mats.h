#pragma once
// Compatibility 4x4 matrix for ParRelRay metric plug-in headers: the class
// name, storage (e[16], row-major, index order x, y, z, t) and members of the
// reference's mat4 (cudamaths/mat4.cuh, included through cudamaths/mats.h),
// which getMetric() implementations fill (metrics/schwarzschild.cuh:123-141).
#include "vecs.h"

class mat4 {
public:
    float e[16];
    PRR_VHD mat4() { for (int i = 0; i < 16; i++) e[i] = 0.0f; }
    PRR_VHD float operator[](int i) const { return e[i]; }
    PRR_VHD float &operator[](int i) { return e[i]; }
    PRR_VHD const mat4 &operator+() const { return *this; }
    PRR_VHD mat4 operator-() const { mat4 m; for (int i = 0; i < 16; i++) m.e[i] = -e[i]; return m; }
    // copies entries 1, 2, 6, 3, 7 and (as the reference does) 8 into the
    // lower triangle (cudamaths/mat4.cuh:27-29)
    PRR_VHD void sym() { e[4] = e[1]; e[8] = e[2]; e[9] = e[6]; e[12] = e[3]; e[13] = e[7]; e[14] = e[8]; }
    PRR_VHD void cinv() { for (int i = 0; i < 16; i++) e[i] = 1.0f / e[i]; }
    PRR_VHD float x() const { return e[0]; }
    PRR_VHD float m(int i, int j) { return e[i * 4 + j]; }
};

PRR_VHD float dot(const mat4 &a, const mat4 &b)
{
    float s = 0.0f;
    for (int i = 0; i < 16; i++) s += a[i] * b[i];
    return s;
}
PRR_VHD mat4 mat4_id() { mat4 m; m[0] = 1; m[5] = 1; m[10] = 1; m[15] = 1; return m; }
PRR_VHD mat4 mat4_full(float k) { mat4 m; for (int i = 0; i < 16; i++) m[i] = k; return m; }
PRR_VHD mat4 mat4_comb(const f4 &v)
{
    mat4 m;
    const float c[4] = {v.x, v.y, v.z, v.w};
    for (int i = 0; i < 4; i++)
        for (int j = i; j < 4; j++) m[4 * i + j] = c[i] * c[j];
    m.sym();
    return m;
}
