#pragma once
// Compatibility texture for ParRelRay metric plug-in headers: the reference's
// tex2d (cudamaths/tex2d.cuh) as seen from device code - a resolution `res`
// and indexing by texel (operator[](i2), clamped to [0, res-1]), by linear
// index (operator[](int)) and by normalised coordinates (operator[](f2),
// bilinear with the cell clamped to [0, res-2] after the fraction is taken,
// the reference's edge behaviour).  Texels are the library's RGBA8 uploads
// read as byte/255, the value the reference's stbi_loadf(gamma 1) gives.
// Loading, saving and device allocation belong to the host library
// (prr_upload_texture), so those members are absent.
#include "vecs.h"
#include "prr_device.cuh"

class tex2d {
public:
    i2 res;
    prr::DevTex dt;
    PRR_VHD tex2d() : res(0, 0), dt{nullptr, 0, 0} {}
    PRR_VHD tex2d(const prr::DevTex &t) : res(t.w, t.h), dt(t) {}
    __device__ inline f3 operator[](f2 uv) const
    {
        prr::V3<float> c = prr::tex_bilinear<float>(dt, uv.x, uv.y);
        return f3(c.x, c.y, c.z);
    }
    __device__ inline f3 operator[](i2 ij) const
    {
        prr::V3<float> c = prr::tex_at<float>(dt, ij.x, ij.y);
        return f3(c.x, c.y, c.z);
    }
    __device__ inline f3 operator[](int i) const
    {
        prr::V3<float> c = prr::texel<float>(dt, i % dt.w, i / dt.w);
        return f3(c.x, c.y, c.z);
    }
    PRR_VHD size_t getSize() { return (size_t)res.x * res.y * sizeof(f3); }
};
