"""The metric plug-in build (no GPU needed): a header in the reference's
plug-in shape - here one written by this test, a flat spacetime with a custom
horizon-free ENDLOOP - compiles UNCHANGED against the compatibility tree
(parrelray_b200/compat) into a library with the prr_plugin_* entry points the
loader checks; the libraries built from the shipped Kerr header and (where
the reference tree is mounted) the reference's own headers exist."""
import ctypes as C
from pathlib import Path

import pytest

from parrelray_b200 import abi, build

USER_HEADER = r"""
#pragma once
#include "../main/base.h"
#include "../main/Camera.h"
#include "../main/Spacetime.h"
#include "../cudamaths/mats.h"

__host__ void User_INIT(ray *rays, Camera *cam, Spacetime *space) {}
__device__ bool User_LOOP(ray *iray, Camera cam, Spacetime space) { return true; }
__device__ bool User_UPDATE(ray *iray, Camera cam, Spacetime space, float h)
{
    f3 c = space.IntersectsScene(iray->r.xyz(), iray->u.xyz(), h);
    if (c.x >= 0.0f) { iray->result = RESULT::INTERSECTION; return false; }
    return true;
}
__device__ bool User_ENDLOOP(ray *iray, Camera cam, Spacetime space, tracer trace)
{
    if (iray->r.xyz().norm() >= trace.sph1.rout) { iray->result = RESULT::SUCCESS; return false; }
    f3 c = space.IntersectsScene(iray->r.xyz(), iray->u.xyz(), trace.h);
    if (c.x >= 0.0f) { iray->u = f4(c, 0.0f); iray->result = RESULT::INTERSECTION; return false; }
    return true;
}
__device__ f4 getGeod(f4 p, f4 u, Spacetime space) { return f4(); }
__device__ mat4 getMetric(ray *R, Spacetime space) { mat4 g = mat4_id(); g[15] = -1; return g; }
__global__ void rayToRGB(ray *rays, Camera cam, Spacetime space, tracer trace, int samples)
{
    i2 ij = i2(blockIdx.x * blockDim.x + threadIdx.x, blockIdx.y * blockDim.y + threadIdx.y);
    if ((ij.x >= cam.getRes().x * samples) || (ij.y >= cam.getRes().y)) return;
    int pid = ij.y * cam.getRes().x * samples + ij.x;
    if (rays[pid].result == RESULT::SUCCESS) rays[pid].u = f4(trace.sph1.getColorDefault2(rays[pid].u), 0.0f);
    else if (rays[pid].result != RESULT::INTERSECTION) rays[pid].u = f4(0.0f);
}
"""


def _exports(path: Path):
    lib = C.CDLL(str(path))
    lib.prr_plugin_name.restype = C.c_char_p
    lib.prr_plugin_ray_bytes.restype = C.c_size_t
    lib.prr_plugin_frame_params_size.restype = C.c_size_t
    return lib


def test_user_header_builds_unchanged(built, tmp_path):
    h = tmp_path / "myflat.cuh"
    h.write_text(USER_HEADER)
    out = build.build_metric_plugin(h, "testflat", lib_dir=tmp_path / "lib")
    lib = _exports(out)
    assert lib.prr_plugin_name() == b"testflat"
    assert lib.prr_plugin_ray_bytes() == 48  # the reference's Ray layout (main/base.h:172-176)
    assert lib.prr_plugin_abi_version() == abi.load().prr_abi_version()  # plug-ins embed the frame layout
    # the REFERENCE unit (-fmad=false) and the PHYSICAL unit (contraction on) both export their entry points
    for sym in ("prr_plugin_trace", "prr_plugin_trace_physical", "prr_plugin_colour"):
        assert hasattr(lib, sym), sym
    assert h.read_text() == USER_HEADER  # the header itself is not touched
    assert not (build.BUILD / "plugins" / "testflat").exists()  # staging copy removed


def test_shipped_plugins_are_built(built):
    outs = build.build_plugins()
    names = {p.name for p in outs}
    assert "libprr_metric_kerr.so" in names
    for p in outs:
        assert _exports(p).prr_plugin_frame_params_size() > 0
    if build.reference_tree() is not None:
        assert {"libprr_metric_schwarzschild.so", "libprr_metric_flat.so", "libprr_metric_schwarzschildcart.so",
                "libprr_metric_schwarzschildsph.so"} <= names


SPHERICAL_HEADER = r"""
#pragma once
#include "../main/base.h"
#include "../main/Camera.h"
#include "../main/Spacetime.h"
#include "../cudamaths/mats.h"

__device__ bool User_LOOP(ray *iray, Camera cam, Spacetime space) { return true; }
__device__ bool User_UPDATE(ray *iray, Camera cam, Spacetime space, float h) { return true; }
__device__ bool User_ENDLOOP(ray *iray, Camera cam, Spacetime space, tracer trace)
{
    if (iray->r.x >= trace.sph1.rout) { iray->result = RESULT::SUCCESS; return false; }
    return true;
}
__device__ f4 getGeod(f4 p, f4 u, Spacetime space)
{
    // flat space in (r, theta, phi, t)
    float r = p.x, st = sinf(p.y), ct = cosf(p.y);
    return f4(r * (u.y * u.y + st * st * u.z * u.z), -2.0f / r * u.x * u.y + st * ct * u.z * u.z,
              -2.0f / r * u.x * u.z - 2.0f * ct / st * u.y * u.z, 0.0f);
}
__device__ mat4 getMetric(ray *R, Spacetime space)
{
    mat4 g; float r = R->r.x, st = sinf(R->r.y);
    g[0] = 1.0f; g[5] = r * r; g[10] = r * r * st * st; g[15] = -1.0f;
    return g;
}
__global__ void rayToRGB(ray *rays, Camera cam, Spacetime space, tracer trace, int samples)
{
    i2 ij = i2(blockIdx.x * blockDim.x + threadIdx.x, blockIdx.y * blockDim.y + threadIdx.y);
    if ((ij.x >= cam.getRes().x * samples) || (ij.y >= cam.getRes().y)) return;
    int pid = ij.y * cam.getRes().x * samples + ij.x;
    f3 back = pos_spherTOcart(pos_cartTOspher(f3(1.0f, 2.0f, 3.0f)));  // the conversions are there
    rays[pid].u = f4(trace.sph1.getColorDefault(rays[pid].r) + 0.0f * back, 0.0f);
}
"""


def test_spherical_header_builds_with_the_switch(built, tmp_path):
    """A header written for the reference's SPHERICAL build (states (r, theta, phi, t); the sky looked
    up at the final angles; the Cartesian <-> spherical conversions of cudamaths/transform.cuh) builds
    unchanged with spherical=True."""
    h = tmp_path / "flatsph.cuh"
    h.write_text(SPHERICAL_HEADER)
    out = build.build_metric_plugin(h, "testflatsph", lib_dir=tmp_path / "lib", spherical=True)
    lib = _exports(out)
    assert lib.prr_plugin_name() == b"testflatsph"
    assert lib.prr_plugin_ray_bytes() == 48
