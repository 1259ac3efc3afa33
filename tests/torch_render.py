"""A thin torch.autograd.Function over the C ABI, used only by tests and the
bench's fit demo: forward = FP64 render of an orbit-camera Kerr frame
(prr_render), backward = prr_adjoint.

Parameters (a 5-vector, float64): spin a, mass M, camera inclination i
[radians], camera distance r, orbital phase of sphere 0 [radians].
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from parrelray_b200 import abi, scenes


def frame_from_params(p, width, height, sphere_orbit=9.0, sphere_radius=1.0, fov_deg=40.0, tol=1e-6, samples=1):
    spin, mass, incl, cam_r, phase = [float(v) for v in p]
    return scenes.make_frame(width, height, r=cam_r, incl_deg=math.degrees(incl), fov_deg=fov_deg,
                             metric=abi.METRIC_KERR, mass=mass, spin=spin, samples=samples,
                             spheres=[(*scenes.orbit_point(sphere_orbit, math.degrees(phase)), sphere_radius,
                                       scenes.SPHERE_ID0)],
                             bg_filter=abi.BG_BILINEAR, precision=abi.PREC_FP64, tol=tol)


class KerrRender(torch.autograd.Function):
    @staticmethod
    def forward(ctx, params, gpu, width, height, opts):
        d = frame_from_params(params.detach().cpu().numpy(), width, height, **opts)
        _, imgs, _ = gpu.render(d, want_float=True)
        ctx.gpu, ctx.frame = gpu, d
        return torch.from_numpy(np.ascontiguousarray(imgs[0])).to(params.dtype)

    @staticmethod
    def backward(ctx, grad_out):
        g = np.zeros(5, dtype=np.float64)
        dl = np.ascontiguousarray(grad_out.detach().cpu().numpy(), dtype=np.float32)
        st = abi.Stats()
        abi.check(abi.load().prr_adjoint(ctx.gpu.h, C.byref(ctx.frame), dl.ctypes.data_as(abi._fp), 0,
                                         g.ctypes.data_as(abi._dp), C.byref(st)), ctx.gpu.h)
        ctx.gpu.last_adjoint_stats = st
        return torch.from_numpy(g), None, None, None, None


def render(params, gpu, width, height, **opts):
    return KerrRender.apply(params, gpu, width, height, opts)
