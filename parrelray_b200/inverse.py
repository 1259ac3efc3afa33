"""The inverse problem on top of prr_adjoint: fit frame parameters (spin,
mass, camera inclination and distance, sphere phase) to a target image by
Adam on an L2 loss, every gradient from the discrete adjoint.

The adjoint freezes each ray's discrete events (accept/reject sequence,
termination, which surface is hit), so it is the derivative of the image with
those events held fixed.  Two kinds of pixel break that premise:

* pixels on the shadow's silhouette, whose ray switches between sky and
  horizon within a small change of the parameters (a jump the frozen
  derivative cannot see);
* pixels just outside it, whose ray winds near the photon orbit: their escape
  direction, and so their derivative, grows without bound towards the edge,
  and one such pixel can outweigh the rest of the image.

`sky_weights` therefore restricts the loss to pixels that show sky in both
the current and the target image and lie at least `margin` pixels (Chebyshev
distance) from a black pixel of either.  Captured and unfinished rays are
black (0, 0, 0) in every render; sky texels are assumed never to be black,
which holds for any sky whose darkest texel has a non-zero channel.  Sphere
silhouettes are not detected (a sphere is not black).
"""
from __future__ import annotations

import time
from typing import Callable, Sequence

import numpy as np

from .abi import FrameDesc


def sky_weights(image: np.ndarray, target: np.ndarray, margin: int = 2) -> np.ndarray:
    """(h, w) float32 weights in {0, 1}: 1 where both (h, w, 3) images show
    sky and no pixel within `margin` of it is black in either (pixels beyond
    the image border count as sky)."""
    if image.shape != target.shape or image.ndim != 3:
        raise ValueError("image and target must be (h, w, 3) arrays of the same shape")
    if margin < 0:
        raise ValueError("margin must be >= 0")
    sky = (np.asarray(image).max(axis=2) > 0) & (np.asarray(target).max(axis=2) > 0)
    h, w = sky.shape
    pad = np.ones((h + 2 * margin, w + 2 * margin), dtype=bool)
    pad[margin:margin + h, margin:margin + w] = sky
    out = np.ones_like(sky)
    for dy in range(2 * margin + 1):
        for dx in range(2 * margin + 1):
            out &= pad[dy:dy + h, dx:dx + w]
    return out.astype(np.float32)


class Adam:
    """Adam (Kingma and Ba, 2015) with bias correction and a step size
    lr * decay^(t-1) at step t; `lo`/`hi` clip the parameters after each step."""

    def __init__(self, q0: Sequence[float], lr: float, decay: float = 1.0, b1: float = 0.9, b2: float = 0.999,
                 eps: float = 1e-8, lo: Sequence[float] | None = None, hi: Sequence[float] | None = None):
        self.q = np.array(q0, dtype=np.float64)
        self.m = np.zeros_like(self.q)
        self.v = np.zeros_like(self.q)
        self.t = 0
        self.lr, self.decay, self.b1, self.b2, self.eps = lr, decay, b1, b2, eps
        self.lo = None if lo is None else np.array(lo, dtype=np.float64)
        self.hi = None if hi is None else np.array(hi, dtype=np.float64)

    def step(self, grad: Sequence[float]) -> np.ndarray:
        g = np.asarray(grad, dtype=np.float64)
        self.t += 1
        self.m = self.b1 * self.m + (1 - self.b1) * g
        self.v = self.b2 * self.v + (1 - self.b2) * g * g
        mh = self.m / (1 - self.b1 ** self.t)
        vh = self.v / (1 - self.b2 ** self.t)
        self.q = self.q - self.lr * self.decay ** (self.t - 1) * mh / (np.sqrt(vh) + self.eps)
        if self.lo is not None:
            self.q = np.maximum(self.q, self.lo)
        if self.hi is not None:
            self.q = np.minimum(self.q, self.hi)
        return self.q


def fit(ctx, frame_at: Callable[[np.ndarray], FrameDesc], target: np.ndarray, q0: Sequence[float],
        grad_index: Sequence[int], iters: int, lr: float = 0.01, decay: float = 0.99, margin: int | None = 2,
        sphere_index: int = -1, lo: Sequence[float] | None = None, hi: Sequence[float] | None = None) -> dict:
    """Adam on the parameters q (frame_at(q) builds the frame; grad_index
    picks each parameter's entry of prr_adjoint's gradient, e.g. (0, 2) for
    spin and inclination) minimising sum(weights * (image - target)^2) with
    weights = sky_weights(image, target, margin), recomputed from each
    iteration's render (margin None: every pixel).  Returns the history:
    full and weighted losses, the weighted pixel fraction, the parameters and
    the device time of each iteration."""
    tgt = np.asarray(target, dtype=np.float64)
    opt = Adam(q0, lr, decay, lo=lo, hi=hi)
    out = {"loss": [], "weighted_loss": [], "weighted_fraction": [], "q": [], "device_ms": []}
    t0 = time.perf_counter()
    for _ in range(iters):
        q = opt.q.copy()
        d = frame_at(q)
        _, cur, rs = ctx.render(d, want_float=True)
        img = cur[0].astype(np.float64)
        w = np.ones(img.shape[:2], np.float32) if margin is None else sky_weights(img, tgt, margin)
        diff = img - tgt
        out["loss"].append(float(np.sum(diff * diff)))
        out["weighted_loss"].append(float(np.sum(w[:, :, None] * diff * diff)))
        out["weighted_fraction"].append(float(w.mean()))
        out["q"].append(q)
        g, st = ctx.adjoint(d, 2.0 * w[:, :, None] * diff, sphere_index)
        out["device_ms"].append(rs.kernel_ms + st.kernel_ms + st.trace_ms)
        opt.step([g[k] for k in grad_index])
    out["q_final"] = opt.q.copy()
    out["wall_s"] = time.perf_counter() - t0
    return out
