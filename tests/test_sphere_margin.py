"""The FP32 renderer's per-ray sphere margins (parrelray_b200/csrc/k_ham.cu, ham_accept), restated in numpy
and checked as a property: a point that the exact per-sphere far test would call near is never skipped.

The rule restated: each ray keeps `safe`, the distance from the last tested point to the nearest sphere's
far radius less 1e-3; every accepted step takes the L1 length of its position increment off it; when any
lane of a warp has `safe <= 0`, every active lane of that warp tests all spheres and resets its margin.
The exact far test (scene/sphere.h:34-50 bounded by the window hmax) is |p - c|^2 > far2.

Pure host logic: no GPU, no oracle.
"""
import numpy as np


def far_radius2(radius, hmax=0.1):
    reach = 0.5 * (np.sqrt(hmax) + radius)
    return (reach * reach + radius * radius) * 1.01 + 1e-3


def simulate(rng, lanes=32, steps=3000, nspheres=8):
    centres = rng.uniform(-12, 12, (nspheres, 3)).astype(np.float32)
    radii = rng.uniform(0.3, 1.6, nspheres)
    far2 = far_radius2(radii).astype(np.float32)
    far = np.sqrt(far2.astype(np.float64)).astype(np.float32)
    pos = rng.uniform(-20, 20, (lanes, 3)).astype(np.float32)
    safe = np.full(lanes, -1.0, np.float32)
    skipped_near = tested = 0
    for _ in range(steps):
        active = rng.random(lanes) < 0.9  # lanes that reach the accept step this attempt
        h = np.where(rng.random(lanes) < 0.7, 0.1, 10.0 ** rng.uniform(-4, -1, lanes))
        inc = (rng.normal(size=(lanes, 3)) * h[:, None] * rng.uniform(0.3, 1.5, (lanes, 1))).astype(np.float32)
        new = pos + inc
        cand = safe - np.abs(inc).sum(axis=1).astype(np.float32)
        d2 = ((new[:, None, :] - centres[None, :, :]) ** 2).sum(axis=2)
        exact_near = (d2 <= far2[None, :]).any(axis=1)
        vote = bool(np.any(active & ~(cand > 0)))  # one vote over the active lanes
        check = active & vote
        if vote:
            dist = np.sqrt(np.maximum(d2, 1e-30)) - far[None, :]
            cand = np.where(active, dist.min(axis=1).astype(np.float32) - np.float32(1e-3), cand)
            tested += int(active.sum())
        skipped_near += int(np.sum(active & ~check & exact_near))
        pos = np.where(active[:, None], new, pos)
        safe = np.where(active, cand, safe)
    return skipped_near, tested


def test_margin_never_skips_a_near_point():
    rng = np.random.default_rng(7)
    for _ in range(4):
        skipped_near, tested = simulate(rng)
        assert skipped_near == 0
        assert tested > 0


def test_margin_skips_most_tests_far_from_the_spheres():
    """Rays far from every sphere test rarely: with no sphere within reach a lane tests once and then runs
    on its margin."""
    rng = np.random.default_rng(11)
    lanes, steps = 32, 400
    centre = np.array([[0.0, 0.0, 0.0]], np.float32)
    far = np.float32(np.sqrt(far_radius2(np.array([1.0]))[0]))
    pos = rng.uniform(40, 60, (lanes, 3)).astype(np.float32)
    safe = np.full(lanes, -1.0, np.float32)
    checks = 0
    for _ in range(steps):
        inc = (rng.normal(size=(lanes, 3)) * 0.05).astype(np.float32)
        cand = safe - np.abs(inc).sum(axis=1)
        if np.any(~(cand > 0)):
            checks += 1
            cand = (np.linalg.norm(pos + inc - centre, axis=1) - far - 1e-3).astype(np.float32)
        pos = pos + inc
        safe = cand
    assert checks <= 3, checks
