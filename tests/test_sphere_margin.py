"""The FP32 renderer's per-ray sphere margins (parrelray_b200/csrc/k_ham.cu, ham_accept), restated in numpy
and checked as a property: a point that the exact per-sphere far test would call near is never skipped.

The rule restated: each ray keeps `safe`, the distance from the last tested point to the nearest sphere's
far radius less 1e-3; every accepted step takes the L1 length of its position increment off it, the length
summed rounding up and subtracted rounding down in FP32; when any lane of a warp has `safe <= 0`, every
active lane of that warp tests all spheres and resets its margin.
The exact far test (scene/sphere.h:34-50 bounded by the window hmax) is |p - c|^2 > far2.

Pure host logic: no GPU, no oracle.
"""
import numpy as np


def f32_up(x):
    """FP32 value of x rounded toward +inf (an FP32 add with .ru of the exact sum held in FP64)."""
    y = np.float32(x)
    return np.where(y.astype(np.float64) < x, np.nextafter(y, np.float32(np.inf)), y).astype(np.float32)


def f32_down(x):
    y = np.float32(x)
    return np.where(y.astype(np.float64) > x, np.nextafter(y, np.float32(-np.inf)), y).astype(np.float32)


def decrement(safe, inc, directed=True):
    """safe - (|dx| + |dy| + |dz|) as the kernel forms it: __fadd_ru twice, then __fsub_rd."""
    a = np.abs(inc.astype(np.float64))
    if not directed:  # round to nearest at every operation
        l1 = (np.abs(inc[..., 0]) + np.abs(inc[..., 1])) + np.abs(inc[..., 2])
        return (safe - l1).astype(np.float32)
    l1 = f32_up(f32_up(a[..., 0] + a[..., 1]).astype(np.float64) + a[..., 2])
    return f32_down(safe.astype(np.float64) - l1.astype(np.float64))


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
        cand = decrement(safe, inc)
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
        cand = decrement(safe, inc)
        if np.any(~(cand > 0)):
            checks += 1
            cand = (np.linalg.norm(pos + inc - centre, axis=1) - far - 1e-3).astype(np.float32)
        pos = pos + inc
        safe = cand
    assert checks <= 3, checks


def test_margin_stays_below_the_distance_over_many_small_steps():
    """A margin near 100 (FP32 ulp 7.6e-6) taking 1e-4-long steps: rounded to nearest, each subtraction can
    drop the same fraction of an ulp, and over 20,000 steps the margin drifts above the true remaining
    distance; with the length rounded up and the subtraction rounded down it never does."""
    steps = 20000
    inc = np.tile(np.array([[1.0e-4, 0.0, 0.0]], np.float32), (steps, 1))
    for directed, drifts in ((True, False), (False, True)):
        safe = np.array([100.0], np.float32)
        travelled = 0.0
        worst = -np.inf
        for k in range(steps):
            safe = decrement(safe, inc[k:k + 1], directed)
            travelled += float(np.float32(1.0e-4))
            worst = max(worst, float(safe[0]) - (100.0 - travelled))
        assert (worst > 0.0) == drifts, (directed, worst)
