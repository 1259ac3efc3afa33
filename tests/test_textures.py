"""Seeded procedural textures: deterministic bytes and the statistics the
workloads assume (point-star density, log-normal brightness, opaque alpha)."""
import hashlib

import numpy as np

from parrelray_b200 import scenes


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def test_deterministic(built):
    a = scenes.make_texture(1, 7, 512, 256)
    b = scenes.make_texture(1, 7, 512, 256)
    c = scenes.make_texture(1, 8, 512, 256)
    assert digest(a) == digest(b)
    assert digest(a) != digest(c)
    s = scenes.make_texture(0, 3, 128, 64)
    assert digest(s) == digest(scenes.make_texture(0, 3, 128, 64))


def test_golden_texture_digest_is_stable(built):
    """The golden fixtures were produced from these exact bytes."""
    import json

    from pathlib import Path

    meta = json.loads(str(np.load(Path(__file__).parent / "golden" / "schw_160x90_s1.npz")["meta"]))
    from golden.make_golden import texture_digest, textures

    assert texture_digest(textures()) == meta["texture_sha256"]


def test_starfield_statistics(built):
    w, h = 2048, 1024
    sky = scenes.make_texture(1, 1234, w, h).astype(np.int32)
    assert (sky[:, :, 3] == 255).all()
    lum = sky[:, :, :3].max(axis=2)
    stars = lum > 40  # background gradient stays below 40
    dens = stars.mean()
    assert 0.0015 < dens < 0.0035, dens
    # point stars: almost no two stars are 4-neighbours
    adj = (stars[:, 1:] & stars[:, :-1]).sum() + (stars[1:, :] & stars[:-1, :]).sum()
    assert adj < 0.02 * stars.sum()
    # log-normal brightness: log of the star peak is roughly symmetric
    b = np.log(lum[stars] / 255.0)
    assert abs(np.median(b) - np.log(0.30)) < 0.25


def test_sphere_texture_has_checkerboard(built):
    t = scenes.make_texture(0, 100, 512, 256).astype(np.int32)
    cell_a = t[0:16, 0:32, :3].mean()
    cell_b = t[0:16, 32:64, :3].mean()
    assert abs(cell_a - cell_b) > 40


def test_oracle_makes_the_same_textures(oracle):
    """The CPU side of the bench makes the workload's textures with the oracle library (which
    compiles the same generator), so it never loads the product library: same bytes."""
    std = scenes.standard_textures()
    mine = oracle.standard_textures()
    assert sorted(std) == sorted(mine)
    for k in std:
        assert np.array_equal(std[k], mine[k]), k
