import contextlib
import os
import sys
from pathlib import Path

import numpy as np
import pytest

REPO = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(REPO))
sys.path.insert(0, str(Path(__file__).resolve().parent))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")
    config.addinivalue_line("markers", "slow: takes more than a few seconds on CPU")


@pytest.fixture(scope="session")
def built():
    """Builds the library and the CPU oracle if needed (cheap when up to date)."""
    from parrelray_b200 import build

    build.build_library()
    build.build_plugins()
    build.build_oracle()
    build.build_reference()
    return True


@pytest.fixture(scope="session")
def oracle(built):
    from oracles import Oracle

    return Oracle()


@pytest.fixture(scope="session")
def small_textures(built):
    """Small seeded textures (fast oracle runs): sky 256x128, three 128x64 sphere textures."""
    from parrelray_b200 import scenes

    tex = {scenes.SKY_ID: scenes.make_texture(1, 1234, 256, 128)}
    for k in range(3):
        tex[scenes.SPHERE_ID0 + k] = scenes.make_texture(0, 100 + k, 128, 64)
    return tex


@pytest.fixture(scope="session")
def std_textures(built):
    from parrelray_b200 import scenes

    return scenes.standard_textures()


@pytest.fixture(scope="session")
def gpu(built):
    """A device context.  Fails (does not skip) when no device is usable:
    GPU tests must never pass on a fallback."""
    from parrelray_b200 import Context

    ctx = Context(0)
    yield ctx
    ctx.close()


@contextlib.contextmanager
def hamiltonian_forms(ctx, mask: int):
    """Sets PRR_OPT_HAMILTONIAN on a (session-wide) context for a block and
    restores the default (both precisions in Hamiltonian form) after it."""
    from parrelray_b200 import abi

    ctx.set_option(abi.OPT_HAMILTONIAN, mask)
    try:
        yield ctx
    finally:
        ctx.set_option(abi.OPT_HAMILTONIAN, abi.HAM_FP32 | abi.HAM_FP64)


def pixel_rule(a8: np.ndarray, b8: np.ndarray) -> float:
    """Fraction of pixels whose RGB differ by at most 1/255 in every channel."""
    d = np.abs(a8.astype(np.int32) - b8.astype(np.int32)).max(axis=-1)
    return float(np.mean(d <= 1))


def quantize(img: np.ndarray) -> np.ndarray:
    """roundf(255.0f*x) of cudamaths/image.cu:31 on a clamped float image
    (FP32 product, halves rounded away from zero)."""
    v = np.float32(255.0) * np.clip(img.astype(np.float32), np.float32(0.0), np.float32(1.0))
    return np.floor(v.astype(np.float64) + 0.5).astype(np.uint8)
