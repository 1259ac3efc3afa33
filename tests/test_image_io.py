"""Image files of the deck-driven host (prr_image_load / prr_png_write).  No
GPU needed.

The reference loads textures with stbi_loadf(path, ..., 3) under gamma 1
(cudamaths/image.cu:13-21) and writes frames with stbi_write_png after
roundf(255*x) (cudamaths/image.cu:28-39).  Decoded pixels must follow
stb_image's channel rules: grey replicated to RGB, 16-bit samples keep their
high byte, low-bit grey scaled to 0..255, palette indices looked up, alpha
dropped.  The PNG files here are written by this test's own small encoder
(zlib + the PNG chunk layout), so every colour type, bit depth and both
interlace methods are covered without an imaging library.
"""
import struct
import zlib

import numpy as np
import pytest

from parrelray_b200 import PrrError, abi, load_image, write_png

ADAM7 = [(0, 0, 8, 8), (4, 0, 8, 8), (0, 4, 4, 8), (2, 0, 4, 4), (0, 2, 2, 4), (1, 0, 2, 2), (0, 1, 1, 2)]


def _chunk(t: bytes, data: bytes) -> bytes:
    return struct.pack(">I", len(data)) + t + data + struct.pack(">I", zlib.crc32(t + data) & 0xFFFFFFFF)


def _pack_row(samples: np.ndarray, depth: int) -> bytes:
    """samples: 1-D array of integer samples of one row."""
    if depth == 8:
        return samples.astype(np.uint8).tobytes()
    if depth == 16:
        return samples.astype(">u2").tobytes()
    bits = np.unpackbits(samples.astype(np.uint8)[:, None], axis=1)[:, 8 - depth:].reshape(-1)
    return np.packbits(bits).tobytes()


def _filter(row: bytes, prev: bytes, bpp: int, ft: int) -> bytes:
    out = bytearray(len(row))
    for i, v in enumerate(row):
        a = row[i - bpp] if i >= bpp else 0
        b = prev[i] if prev else 0
        c = prev[i - bpp] if prev and i >= bpp else 0
        if ft == 0:
            p = 0
        elif ft == 1:
            p = a
        elif ft == 2:
            p = b
        elif ft == 3:
            p = (a + b) >> 1
        else:
            pa, pb, pc = abs(b - c), abs(a - c), abs(a + b - 2 * c)
            p = a if pa <= pb and pa <= pc else (b if pb <= pc else c)
        out[i] = (v - p) & 0xFF
    return bytes(out)


def encode_png(samples: np.ndarray, ctype: int, depth: int, interlace: bool = False, palette=None) -> bytes:
    """samples: (h, w, channels) integer array."""
    h, w, ch = samples.shape
    bpp = max(1, ch * depth // 8)
    passes = ADAM7 if interlace else [(0, 0, 1, 1)]
    raw = bytearray()
    ft = 0
    for x0, y0, dx, dy in passes:
        sub = samples[y0::dy, x0::dx]
        if sub.size == 0:
            continue
        prev = None
        for r in sub:
            row = _pack_row(r.reshape(-1), depth)
            raw.append(ft)
            raw += _filter(row, prev, bpp, ft)
            prev = row
            ft = (ft + 1) % 5
    out = b"\x89PNG\r\n\x1a\n" + _chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, depth, ctype, 0, 0, 1 if interlace else 0))
    if palette is not None:
        out += _chunk(b"PLTE", palette.astype(np.uint8).tobytes())
    comp = zlib.compress(bytes(raw), 9)
    out += _chunk(b"IDAT", comp[: len(comp) // 2]) + _chunk(b"IDAT", comp[len(comp) // 2:])
    return out + _chunk(b"IEND", b"")


def expected_rgb(samples: np.ndarray, ctype: int, depth: int, palette=None) -> np.ndarray:
    s = samples.astype(np.int64)
    if depth == 16:
        s = s >> 8
    elif depth < 8 and ctype == 0:
        s = s * {1: 255, 2: 0x55, 4: 0x11}[depth]
    if ctype == 3:
        return palette[s[..., 0]].astype(np.uint8)
    if ctype in (0, 4):
        return np.repeat(s[..., :1], 3, axis=2).astype(np.uint8)
    return s[..., :3].astype(np.uint8)


CASES = [(0, 1), (0, 2), (0, 4), (0, 8), (0, 16), (2, 8), (2, 16), (3, 1), (3, 2), (3, 4), (3, 8), (4, 8), (4, 16),
         (6, 8), (6, 16)]


@pytest.mark.parametrize("interlace", [False, True])
@pytest.mark.parametrize("ctype,depth", CASES)
def test_png_decoding_follows_stb_rules(built, tmp_path, ctype, depth, interlace):
    rng = np.random.default_rng(ctype * 100 + depth)
    h, w = 13, 19  # odd sizes exercise partial Adam7 passes and sub-byte row padding
    ch = {0: 1, 2: 3, 3: 1, 4: 2, 6: 4}[ctype]
    palette = None
    if ctype == 3:
        n = 1 << depth
        palette = rng.integers(0, 256, size=(n, 3))
        samples = rng.integers(0, n, size=(h, w, 1))
    else:
        samples = rng.integers(0, 1 << depth, size=(h, w, ch))
    p = tmp_path / "t.png"
    p.write_bytes(encode_png(samples, ctype, depth, interlace, palette))
    got = load_image(p)
    assert got.shape == (h, w, 4)
    assert np.array_equal(got[..., :3], expected_rgb(samples, ctype, depth, palette))
    assert np.all(got[..., 3] == 255)


def test_png_write_roundtrip(built, tmp_path):
    rng = np.random.default_rng(1)
    img = rng.integers(0, 256, size=(37, 53, 3), dtype=np.uint8)
    p = tmp_path / "o.png"
    write_png(p, img)
    assert np.array_equal(load_image(p)[..., :3], img)
    # an independent decoder reads it too
    PIL = pytest.importorskip("PIL.Image")
    assert np.array_equal(np.asarray(PIL.open(p).convert("RGB")), img)


def test_pnm_p6_and_p5(built, tmp_path):
    rng = np.random.default_rng(2)
    rgb = rng.integers(0, 256, size=(7, 11, 3), dtype=np.uint8)
    p6 = tmp_path / "a.ppm"
    p6.write_bytes(b"P6\n# a comment\n11 7\n255\n" + rgb.tobytes())
    assert np.array_equal(load_image(p6)[..., :3], rgb)
    g = rng.integers(0, 256, size=(5, 4), dtype=np.uint8)
    p5 = tmp_path / "b.pgm"
    p5.write_bytes(b"P5 4 5 255\n" + g.tobytes())
    assert np.array_equal(load_image(p5)[..., :3], np.repeat(g[..., None], 3, axis=2))


def test_unsupported_and_corrupt_files(built, tmp_path):
    jpg = tmp_path / "x.jpg"
    jpg.write_bytes(b"\xff\xd8\xff\xe0" + b"\0" * 64)
    with pytest.raises(PrrError) as e:
        load_image(jpg)
    assert e.value.status == abi.ERR_UNSUPPORTED and "JPEG" in str(e.value)
    good = encode_png(np.zeros((4, 4, 3), dtype=np.int64), 2, 8)
    for bad in (good[:40], good[:-20], b"P6\n4 4\n255\n" + b"\0" * 10, b"P6\n4 4\n65535\n" + b"\0" * 96):
        f = tmp_path / "bad.png"
        f.write_bytes(bad)
        with pytest.raises(PrrError) as e:
            load_image(f)
        assert e.value.status in (abi.ERR_IO, abi.ERR_UNSUPPORTED)
    with pytest.raises(PrrError) as e:
        load_image(tmp_path / "missing.png")
    assert e.value.status == abi.ERR_IO
