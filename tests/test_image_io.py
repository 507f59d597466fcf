"""Image output against the reference's own output drivers (PNGWriter,
EXRWriter: OUPN001A.cpp, OUEW001A.cpp, compiled from the reference sources into
oracle/_ref/libsirius_ref_io.so): both write the same float buffer; the files
are decoded here (PNG filters, OpenEXR ZIP blocks, from the format
specifications) and the pixel values must be identical. The compressed bytes
may differ (each side chooses its own deflate)."""
import ctypes as C
import os
import struct
import zlib

import numpy as np
import pytest

from sirius_b200.engine import write_image

REF_IO = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                      "libsirius_ref_io.so")


def ref_lib():
    if not os.path.exists(REF_IO):
        pytest.skip("oracle/_ref/libsirius_ref_io.so not built (reference sources absent when building)")
    L = C.CDLL(REF_IO)
    for name in ("ref_write_png", "ref_write_exr"):
        getattr(L, name).argtypes = [C.c_char_p, C.c_int32, C.c_int32, C.c_int32, C.c_void_p]
    for name in ("ref_write_pfm", "ref_write_ppm"):
        getattr(L, name).argtypes = [C.c_char_p, C.c_int32, C.c_int32, C.c_void_p]
    return L


def decode_png(path):
    data = open(path, "rb").read()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, idat, hdr = 8, b"", None
    while pos < len(data):
        n, = struct.unpack(">I", data[pos:pos + 4])
        typ, body = data[pos + 4:pos + 8], data[pos + 8:pos + 8 + n]
        assert zlib.crc32(typ + body) == struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])[0]
        if typ == b"IHDR":
            hdr = struct.unpack(">IIBBBBB", body)
        elif typ == b"IDAT":
            idat += body
        pos += 12 + n
    w, h, depth, ctype = hdr[:4]
    assert depth == 8 and ctype in (2, 6)
    bpp = 3 if ctype == 2 else 4
    raw = zlib.decompress(idat)
    stride = w * bpp
    out = np.zeros((h, stride), dtype=np.int32)
    prev = np.zeros(stride, dtype=np.int32)
    for y in range(h):
        f = raw[y * (stride + 1)]
        line = np.frombuffer(raw, dtype=np.uint8, count=stride, offset=y * (stride + 1) + 1).astype(np.int32)
        cur = np.zeros(stride, dtype=np.int32)
        for i in range(stride):
            a = cur[i - bpp] if i >= bpp else 0
            b = prev[i]
            c = prev[i - bpp] if i >= bpp else 0
            if f == 0:
                p = 0
            elif f == 1:
                p = a
            elif f == 2:
                p = b
            elif f == 3:
                p = (a + b) // 2
            else:
                pa, pb, pc = abs(b - c), abs(a - c), abs(a + b - 2 * c)
                p = a if (pa <= pb and pa <= pc) else (b if pb <= pc else c)
            cur[i] = (line[i] + p) & 0xFF
        out[y] = cur
        prev = cur
    return out.reshape(h, w, bpp).astype(np.uint8)


def decode_exr(path):
    """{channel name: (h, w) uint16 half bits} of a single-part scanline EXR
    (NO / ZIPS / ZIP compression, HALF channels)."""
    d = open(path, "rb").read()
    assert d[:4] == b"\x76\x2f\x31\x01"
    pos, attrs = 8, {}
    while d[pos] != 0:
        e = d.index(b"\0", pos)
        name = d[pos:e].decode()
        e2 = d.index(b"\0", e + 1)
        size, = struct.unpack("<i", d[e2 + 1:e2 + 5])
        attrs[name] = d[e2 + 5:e2 + 5 + size]
        pos = e2 + 5 + size
    pos += 1
    chans, q = [], attrs["channels"]
    i = 0
    while q[i] != 0:
        e = q.index(b"\0", i)
        ptype, = struct.unpack("<i", q[e + 1:e + 5])
        assert ptype == 1
        chans.append(q[i:e].decode())
        i = e + 17
    comp = attrs["compression"][0]
    x0, y0, x1, y1 = struct.unpack("<iiii", attrs["dataWindow"])
    w, h = x1 - x0 + 1, y1 - y0 + 1
    lines = {0: 1, 2: 1, 3: 16}[comp]
    n_chunks = (h + lines - 1) // lines
    offsets = struct.unpack(f"<{n_chunks}Q", d[pos:pos + 8 * n_chunks])
    out = {c: np.zeros((h, w), dtype=np.uint16) for c in chans}
    for off in offsets:
        yy, size = struct.unpack("<ii", d[off:off + 8])
        body = d[off + 8:off + 8 + size]
        nl = min(lines, y1 + 1 - yy)
        raw_size = nl * len(chans) * w * 2
        if comp != 0 and size < raw_size:
            t = np.frombuffer(zlib.decompress(body), dtype=np.uint8).astype(np.int64)
            t = (np.cumsum(t - 128) + 128) % 256  # undo the delta predictor (first byte kept)
            t[0] = np.frombuffer(zlib.decompress(body), dtype=np.uint8)[0]
            half = (len(t) + 1) // 2
            raw = np.empty(len(t), dtype=np.uint8)
            raw[0::2] = t[:half]
            raw[1::2] = t[half:]
        else:
            raw = np.frombuffer(body, dtype=np.uint8)
        v = raw.view("<u2").reshape(nl, len(chans), w)
        for k, c in enumerate(chans):
            out[c][yy - y0:yy - y0 + nl] = v[:, k]
    return out


def test_image(rng, h=37, w=53, c=3, extremes=False):
    img = rng.uniform(-0.2, 1.3, size=(h, w, c)).astype(np.float32)
    img[0, :8, 0] = [0.0, 0.0031308, 0.0031309, 1e-4, 0.5, 1.0, 2.0, -1.0]
    if extremes:
        img[1, :10, 0] = [6e-8, 3e-8, 1e-5, 65504.0, 65520.0, 1e6, -1e6, np.inf, -np.inf, 5.96e-8]
        img[2, :3, 1] = [2.0 ** -24, 2.0 ** -25, 1.5 * 2.0 ** -24]
        img[3, 0, 2] = np.nan
    return img


test_image.__test__ = False


@pytest.mark.parametrize("channels", [3, 4])
def test_png_pixels_match_the_reference_writer(tmp_path, channels):
    ref = ref_lib()
    img = test_image(np.random.default_rng(1), c=channels)
    ours, theirs = str(tmp_path / "ours.png"), str(tmp_path / "ref.png")
    write_image(ours, img)
    assert ref.ref_write_png(theirs.encode(), img.shape[1], img.shape[0], channels, img.ctypes.data) == 1
    a, b = decode_png(ours), decode_png(theirs)
    np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("channels", [3, 4])
def test_exr_pixels_match_the_reference_writer(tmp_path, channels):
    ref = ref_lib()
    img = test_image(np.random.default_rng(2), c=channels, extremes=True, h=41)
    ours, theirs = str(tmp_path / "ours.exr"), str(tmp_path / "ref.exr")
    write_image(ours, img)
    assert ref.ref_write_exr(theirs.encode(), img.shape[1], img.shape[0], channels, img.ctypes.data) == 1
    a, b = decode_exr(ours), decode_exr(theirs)
    assert sorted(a) == sorted(b) == sorted("RGBA"[:channels])
    for ch in a:
        np.testing.assert_array_equal(a[ch], b[ch], err_msg=ch)
    # and the half values are the image's
    np.testing.assert_allclose(a["R"].view(np.float16).astype(np.float32)[5:, :], img[5:, :, 0], rtol=1e-3)


@pytest.mark.parametrize("fmt", ["pfm", "ppm"])
def test_pfm_and_ppm_bytes_match_the_reference_writer(tmp_path, fmt):
    ref = ref_lib()
    img = test_image(np.random.default_rng(3))
    ours, theirs = str(tmp_path / f"ours.{fmt}"), str(tmp_path / f"ref.{fmt}")
    write_image(ours, img)
    assert getattr(ref, f"ref_write_{fmt}")(theirs.encode(), img.shape[1], img.shape[0], img.ctypes.data) == 1
    assert open(ours, "rb").read() == open(theirs, "rb").read()


def test_bad_arguments(tmp_path):
    with pytest.raises(ValueError):
        write_image(str(tmp_path / "x.png"), np.zeros((4, 4, 2), np.float32))
    with pytest.raises(ValueError):
        write_image(str(tmp_path / "x.bmp"), np.zeros((4, 4, 3), np.float32))
    from sirius_b200.engine import SiriusError
    with pytest.raises(SiriusError):
        write_image(str(tmp_path / "no_such_dir" / "x.png"), np.zeros((4, 4, 3), np.float32))
