"""gg_write_png (the headless stand-in for Capture.writePNG,
Capture.swift:38-94) is host code: a PNG it writes decodes, with its
chunks' CRCs checked and the image data inflated, to the very pixels it was
given."""
import struct
import zlib

import numpy as np
import pytest


def decode_png(data: bytes):
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, chunks = 8, []
    while pos < len(data):
        (n,) = struct.unpack(">I", data[pos:pos + 4])
        kind = data[pos + 4:pos + 8]
        body = data[pos + 8:pos + 8 + n]
        (crc,) = struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])
        assert zlib.crc32(kind + body) & 0xFFFFFFFF == crc, kind
        chunks.append((kind, body))
        pos += 12 + n
    kinds = [k for k, _ in chunks]
    assert kinds[0] == b"IHDR" and kinds[-1] == b"IEND"
    w, h, depth, colour, comp, filt, interlace = struct.unpack(">IIBBBBB", chunks[0][1])
    assert (depth, colour, comp, filt, interlace) == (8, 6, 0, 0, 0)
    raw = zlib.decompress(b"".join(b for k, b in chunks if k == b"IDAT"))
    rows = np.frombuffer(raw, np.uint8).reshape(h, 1 + 4 * w)
    assert (rows[:, 0] == 0).all()  # filter type none on every row
    return rows[:, 1:].reshape(h, w, 4), kinds


@pytest.mark.parametrize("w,h", [(1, 1), (37, 5), (320, 180)])
def test_png_round_trips_its_pixels(tmp_path, w, h):
    import gargantua_b200 as g

    rng = np.random.default_rng(w * h)
    px = rng.integers(0, 256, (h, w, 4), dtype=np.uint8)
    path = str(tmp_path / "frame.png")
    g.write_png(path, px)
    got, kinds = decode_png(open(path, "rb").read())
    assert np.array_equal(got, px)
    assert b"sRGB" in kinds  # the pixels are sRGB-encoded (the tone map's output)


def test_png_refuses_a_bad_shape(tmp_path):
    import gargantua_b200 as g

    with pytest.raises(ValueError):
        g.write_png(str(tmp_path / "x.png"), np.zeros((4, 4, 3), np.uint8))
