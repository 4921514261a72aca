"""Image files written through the C ABI (vlrbWriteOutputImages, host code):
the PNG decodes to the host program's tone mapping of the image
(HostProgram/main.cpp:120-168) and the EXR holds the image as half floats
in A, B, G, R order (HostProgram/image.cpp:197-256).  No GPU needed."""
import struct
import zlib

import numpy as np

from vlr_b200 import vlr as VV


def _tone_map(rgb, brightness):
    """The reference's per-channel mapping in float32: max(0), x brightness,
    1 - exp(-x), sRGB gamma, x 256 truncated, at most 255."""
    v = np.maximum(rgb.astype(np.float32), np.float32(0)) * np.float32(brightness)
    v = np.float32(1) - np.exp(-v)
    g = np.where(v <= np.float32(0.0031308), np.float32(12.92) * v,
                 np.float32(1.055) * np.power(v, np.float32(1 / 2.4)) - np.float32(0.055)).astype(np.float32)
    return np.minimum((g * np.float32(256)).astype(np.uint32), 255).astype(np.uint8)


def _read_png(path):
    data = open(path, "rb").read()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, chunks = 8, []
    while pos < len(data):
        n, = struct.unpack(">I", data[pos:pos + 4])
        typ = data[pos + 4:pos + 8]
        body = data[pos + 8:pos + 8 + n]
        crc, = struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])
        assert crc == zlib.crc32(typ + body) & 0xFFFFFFFF, typ
        chunks.append((typ, body))
        pos += 12 + n
    assert [c[0] for c in chunks] == [b"IHDR", b"IDAT", b"IEND"]
    w, h, depth, ctype, comp, filt, inter = struct.unpack(">IIBBBBB", chunks[0][1])
    assert (depth, ctype, comp, filt, inter) == (8, 6, 0, 0, 0)
    raw = zlib.decompress(chunks[1][1])
    rows = np.frombuffer(raw, np.uint8).reshape(h, 1 + 4 * w)
    assert np.all(rows[:, 0] == 0)
    return rows[:, 1:].reshape(h, w, 4)


def _read_exr(path):
    data = open(path, "rb").read()
    magic, version = struct.unpack("<ii", data[:8])
    assert magic == 20000630 and version == 2
    pos, attrs = 8, {}
    while data[pos] != 0:
        name_end = data.index(b"\0", pos)
        name = data[pos:name_end].decode()
        type_end = data.index(b"\0", name_end + 1)
        typ = data[name_end + 1:type_end].decode()
        size, = struct.unpack("<i", data[type_end + 1:type_end + 5])
        attrs[name] = (typ, data[type_end + 5:type_end + 5 + size])
        pos = type_end + 5 + size
    pos += 1
    assert attrs["compression"] == ("compression", b"\0")
    x0, y0, x1, y1 = struct.unpack("<iiii", attrs["dataWindow"][1])
    w, h = x1 - x0 + 1, y1 - y0 + 1
    ch = attrs["channels"][1]
    names, p = [], 0
    while ch[p] != 0:
        e = ch.index(b"\0", p)
        names.append(ch[p:e].decode())
        ptype, = struct.unpack("<i", ch[e + 1:e + 5])
        assert ptype == 1                       # HALF
        p = e + 17
    offsets = struct.unpack("<%dQ" % h, data[pos:pos + 8 * h])
    img = {n: np.zeros((h, w), np.float16) for n in names}
    for y, off in enumerate(offsets):
        ly, size = struct.unpack("<ii", data[off:off + 8])
        assert ly == y and size == len(names) * w * 2
        line = np.frombuffer(data[off + 8:off + 8 + size], np.float16).reshape(len(names), w)
        for k, n in enumerate(names):
            img[n][y] = line[k]
    return names, img


def test_png_and_exr_round_trip(tmp_path):
    rng = np.random.default_rng(5)
    h, w = 37, 300                               # rows of 1201 bytes: several stored deflate blocks
    img = rng.uniform(-0.2, 4.0, (h, w, 4)).astype(np.float32)
    img[..., 3] = 1.0
    img[0, :4, :3] = np.array([0.0, 1e-4, 0.0031308, 50.0], np.float32)[:, None]
    base = tmp_path / "out"
    VV.write_images(img, base, brightness=0.75)
    png = _read_png(str(base) + ".png")
    expect = _tone_map(img[..., :3], 0.75)
    diff = np.abs(png[..., :3].astype(int) - expect.astype(int))
    # exp and pow of the C library and numpy may differ by an ulp, moving a
    # truncation boundary by one level
    assert diff.max() <= 1 and np.mean(diff > 0) < 1e-3, (diff.max(), np.mean(diff > 0))
    assert np.all(png[..., 3] == 255)
    names, exr = _read_exr(str(base) + ".exr")
    assert names == ["A", "B", "G", "R"]
    for n, c in zip("RGBA", range(4)):
        assert np.array_equal(exr[n].view(np.uint16), img[..., c].astype(np.float16).view(np.uint16)), n


def test_writer_rejects_bad_arguments(tmp_path):
    L = VV._api()
    img = np.zeros((2, 2, 4), np.float32)
    from ctypes import c_void_p, c_float
    assert L.vlrbWriteOutputImages(img.ctypes.data_as(c_void_p), 0, 2, str(tmp_path / "x").encode(), c_float(1)) != 0
    assert L.vlrbWriteOutputImages(None, 2, 2, str(tmp_path / "x").encode(), c_float(1)) != 0
    assert L.vlrbWriteOutputImages(img.ctypes.data_as(c_void_p), 2, 2, str(tmp_path / "no_dir" / "x").encode(),
                                   c_float(1)) != 0
