"""Headless image files (OpenEXR scanline, PFM): byte layout and round trips.

The EXR layout is checked by a small parser written here from the OpenEXR
file-layout description, independent of the library's reader.
"""
import struct

import numpy as np
import pytest


def _img(h, w, c, seed=0):
    rng = np.random.default_rng(seed)
    a = rng.uniform(-2, 50, (h, w, c)).astype(np.float32)
    a[0, 0, 0] = 1.0e30
    return a


def _parse_exr(data: bytes):
    magic, version = struct.unpack_from("<ii", data, 0)
    p, attrs = 8, {}
    while True:
        e = data.index(b"\0", p)
        name = data[p:e].decode()
        p = e + 1
        if not name:
            break
        e = data.index(b"\0", p)
        typ = data[p:e].decode()
        size = struct.unpack_from("<i", data, e + 1)[0]
        attrs[name] = (typ, data[e + 5:e + 5 + size])
        p = e + 5 + size
    chans, q, raw = [], 0, attrs["channels"][1]
    while raw[q] != 0:
        e = raw.index(b"\0", q)
        nm = raw[q:e].decode()
        ptype, plin = struct.unpack_from("<iB", raw, e + 1)
        chans.append((nm, ptype, plin))
        q = e + 17
    x0, y0, x1, y1 = struct.unpack_from("<4i", attrs["dataWindow"][1])
    W, H = x1 - x0 + 1, y1 - y0 + 1
    offsets = struct.unpack_from(f"<{H}Q", data, p)
    lines = {}
    for off in offsets:
        y, size = struct.unpack_from("<ii", data, off)
        lines[y] = data[off + 8:off + 8 + size]
    return magic, version, attrs, chans, W, H, lines


@pytest.mark.parametrize("half", [False, True])
def test_exr_layout(tmp_path, half):
    from meturay_b200 import imageio
    a = _img(5, 7, 4)
    f = tmp_path / "a.exr"
    imageio.write_exr(f, a, half=half)
    magic, version, attrs, chans, W, H, lines = _parse_exr(f.read_bytes())
    assert magic == 20000630 and version == 2
    assert [c[0] for c in chans] == ["A", "B", "G", "R"]
    assert all(c[1] == (1 if half else 2) and c[2] == 1 for c in chans)
    assert attrs["compression"][1] == b"\0" and attrs["lineOrder"][1] == b"\0"
    assert (W, H) == (7, 5) and sorted(lines) == list(range(5))
    dt = np.float16 if half else np.float32
    for y, raw in lines.items():
        v = np.frombuffer(raw, dt).reshape(4, W).astype(np.float32)
        row = a[H - 1 - y]  # the file's first line is the image's top row
        with np.errstate(over="ignore"):  # 1e30 rounds to infinity in binary16
            exp = row.astype(np.float16).astype(np.float32) if half else row
        for k, ch in enumerate((3, 2, 1, 0)):
            assert np.array_equal(v[k], exp[:, ch])


@pytest.mark.parametrize("c", [1, 3, 4])
def test_exr_round_trip(tmp_path, c):
    from meturay_b200 import imageio
    a = _img(9, 4, c, seed=c)
    f = tmp_path / "b.exr"
    imageio.write_exr(f, a if c > 1 else a[..., 0])
    b = imageio.read_image(f)
    assert b.shape == a.shape and np.array_equal(b, a)


def test_pfm_layout_and_round_trip(tmp_path):
    from meturay_b200 import imageio
    a = _img(3, 6, 4)
    f = tmp_path / "c.pfm"
    imageio.write_pfm(f, a)
    raw = f.read_bytes()
    head = b"PF\n6 3\n-1.0\n"
    assert raw.startswith(head)
    body = np.frombuffer(raw[len(head):], "<f4").reshape(3, 6, 3)
    assert np.array_equal(body, a[..., :3])  # rows bottom to top, alpha dropped
    assert np.array_equal(imageio.read_image(f), a[..., :3])
    g = tmp_path / "g.pfm"
    imageio.write_pfm(g, a[..., 1])
    assert g.read_bytes().startswith(b"Pf\n6 3\n-1.0\n")
    assert np.array_equal(imageio.read_image(g)[..., 0], a[..., 1])
    # a big-endian file written here by hand reads the same
    be = tmp_path / "be.pfm"
    be.write_bytes(b"PF\n6 3\n1.0\n" + a[..., :3].astype(">f4").tobytes())
    assert np.array_equal(imageio.read_image(be), a[..., :3])


def test_image_file_errors(tmp_path):
    import meturay_b200 as m
    from meturay_b200 import imageio
    a = _img(4, 4, 3)
    with pytest.raises(m.MrbError, match=".exr or .pfm"):
        imageio.read_image(tmp_path / "x.png")
    f = tmp_path / "d.exr"
    imageio.write_exr(f, a)
    data = bytearray(f.read_bytes())
    k = data.index(b"compression\0compression\0") + len(b"compression\0compression\0") + 4
    data[k] = 3  # ZIP
    f.write_bytes(bytes(data))
    with pytest.raises(m.MrbError, match="NO_COMPRESSION"):
        imageio.read_image(f)
    imageio.write_exr(f, a)
    f.write_bytes(f.read_bytes()[:-10])
    with pytest.raises(m.MrbError):
        imageio.read_image(f)
    (tmp_path / "e.pfm").write_bytes(b"PF\n6 3\n")
    with pytest.raises(m.MrbError):
        imageio.read_image(tmp_path / "e.pfm")
    with pytest.raises(m.MrbError):
        imageio.read_image(tmp_path / "missing.exr")
