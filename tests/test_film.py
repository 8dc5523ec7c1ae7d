"""EXR film output in the layout SoL's Image::save produces (float channels
named B, G, R, stored in that order, uncompressed scanlines)."""
import struct

import numpy as np

from sol_b200.film import load_exr, save_exr
from sol_b200.renderer import Image


def test_roundtrip_and_channel_order(tmp_path):
    rng = np.random.default_rng(0)
    img = Image(37, 21)
    img.channels[...] = rng.random((3, 21, 37), dtype=np.float32) * 10
    img.channels[0, 3, 5] = np.inf
    img.channels[1, 4, 6] = -0.0
    p = tmp_path / "film.exr"
    img.save(str(p))
    planes, names = load_exr(str(p))
    assert names == ["B", "G", "R"]
    assert np.array_equal(planes[0], img.channels[2]) and np.array_equal(planes[2], img.channels[0])
    back = Image.load(str(p))
    assert np.array_equal(back.channels.view(np.uint32), img.channels.view(np.uint32))


def test_header_fields(tmp_path):
    p = tmp_path / "f.exr"
    save_exr(str(p), np.zeros((3, 4, 5), np.float32))
    data = p.read_bytes()
    assert struct.unpack_from("<ii", data, 0) == (20000630, 2)
    assert b"channels\0chlist\0" in data and b"compression\0compression\0" in data
    i = data.index(b"dataWindow\0box2i\0") + len(b"dataWindow\0box2i\0")
    assert struct.unpack_from("<iiiii", data, i) == (16, 0, 0, 4, 3)
    # offset table: 4 scanlines, each block 8 + 3 * 5 * 4 bytes
    planes, _ = load_exr(str(p))
    assert planes.shape == (3, 4, 5)
    assert len(data) == data.index(b"screenWindowWidth\0float\0") + len(b"screenWindowWidth\0float\0") + 4 + 4 + 1 \
        + 8 * 4 + 4 * (8 + 60)


def test_more_and_fewer_channels(tmp_path):
    a = np.arange(4 * 2 * 3, dtype=np.float32).reshape(4, 2, 3)
    save_exr(str(tmp_path / "a.exr"), a)
    planes, names = load_exr(str(tmp_path / "a.exr"))
    assert names == ["B", "G", "R", "A"] and np.array_equal(planes[3], a[3]) and np.array_equal(planes[0], a[2])
    b = np.ones((1, 2, 2), np.float32)
    save_exr(str(tmp_path / "b.exr"), b)
    planes, names = load_exr(str(tmp_path / "b.exr"))
    assert names == ["Channel_0"] and np.array_equal(planes, b)


def test_independent_reader(tmp_path, monkeypatch):
    """OpenCV's OpenEXR decoder (an implementation independent of this one)
    reads the file back bit for bit, with B, G, R as its channels."""
    monkeypatch.setenv("OPENCV_IO_ENABLE_OPENEXR", "1")
    try:
        import cv2
    except ImportError:
        import pytest
        pytest.skip("OpenCV is not installed")
    rng = np.random.default_rng(1)
    a = rng.random((3, 9, 13), dtype=np.float32) * 5
    save_exr(str(tmp_path / "t.exr"), a)
    im = cv2.imread(str(tmp_path / "t.exr"), cv2.IMREAD_UNCHANGED)
    if im is None:
        import pytest
        pytest.skip("this OpenCV build reads no EXR")
    assert im.shape == (9, 13, 3)
    assert np.array_equal(im[:, :, 0], a[2]) and np.array_equal(im[:, :, 1], a[1]) and np.array_equal(im[:, :, 2], a[0])
