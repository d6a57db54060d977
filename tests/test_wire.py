"""The host-side file formats of libpm_stereo.so (csrc/wire.cpp): the PFM / NPY / PPM writers that
replace the reference's "32FC1" image message and colour window (evaluate.cc:271-307), and the
frame reader of the sequence driver, checked against numpy and OpenCV.  No GPU needed."""
import ctypes
import os
import struct
import zlib

import numpy as np
import pytest

from oracle import imgproc as ip

cv2 = pytest.importorskip("cv2")


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


def read(pm_lib, path, cap=None):
    W, H = ctypes.c_int(), ctypes.c_int()
    st = pm_lib.pm_read_image_u8(path.encode(), ctypes.byref(W), ctypes.byref(H), None, 0)
    if st != 0:
        return st, None
    out = np.empty((H.value, W.value), np.uint8)
    st = pm_lib.pm_read_image_u8(path.encode(), ctypes.byref(W), ctypes.byref(H), _p(out),
                                 out.size if cap is None else cap)
    return st, out


def test_pfm_and_npy_round_trip(pm_lib, tmp_path):
    from probabilistic_mapping_b200.sequence import read_pfm
    rng = np.random.default_rng(1)
    d = rng.random((37, 53)).astype(np.float32) * 20
    d[3, 4] = 1000.0
    big = np.zeros((37, 64), np.float32)          # a pitched source: 64 floats per row
    big[:, :53] = d
    for pitch, src in ((0, d), (64 * 4, big)):
        pfm, npy = str(tmp_path / "d.pfm"), str(tmp_path / "d.npy")
        assert pm_lib.pm_write_pfm(pfm.encode(), 53, 37, _p(src), pitch) == 0
        assert pm_lib.pm_write_npy(npy.encode(), 53, 37, _p(src), pitch) == 0
        np.testing.assert_array_equal(read_pfm(pfm), d)
        np.testing.assert_array_equal(np.load(npy), d)
        got = cv2.imread(pfm, cv2.IMREAD_UNCHANGED)
        if got is not None:   # OpenCV reads PFM too
            np.testing.assert_array_equal(got, d)
    assert pm_lib.pm_write_pfm(str(tmp_path / "no" / "x.pfm").encode(), 53, 37, _p(d), 0) != 0
    assert pm_lib.pm_write_npy(npy.encode(), 53, 37, _p(d), 4) != 0     # pitch below a row


def test_ppm_writes_bgr_as_rgb(pm_lib, tmp_path):
    rng = np.random.default_rng(2)
    bgr = rng.integers(0, 256, (21, 34, 3), dtype=np.uint8)
    path = str(tmp_path / "c.ppm")
    assert pm_lib.pm_write_ppm(path.encode(), 34, 21, _p(bgr), 0) == 0
    np.testing.assert_array_equal(cv2.imread(path, cv2.IMREAD_COLOR), bgr)


def _png(path, W, H, depth, ctype, rows, plte=None):
    def chunk(tag, data):
        return struct.pack(">I", len(data)) + tag + data + struct.pack(">I", zlib.crc32(tag + data) & 0xffffffff)
    body = chunk(b"IHDR", struct.pack(">IIBBBBB", W, H, depth, ctype, 0, 0, 0))
    if plte is not None:
        body += chunk(b"PLTE", plte.astype(np.uint8).tobytes())
    raw = b"".join(b"\x00" + r for r in rows)
    with open(path, "wb") as f:
        f.write(b"\x89PNG\r\n\x1a\n" + body + chunk(b"IDAT", zlib.compress(raw)) + chunk(b"IEND", b""))


def test_reader_formats(pm_lib, tmp_path):
    rng = np.random.default_rng(3)
    g = rng.integers(0, 256, (29, 41), dtype=np.uint8)
    bgr = rng.integers(0, 256, (29, 41, 3), dtype=np.uint8)
    grey_of_bgr = ip.rgb_to_grey(bgr[..., 2], bgr[..., 1], bgr[..., 0])
    cases = []
    # OpenCV-written PNGs use the adaptive filters (Sub, Up, Average, Paeth)
    cv2.imwrite(str(tmp_path / "g8.png"), g); cases.append(("g8.png", g))
    cv2.imwrite(str(tmp_path / "c8.png"), bgr); cases.append(("c8.png", grey_of_bgr))
    bgra = np.concatenate([bgr, rng.integers(0, 256, (29, 41, 1), dtype=np.uint8)], -1)
    cv2.imwrite(str(tmp_path / "c8a.png"), bgra); cases.append(("c8a.png", grey_of_bgr))
    g16 = rng.integers(0, 65536, (29, 41), dtype=np.uint16)
    cv2.imwrite(str(tmp_path / "g16.png"), g16); cases.append(("g16.png", (g16 >> 8).astype(np.uint8)))
    c16 = rng.integers(0, 65536, (29, 41, 3), dtype=np.uint16)
    cv2.imwrite(str(tmp_path / "c16.png"), c16)
    cases.append(("c16.png", ip.rgb_to_grey(c16[..., 2] >> 8, c16[..., 1] >> 8, c16[..., 0] >> 8)))
    cv2.imwrite(str(tmp_path / "g.pgm"), g); cases.append(("g.pgm", g))
    cv2.imwrite(str(tmp_path / "c.ppm"), bgr); cases.append(("c.ppm", grey_of_bgr))
    np.save(tmp_path / "g.npy", g); cases.append(("g.npy", g))
    # palette and 4-bit grey PNGs, written by hand
    plte = rng.integers(0, 256, (16, 3))
    idx = rng.integers(0, 16, (29, 41), dtype=np.uint8)
    packed = [bytes(((r[0::2] << 4) | np.append(r[1::2], 0)[:len(r[0::2])]).astype(np.uint8)) for r in idx]
    _png(str(tmp_path / "p4.png"), 41, 29, 4, 3, packed, plte)
    cases.append(("p4.png", ip.rgb_to_grey(plte[idx, 0], plte[idx, 1], plte[idx, 2])))
    _png(str(tmp_path / "g4.png"), 41, 29, 4, 0, packed)
    cases.append(("g4.png", (idx * 17).astype(np.uint8)))
    for name, want in cases:
        st, got = read(pm_lib, str(tmp_path / name))
        assert st == 0, name
        np.testing.assert_array_equal(got, want, err_msg=name)


def test_reader_errors(pm_lib, tmp_path):
    assert read(pm_lib, str(tmp_path / "missing.png"))[0] != 0
    (tmp_path / "junk.png").write_bytes(b"not an image at all")
    assert read(pm_lib, str(tmp_path / "junk.png"))[0] != 0
    g = np.zeros((10, 12), np.uint8)
    cv2.imwrite(str(tmp_path / "g.png"), g)
    W, H = ctypes.c_int(), ctypes.c_int()
    buf = np.empty(50, np.uint8)
    assert pm_lib.pm_read_image_u8(str(tmp_path / "g.png").encode(), ctypes.byref(W), ctypes.byref(H), _p(buf), 50) != 0
    assert (W.value, H.value) == (12, 10)
