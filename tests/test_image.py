"""PFM output and PSNR (include/bmfr_image.h): host code, no GPU."""
import numpy as np
import pytest

import bmfr_b200 as B


def test_pfm_round_trip(tmp_path):
    rng = np.random.default_rng(5)
    img = rng.standard_normal((7, 11, 3)).astype(np.float32)
    img[0, 0] = [np.inf, -0.0, 1e-40]
    path = tmp_path / "frame.pfm"
    B.write_pfm(path, img)
    raw = path.read_bytes()
    assert raw.startswith(b"PF\n11 7\n-1.0\n")
    # bottom row first in the file
    body = np.frombuffer(raw[len(b"PF\n11 7\n-1.0\n"):], dtype="<f4").reshape(7, 11, 3)
    np.testing.assert_array_equal(body[::-1], img)
    back = B.read_pfm(path)
    assert back.tobytes() == img.tobytes()


def test_pfm_big_endian_and_errors(tmp_path):
    img = np.arange(2 * 3 * 3, dtype=np.float32).reshape(2, 3, 3)
    path = tmp_path / "be.pfm"
    path.write_bytes(b"PF\n3 2\n1.0\n" + img[::-1].astype(">f4").tobytes())
    np.testing.assert_array_equal(B.read_pfm(path), img)
    bad = tmp_path / "bad.pfm"
    bad.write_bytes(b"Pf\n3 2\n-1.0\n" + bytes(24))
    with pytest.raises(B.BmfrError):
        B.read_pfm(bad)
    with pytest.raises(B.BmfrError):
        B.read_pfm(tmp_path / "missing.pfm")


def test_psnr():
    a = np.zeros((4, 4, 3), np.float32)
    b = a.copy()
    assert B.psnr(a, b) == float("inf")
    b[0, 0, 0] = 0.1   # MSE = d^2 / 48 with d the float32 nearest 0.1
    d2 = float(np.float32(0.1)) ** 2
    assert B.psnr(a, b) == pytest.approx(10 * np.log10(48 / d2), rel=1e-12)
    assert B.psnr(a, b, peak=2.0) == pytest.approx(10 * np.log10(4 * 48 / d2), rel=1e-12)
