"""The C-ABI library loads and exports every declared entry point (no GPU)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

import bmfr_b200 as B
from bmfr_b200 import _native

ROOT = Path(__file__).resolve().parent.parent


def declared_functions(headers):
    names = []
    for h in headers:
        text = re.sub(r"/\*.*?\*/", "", (ROOT / "include" / h).read_text(), flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(bmfr_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


# Which library exports the entry points of each header.
LIBRARY_HEADERS = {
    "pipeline": ["bmfr_b200.h", "bmfr_batch.h", "bmfr_image.h"],
    "scene": ["bmfr_scene.h"],
}


def test_every_header_belongs_to_a_library():
    listed = sorted(h for hs in LIBRARY_HEADERS.values() for h in hs)
    assert listed == sorted(p.name for p in (ROOT / "include").glob("*.h"))


def test_every_declared_symbol_is_exported():
    import bmfr_scene
    paths = {"pipeline": _native.library_path(), "scene": bmfr_scene.library_path()}
    total = 0
    for which, headers in LIBRARY_HEADERS.items():
        names = declared_functions(headers)
        total += len(names)
        lib = C.CDLL(paths[which])
        missing = [n for n in names if not hasattr(lib, n)]
        assert not missing, (which, missing)
    assert total > 20


def test_scene_library_holds_no_pipeline_code():
    """The input source is a library of its own, so code that only renders
    inputs (the reference arm of the benchmark) maps no pipeline code."""
    import bmfr_scene
    lib = C.CDLL(bmfr_scene.library_path())
    for n in declared_functions(LIBRARY_HEADERS["pipeline"]):
        assert not hasattr(lib, n), n
    pipe = C.CDLL(_native.library_path())
    for n in declared_functions(LIBRARY_HEADERS["scene"]):
        assert not hasattr(pipe, n), n


def test_defaults_are_the_reference_values():
    p = B.default_params()
    assert p.noise_amount == 1e-2                      # bmfr.cpp:58
    assert p.blend_alpha == np.float32(0.2)            # bmfr.cpp:60
    assert p.second_blend_alpha == np.float32(0.1)     # bmfr.cpp:61
    assert p.taa_blend_alpha == np.float32(0.2)        # bmfr.cpp:62
    assert p.use_half_precision_in_tmp_data == 1       # bmfr.cpp:88
    assert p.compressed_r == 1 and p.cache_tmp_data == 1


def test_block_offset_table():
    """The host copy the ABI exports equals the reference's table
    (opencl/bmfr.cl:267-285), entry by entry; the device copy is checked
    against the oracle over 17 frames on the GPU."""
    from test_oracle_kats import BLOCK_OFFSETS
    t = B.block_offsets()
    assert t.shape == (16, 2)
    np.testing.assert_array_equal(t, np.asarray(BLOCK_OFFSETS, dtype=np.int32))
    assert t.min() >= -16 and t.max() <= 14


def test_status_strings_and_errors():
    assert _native.lib.bmfr_status_string(0) == b"ok"
    assert _native.lib.bmfr_status_string(-10) == b"size beyond the fixed maximum"
    with pytest.raises(B.BmfrError):
        B.Plan(8, 8)           # rejected before any device call
    p = B.default_params(pipeline=7)
    with pytest.raises(B.BmfrError):
        B.Plan(64, 64, params=p)


def test_plan_creation_fails_loudly_without_a_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(B.BmfrError, match="CUDA"):
        B.Plan(256, 256)


def test_scene_is_deterministic_and_in_range():
    sc = B.Scene(42, 96, 64, 12)
    a, b = sc.render(3, clean=True), sc.render(3, clean=True)
    for k in a:
        np.testing.assert_array_equal(a[k], b[k])
    n = np.linalg.norm(a["normals"], axis=-1)
    hit = n > 0
    assert hit.mean() > 0.3
    np.testing.assert_allclose(n[hit], 1.0, atol=1e-5)
    assert (np.abs(a["positions"]) <= 64.0001).all()
    assert ((a["positions"] ** 2) < 65504).all()
    assert (a["noisy"] >= 0).all() and (a["clean"] >= 0).all() and (a["clean"] <= 1).all()
    assert not np.signbit(a["positions"][a["positions"] == 0]).any()
    # Different seeds give different scenes; frames move the camera.
    assert not np.array_equal(B.Scene(43, 96, 64, 12).render(3)["positions"], a["positions"])
    assert not np.array_equal(sc.camera(0), sc.camera(1))
    np.testing.assert_array_equal(sc.pixel_offset(5), [0.5, 0.5])


def test_scene_camera_projects_visible_points_into_the_image():
    W, H = 128, 96
    sc = B.Scene(1, W, H, 12)
    d = sc.render(2)
    m = sc.camera(2).reshape(4, 4)
    p = d["positions"].reshape(-1, 3)
    hit = np.linalg.norm(d["normals"].reshape(-1, 3), axis=-1) > 0
    ph = np.concatenate([p, np.ones((p.shape[0], 1), np.float32)], axis=1)
    clip = ph @ m                     # row-vector convention of bmfr.cl:343-347
    uv = (clip[:, :2] / clip[:, 3:4] + 1) / 2
    pix = uv * [W, H] - 0.5
    yy, xx = np.mgrid[0:H, 0:W]
    expect = np.stack([xx.ravel(), yy.ravel()], axis=1)
    assert np.abs(pix[hit] - expect[hit]).max() < 1e-2
