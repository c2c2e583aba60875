"""The reference's frame loop as a compiled C++ host program
(tests/native/host_loop.cpp) against the C ABI alone: it builds and links
with g++ against include/ and the two libraries; without a GPU it stops with
the plan's error, and on a GPU its frames equal, bit for bit, those of the
same loop through the Python front end (which the parity tests pin to the
oracle)."""
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent


def _build(tmp_path) -> Path:
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.fail("g++ is required to build the host program")
    lib_dirs = [ROOT / "bmfr_b200", ROOT / "bmfr_scene"]
    for d, name in zip(lib_dirs, ("libbmfr_b200.so", "libbmfr_scene.so")):
        assert (d / name).exists(), f"{d / name} is missing: build the libraries first"
    exe = tmp_path / "host_loop"
    cmd = [gxx, "-O2", "-std=c++17", f"-I{ROOT / 'include'}", str(HERE / "native" / "host_loop.cpp"), "-o", str(exe)]
    for d, name in zip(lib_dirs, ("bmfr_b200", "bmfr_scene")):
        cmd += [f"-L{d}", f"-l{name}", f"-Wl,-rpath,{d}"]
    subprocess.run(cmd, check=True)
    return exe


def test_host_program_builds_and_fails_loudly_without_a_gpu(tmp_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present: the GPU test runs the program")
    exe = _build(tmp_path)
    r = subprocess.run([str(exe), "64", "64", "1", "1", str(tmp_path / "out.bin")], capture_output=True, text=True)
    assert r.returncode == 2, r.stdout + r.stderr
    assert "bmfr_plan_create" in r.stderr


@pytest.mark.gpu
def test_host_program_frames_equal_the_python_loop(cuda, tmp_path):
    import bmfr_b200 as B
    W, H, F, SEED = 256, 192, 5, 51
    exe = _build(tmp_path)
    out = tmp_path / "frames.bin"
    r = subprocess.run([str(exe), str(W), str(H), str(F), str(SEED), str(out)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    got = np.fromfile(out, dtype=np.float32).reshape(F, H, W, 3)
    sc = B.Scene(SEED, W, H, 12)
    plan = B.Plan(W, H, position_limit_squared=sc.position_limit_squared,
                  normal_limit_squared=sc.normal_limit_squared)
    for f in range(F):
        d = sc.render(f)
        plan.upload_frame(d["albedo"], d["normals"], d["positions"], d["noisy"])
        plan.denoise_frame(sc.prev_camera(f), sc.pixel_offset(f))
        np.testing.assert_array_equal(got[f], plan.download_result(), err_msg=f"frame {f}")
    plan.close()
