"""The on-device G-buffer generator (bmfr_scene_render_device) against the
host renderer (bmfr_scene_render) that every parity test feeds the oracle.

The batched and served benchmarks render their inputs on the GPU, so this
pins those inputs to the host stream.  The two are not bit-identical, by
construction, and the tolerances below follow from how they differ:

* the device casts rays in float, the host in double.  A hit at distance t
  along a ray whose direction has height d_y moves by about
  t * (error of d_y) / |d_y| = t^2 (error of d_y) / h on the ground plane
  (camera height h = 3, d_y = -h / t), so with float directions (error
  ~1e-7) the position of a pixel that hits the same object agrees to
  |dp| <= 1e-4 + 2e-7 t^2, t <= |p| + 10.5 (the camera's distance from the
  origin), on 99.9 % of the pixels; a ray that grazes a sphere has a small
  discriminant b^2 - c, whose float rounding (b^2 ~ 100) sqrt magnifies, so
  the few such pixels are held to |dp| <= 5e-3; a sphere's normal is
  (p - c) / r, so where the position bound holds the normals agree to that
  bound divided by the smallest radius (0.3), and the plane's are exact;
* a grazing ray at an object's silhouette may hit another object (or
  nothing) in one of them: such pixels are counted (albedo differs, or one
  side misses) and must stay below 0.2 % of the image;
* the noise draws come from the same 64-bit counter hash, as a 24-bit
  uniform on the device and a 53-bit one on the host; Box-Muller's log and
  cos then agree to ~1e-6 except where the uniform is tiny (the far tail of
  the lognormal); the colour also carries the shading max(0, n.l) + 0.1 >=
  0.1, whose relative error is at most 10 times the normal's, so where the
  position bound holds the 1-spp colour is within 1e-4 + 10 times the normal
  bound, relative, on 99.99 % of the channels, and a firefly decision (a
  uniform below 0.001, a factor of 100 when it differs) may differ only where
  a uniform lies within 2^-24 of the threshold: at most 1e-5 of the channels
  are off by more than 10 %;
* the albedo is copied from the same table: exact where the object agrees;
* the noise-free image is clamp(pow(albedo * (max(0, n.l) + 0.1), 0.4545)),
  whose slope in the normal is at most 0.4545 x^-0.545 * albedo <= 8 for
  albedo in [0.05, 0.95] and shading >= 0.1, so it agrees to 1e-4 plus 8
  times the normal bound where the position bound holds, and to 0.05 on the
  grazing pixels.
"""
import numpy as np
import pytest

import bmfr_b200 as B

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("W,H,frames", [(256, 192, (0, 1, 7)), (1280, 720, (0, 30))])
def test_device_render_matches_host_render(cuda, W, H, frames):
    import torch
    sc = B.Scene(77, W, H, 16)
    n = W * H * 3
    dev = {k: torch.empty(n, dtype=torch.float32, device=cuda)
           for k in ("albedo", "normals", "positions", "noisy", "clean")}
    for f in frames:
        host = sc.render(f, clean=True)
        sc.render_device(f, dev["albedo"], dev["normals"], dev["positions"], dev["noisy"], clean=dev["clean"])
        torch.cuda.synchronize()
        got = {k: v.cpu().numpy().reshape(H, W, 3) for k, v in dev.items()}
        hit_h = np.any(host["normals"] != 0, axis=-1)
        hit_d = np.any(got["normals"] != 0, axis=-1)
        same = (hit_h == hit_d) & np.all(host["albedo"] == got["albedo"], axis=-1)
        assert hit_h.mean() > 0.3, "the scene must cover a good part of the image"
        assert (~same).mean() < 2e-3, f"frame {f}: {(~same).mean():.2e} of pixels hit different objects"
        m = same & hit_h
        dp = np.linalg.norm(got["positions"] - host["positions"], axis=-1)[m]
        t = np.linalg.norm(host["positions"], axis=-1)[m] + 10.5
        bound = 1e-4 + 2e-7 * t * t
        ok = dp <= bound
        assert ok.mean() >= 0.999, f"frame {f}: {(~ok).sum()} positions beyond the ray-length bound"
        assert dp.max() <= 5e-3, f"frame {f}: positions {dp.max():.2e}"
        dn = np.linalg.norm(got["normals"] - host["normals"], axis=-1)[m]
        nbound = bound / 0.3 + 1e-5
        assert (dn[ok] <= nbound[ok]).all(), f"frame {f}: normals {(dn[ok] / nbound[ok]).max():.2f} of the bound"
        # Misses are all zero on both sides.
        miss = same & ~hit_h
        for k in ("albedo", "normals", "positions", "noisy", "clean"):
            assert (got[k][miss] == 0).all() and (host[k][miss] == 0).all(), k
        rel = np.abs(got["noisy"] - host["noisy"])[m] / np.maximum(np.abs(host["noisy"][m]), 1e-6)
        rbound = (1e-4 + 10.0 * nbound)[:, None]
        within = (rel <= rbound)[ok]
        assert within.mean() >= 0.9999, f"frame {f}: {(~within).sum()} colour channels beyond the bound"
        assert (rel > 0.1).mean() <= 1e-5, f"frame {f}: {(rel > 0.1).sum()} channels off by more than 10 %"
        dc = np.abs(got["clean"] - host["clean"])[m].max(axis=-1)
        cbound = 1e-4 + 8.0 * nbound
        assert (dc[ok] <= cbound[ok]).all(), f"frame {f}: clean {(dc[ok] / cbound[ok]).max():.2f} of the bound"
        assert dc.max() <= 0.05, f"frame {f}: clean {dc.max():.2e}"
