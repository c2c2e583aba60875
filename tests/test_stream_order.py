"""Stream ordering of the drop-in entry points.  Their kernels are launched
with programmatic stream serialization and wait for the preceding kernel
before touching memory, so a caller's kernel that writes an entry point's
input immediately before it on the same stream (no synchronisation between)
must be complete when the entry point reads: the results equal, bit for bit,
those computed from the same input written and synchronised beforehand."""
import numpy as np
import pytest

import bmfr_b200 as B

pytestmark = pytest.mark.gpu

W, H = 1280, 720   # 984 blocks: the persistent fitter takes several blocks per CTA


def _busy(cuda):
    """Queue ~1 ms of the caller's own kernels on the current stream."""
    import torch
    big = torch.ones(128 << 20, dtype=torch.float32, device=cuda)
    for _ in range(4):
        big.mul_(1.0001)
    return big


def _bits(t):
    return t.detach().cpu().numpy().view(np.uint32)


def test_fitter_reads_tmp_written_by_the_kernel_before_it(cuda):
    import torch
    plan = B.Plan(W, H)
    g = torch.Generator(device="cpu").manual_seed(7)
    n = plan.sizes.blocks * 13 * 1024
    src = (torch.rand(n, generator=g) * 4.0 - 1.0).to(torch.float16).to(cuda)
    w_a = torch.empty(plan.sizes.blocks * 30, dtype=torch.float32, device=cuda)
    mm_a = torch.empty(plan.sizes.blocks * 12, dtype=torch.float32, device=cuda)
    w_b, mm_b = torch.empty_like(w_a), torch.empty_like(mm_a)
    B.fitter(plan, w_a, mm_a, src.clone(), 3)
    torch.cuda.synchronize()
    dst = torch.zeros_like(src)
    torch.cuda.synchronize()
    busy = _busy(cuda)
    torch.mul(src, 1.0, out=dst)          # the caller's kernel writes tmp_data ...
    B.fitter(plan, w_b, mm_b, dst, 3)     # ... and the fitter follows at once
    torch.cuda.synchronize()
    np.testing.assert_array_equal(_bits(w_b), _bits(w_a))
    np.testing.assert_array_equal(_bits(mm_b), _bits(mm_a))
    del busy
    plan.close()


def test_taa_reads_frame_written_by_the_kernel_before_it(cuda):
    import torch
    plan = B.Plan(W, H)
    g = torch.Generator(device="cpu").manual_seed(11)
    ys, xs = torch.meshgrid(torch.arange(H, dtype=torch.float32), torch.arange(W, dtype=torch.float32),
                            indexing="ij")
    pp = torch.stack([xs + 0.3, ys - 0.2], dim=-1).reshape(-1).to(cuda)   # prev_frame_pixel, float2
    tm = torch.rand(W * H * 3, generator=g).to(cuda)
    prev = torch.rand(W * H * 3, generator=g).to(cuda)
    res_a = torch.empty_like(tm)
    res_b = torch.empty_like(tm)
    B.taa(plan, pp, tm.clone(), res_a, prev, 5)
    torch.cuda.synchronize()
    tm_dst = torch.zeros_like(tm)
    torch.cuda.synchronize()
    busy = _busy(cuda)
    torch.mul(tm, 1.0, out=tm_dst)        # the caller's kernel writes the tone-mapped frame ...
    B.taa(plan, pp, tm_dst, res_b, prev, 5)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(_bits(res_b), _bits(res_a))
    del busy
    plan.close()


def test_in_place_accumulation_reads_colour_written_by_the_kernel_before_it(cuda):
    """The in-place accumulate_noisy_data runs two chained kernels (in-image
    pixels, then mirrored margin pixels that read the colour the first pass
    wrote); the colour it blends in place is written by the caller's kernel
    immediately before it."""
    import torch
    plan = B.Plan(W, H)
    sc = B.Scene(13, W, H, 12)
    d0, d1 = sc.render(0), sc.render(1)
    t = lambda a: torch.from_numpy(a).reshape(-1).to(cuda)
    n0, p0, c0 = t(d0["normals"]), t(d0["positions"]), t(d0["noisy"])
    n1, p1, src = t(d1["normals"]), t(d1["positions"]), t(d1["noisy"])
    spp_prev = torch.full((W * H,), 3, dtype=torch.uint8, device=cuda)

    def run(noisy):
        out = {"pp": torch.zeros(W * H * 2, dtype=torch.float32, device=cuda),
               "acc": torch.zeros(W * H, dtype=torch.uint8, device=cuda),
               "spp": torch.zeros(W * H, dtype=torch.uint8, device=cuda),
               "tmp": torch.zeros(plan.sizes.tmp_data_bytes // 2, dtype=torch.int16, device=cuda)}
        B.accumulate_noisy_data(plan, out["pp"], out["acc"], n1, n0, p1, p0, noisy, c0, spp_prev, out["spp"],
                                out["tmp"], sc.prev_camera(1), sc.pixel_offset(1), 1)
        out["noisy"] = noisy
        return out

    a = run(src.clone())
    torch.cuda.synchronize()
    dst = torch.zeros_like(src)
    torch.cuda.synchronize()
    busy = _busy(cuda)
    torch.mul(src, 1.0, out=dst)          # the caller's kernel writes the frame's colour ...
    b = run(dst)                          # ... and the two in-place passes follow at once
    torch.cuda.synchronize()
    for k in a:
        np.testing.assert_array_equal(a[k].cpu().numpy().view(np.uint8), b[k].cpu().numpy().view(np.uint8),
                                      err_msg=k)
    del busy
    plan.close()


def test_noalloc_fitter_reads_tmp_written_by_the_kernel_before_it(cuda):
    """bmfr_fitter_noalloc chains the frame's noise table (into its static
    array) and the fitter; tmp_data comes from the caller's kernel just
    before them."""
    import ctypes as C
    import torch
    from bmfr_b200 import _native
    params = B.default_params()
    g = torch.Generator(device="cpu").manual_seed(9)
    nb = B.Plan(W, H).sizes.blocks
    src = (torch.rand(nb * 13 * 1024, generator=g) * 4.0 - 1.0).to(torch.float16).to(cuda)
    s = torch.cuda.current_stream()

    def fit(tmp, w, mm):
        st = _native.lib.bmfr_fitter_noalloc(C.byref(params), W, H, C.c_void_p(w.data_ptr()),
                                            C.c_void_p(mm.data_ptr()), C.c_void_p(tmp.data_ptr()), 4,
                                            C.c_void_p(s.cuda_stream))
        assert st == 0, _native.lib.bmfr_last_error().decode()

    w_a = torch.empty(nb * 30, dtype=torch.float32, device=cuda)
    mm_a = torch.empty(nb * 12, dtype=torch.float32, device=cuda)
    w_b, mm_b = torch.empty_like(w_a), torch.empty_like(mm_a)
    fit(src.clone(), w_a, mm_a)
    torch.cuda.synchronize()
    dst = torch.zeros_like(src)
    torch.cuda.synchronize()
    busy = _busy(cuda)
    torch.mul(src, 1.0, out=dst)
    fit(dst, w_b, mm_b)
    torch.cuda.synchronize()
    assert _native.lib.bmfr_fitter_noalloc_check(C.c_void_p(s.cuda_stream)) == 0
    np.testing.assert_array_equal(_bits(w_b), _bits(w_a))
    np.testing.assert_array_equal(_bits(mm_b), _bits(mm_a))
    del busy
