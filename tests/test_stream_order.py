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
