"""dort_gpu_render_device_noalloc, the render entry point for callers that
cannot allocate GPU memory during a render (host applications that own all
device memory under a fixed budget, real-time loops that cannot absorb
cudaFree's synchronisation).

It must give the image of the regular entry point, dort_gpu_render_device,
on two calls in a row (the second call finds the first call's data in the
shared scratch array), and reject images larger than its fixed scratch.
Collected last so that a run stopping at the first failure has run every
other test first.
"""
import numpy as np
import pytest

import dort_b200 as db
from dort_b200 import scenes
from tests import ptcheck

pytestmark = pytest.mark.gpu


def test_noalloc_matches_regular_render_twice(cuda):
    import torch
    sd = scenes.cornell_box()
    sc = db.scene_from_dict(sd)
    p = db.render_params(sd["camera"], 96, 64, 16, max_depth=8, seed=21)
    stream = torch.cuda.current_stream().cuda_stream
    ref = torch.zeros(96 * 64 * 3, dtype=torch.float32, device=cuda)
    sc.render_device(p, ref.data_ptr(), stream)
    torch.cuda.synchronize()
    expected = ref.cpu().numpy()
    assert expected.mean() > 0
    for _ in range(2):
        out = torch.full((96 * 64 * 3,), -1.0, dtype=torch.float32, device=cuda)
        sc.render_device_noalloc(p, out.data_ptr(), stream)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert ptcheck.rel_rmse(got, expected) < 1e-6
        assert np.isfinite(got).all()


def test_noalloc_second_scene_and_size_after_first(cuda):
    import torch
    sd = scenes.cornell_variant("delt")
    sc = db.scene_from_dict(sd)
    stream = torch.cuda.current_stream().cuda_stream
    for (w, h, spp) in ((40, 30, 8), (128, 96, 4)):
        p = db.render_params(sd["camera"], w, h, spp, seed=3)
        ref = torch.zeros(w * h * 3, dtype=torch.float32, device=cuda)
        out = torch.zeros(w * h * 3, dtype=torch.float32, device=cuda)
        sc.render_device(p, ref.data_ptr(), stream)
        sc.render_device_noalloc(p, out.data_ptr(), stream)
        torch.cuda.synchronize()
        assert ptcheck.rel_rmse(out.cpu().numpy(), ref.cpu().numpy()) < 1e-6


def test_noalloc_rejects_images_beyond_its_scratch(cuda):
    import torch
    sd = scenes.cornell_box()
    sc = db.scene_from_dict(sd)
    p = db.render_params(sd["camera"], 2048, 1024, 1)
    out = torch.zeros(16, dtype=torch.float32, device=cuda)
    with pytest.raises(db.DortError) as e:
        sc.render_device_noalloc(p, out.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert e.value.status == -1 and "limit" in str(e.value)


def test_noalloc_calls_leave_device_free_memory_unchanged(cuda):
    """The property the entry point exists for: after the first call on a
    device (which looks up the scratch array's address), a call takes no
    device memory.  The regular entry point's first render at this size grows
    the scene's scratch, which the same measurement sees."""
    import torch
    sd = scenes.cornell_box()
    sc = db.scene_from_dict(sd)
    p = db.render_params(sd["camera"], 512, 512, 8, max_depth=4, seed=5)
    stream = torch.cuda.current_stream().cuda_stream
    out = torch.zeros(512 * 512 * 3, dtype=torch.float32, device=cuda)
    ref = torch.zeros(512 * 512 * 3, dtype=torch.float32, device=cuda)
    sc.render_device_noalloc(p, out.data_ptr(), stream)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(2):
        sc.render_device_noalloc(p, out.data_ptr(), stream)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    got = out.cpu().numpy()
    # the regular entry point on the same scene: its scratch (slices x 512 x
    # 512 partial sums of 16 bytes) is allocated by its first call
    sc.render_device(p, ref.data_ptr(), stream)
    torch.cuda.synchronize()
    free2, _ = torch.cuda.mem_get_info()
    assert free2 < free1
    assert ptcheck.rel_rmse(got, ref.cpu().numpy()) < 1e-6
