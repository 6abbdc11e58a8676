"""Error paths of the C ABI, driven without faulting a GPU.

* Allocation failures are injected on the host (dort_gpu_debug_fail_alloc):
  every allocation point of an entry point is made to fail in turn; each
  call must return DORT_ERR_OOM with a message, leak nothing, and leave the
  library working.  On the CPU the host builders' allocations are exercised
  through the host-check entry points (a failed host allocation is a
  std::bad_alloc that must not cross the C ABI); on the GPU, scene creation,
  renders and the wavefront's queues.
* The wavefront's bounded wave loop: a frame capped below the waves it needs
  stops on the device and its host entry returns DORT_ERR_TIMEOUT; the next
  frame on the same scene renders normally.
"""
import numpy as np
import pytest

import dort_b200 as db
from dort_b200 import scenes

OOM, TIMEOUT = -3, -4


@pytest.fixture(autouse=True)
def _injection_off():
    yield
    db.debug_fail_alloc(-1)


def _soup():
    return scenes.random_triangles(3000, seed=11)


def test_host_builder_allocation_failures_become_oom():
    verts, tris = _soup()
    rays = scenes.pinhole_rays(16, 16)
    ref, ref_tb, _ = db.host_check_raycast(verts, tris, rays)
    failures = 0
    for k in range(16):
        db.debug_fail_alloc(k)
        try:
            prim, tb, _ = db.host_check_raycast(verts, tris, rays)
        except db.DortError as e:
            assert e.status == OOM and "allocation" in str(e)
            failures += 1
            continue
        # the injected failure is past the call's allocation points
        assert np.array_equal(prim, ref)
        break
    else:
        pytest.fail("the host check never completed")
    assert failures >= 2
    db.debug_fail_alloc(-1)
    prim, tb, _ = db.host_check_raycast(verts, tris, rays)
    assert np.array_equal(prim, ref) and np.array_equal(tb, ref_tb)


def test_host_render_check_allocation_failure_becomes_oom():
    sd = scenes.cornell_box()
    p = db.render_params(sd["camera"], 8, 8, 1, max_depth=2)
    db.debug_fail_alloc(0)
    with pytest.raises(db.DortError) as e:
        db.host_check_render(sd, p)
    assert e.value.status == OOM
    img = db.host_check_render(sd, p)
    assert np.isfinite(img).all() and img.mean() > 0


@pytest.mark.gpu
def test_scene_create_allocation_failures_leak_nothing(cuda):
    import torch
    sd = scenes.cornell_box()
    verts, tris = _soup()
    p = db.render_params(sd["camera"], 32, 32, 4, max_depth=4)
    # warm: load the kernels and the allocator pools once
    db.Scene(verts, tris).close()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    failures = 0
    for bvh_build in ("device", "host"):
        for k in range(64):
            db.debug_fail_alloc(k)
            try:
                sc = db.Scene(verts, tris, bvh_build=bvh_build)
            except db.DortError as e:
                assert e.status == OOM, str(e)
                failures += 1
                continue
            db.debug_fail_alloc(-1)
            sc.close()
            break
        else:
            pytest.fail("scene creation never completed")
    db.debug_fail_alloc(-1)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert failures >= 4
    # every failed creation freed what it had taken (2 MiB of slack for the
    # driver's own bookkeeping)
    assert free1 >= free0 - (2 << 20)
    sc = db.scene_from_dict(sd)
    img, _ = sc.render(p)
    assert np.isfinite(img).all() and img.mean() > 0


@pytest.mark.gpu
def test_render_allocation_failures_then_recover(cuda):
    sd = scenes.cornell_box()
    p = db.render_params(sd["camera"], 48, 32, 8, max_depth=4, seed=3)
    ref_sc = db.scene_from_dict(sd)
    ref, _ = ref_sc.render(p)
    ref_wf, _ = ref_sc.render_wavefront(p)
    # the host-pointer entries allocate the scene's device image first; the
    # wavefront then allocates its queues
    for render, points in (("render", (0, 1)), ("render_wavefront", (0, 1))):
        sc = db.scene_from_dict(sd)
        for k in points:
            db.debug_fail_alloc(k)
            with pytest.raises(db.DortError) as e:
                getattr(sc, render)(p)
            assert e.value.status == OOM
            db.debug_fail_alloc(-1)
        img, _ = getattr(sc, render)(p)
        if render == "render":
            assert np.array_equal(img, ref)   # slice sums in a fixed order
        else:
            np.testing.assert_allclose(img, ref_wf, rtol=1e-5, atol=1e-6)
        sc.close()


@pytest.mark.gpu
def test_wavefront_wave_bound_reports_timeout_then_renders(cuda):
    sd = scenes.cornell_box()
    sc = db.scene_from_dict(sd)
    p = db.render_params(sd["camera"], 64, 64, 16, max_depth=8, seed=9)
    ref, st = sc.render_wavefront(p)
    assert st["waves"] > 4
    with pytest.raises(db.DortError) as e:
        sc.render_wavefront(p, {"max_waves": 3})
    assert e.value.status == TIMEOUT and "wave" in str(e.value)
    img, st2 = sc.render_wavefront(p)
    assert st2["waves"] == st["waves"]
    np.testing.assert_allclose(img, ref, rtol=1e-5, atol=1e-6)
    # a batch with the same cap stops too and says so in its stats
    b = db.Batch([(sc, p)], {"max_waves": 3})
    b.render()
    assert b.stats()["error"] == 1.0
    b.close()


@pytest.mark.gpu
def test_adjoint_allocation_failure_then_recover(cuda):
    """The adjoint's gradient buffers are the scene's (grown on demand): a
    failed allocation returns DORT_ERR_OOM and the next call computes the
    same gradients as a scene that never failed."""
    sd = scenes.adjoint_scene(n_tris=2000)
    p = db.render_params(sd["camera"], 24, 24, 4, max_depth=3, seed=2)
    alb, em = sd["tri_albedo"], sd["tri_emission"]
    ref_sc = db.scene_from_dict(sd)
    img = ref_sc.adjoint_forward(p, alb, em)
    _, g = db.loss_l2(img, np.zeros_like(img))
    ref_a, ref_e = ref_sc.adjoint_backward(p, g, alb, em)
    sc = db.scene_from_dict(sd)
    sc.adjoint_forward(p, alb, em)          # the per-triangle buffers exist now
    db.debug_fail_alloc(0)
    with pytest.raises(db.DortError) as e:
        sc.adjoint_backward(p, g, alb, em)
    assert e.value.status == OOM
    db.debug_fail_alloc(-1)
    da, de = sc.adjoint_backward(p, g, alb, em)
    # float atomics add in any order: equal to rounding, in norm
    for got, want in ((da, ref_a), (de, ref_e)):
        assert np.abs(want).sum() > 0
        assert np.linalg.norm(got - want) <= 1e-4 * np.linalg.norm(want)
