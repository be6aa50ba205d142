"""Failure detection on the device, without a GPU fault (needs a B200).

Each failure is made by lowering a bound of the library, never by a bad
address, a trap or an endless loop:
* traversal: with the node-step bound at 1 every traversal of a scene deeper
  than one node stops, raises the device error flag and the render / ray
  query returns RG_ERR_DEVICE_STATUS with the flag in the stats; with the
  bound restored the same handle renders the exact image of a fresh renderer;
* tensor cores: with the strip pipeline's barrier polls at 1 the learned
  denoiser's convolution gives up its waits, drains every issued copy and MMA
  under the built-in bound, frees its tensor memory and reports
  RG_ERR_DEVICE_STATUS; restored, the next call returns the exact result.
Host-side failures (cancel, budget refusal, busy handle) are covered in
test_gpu_async.py and test_gpu_serve.py.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ERR_TRAVERSAL_STEPS = 1


def test_traversal_step_bound_raises_device_status(rg):
    lib = rg.load_library()
    sc = rg.Scene.builtin(2, 4, [2000])
    st = rg.RendererSettings(resolutionWidth=32, resolutionHeight=24, samples=2, maxDepth=4, seed=2)
    r = rg.RayRenderer(st)
    r.set_scene(sc)
    rays = np.zeros((64, 6), np.float32)
    rays[:, 5] = -1.0
    rays[:, 3] = np.linspace(-0.4, 0.4, 64)
    try:
        assert lib.rg_debug_set_traversal_step_cap(1) == 0
        with pytest.raises(rg.RayGenError) as e:
            r.render()
        assert e.value.code == rg.RG_ERR_DEVICE_STATUS
        assert r.stats()["device_error"] == ERR_TRAVERSAL_STEPS
        with pytest.raises(rg.RayGenError) as e:
            r.trace_closest(rays)
        assert e.value.code == rg.RG_ERR_DEVICE_STATUS
    finally:
        assert lib.rg_debug_set_traversal_step_cap(0) == 0
    r.render()
    assert r.stats()["device_error"] == 0
    fresh = rg.RayRenderer(st)
    fresh.set_scene(sc)
    fresh.render()
    np.testing.assert_array_equal(r.get_hdr_result(), fresh.get_hdr_result())
    fresh.close()
    r.close()
    sc.close()


def test_tensor_core_wait_limit_reports_and_recovers(rg):
    lib = rg.load_library()
    rng = np.random.default_rng(4)
    H, W = 96, 160
    noisy = rng.random((H, W, 3)).astype(np.float32)
    normal = rng.random((H, W, 3)).astype(np.float32)
    albedo = rng.random((H, W, 3)).astype(np.float32)
    depth = rng.random((H, W)).astype(np.float32)
    d = rg.Denoiser.pretrained()
    want = d.apply(noisy, normal, albedo, depth)
    try:
        assert lib.rg_debug_set_tc_wait_limit(1) == 0
        with pytest.raises(rg.RayGenError) as e:
            d.apply(noisy, normal, albedo, depth)
        assert e.value.code == rg.RG_ERR_DEVICE_STATUS
        assert b"timed out" in lib.rg_last_error()
    finally:
        assert lib.rg_debug_set_tc_wait_limit(0) == 0
    np.testing.assert_array_equal(d.apply(noisy, normal, albedo, depth), want)
    d.close()
