"""The renderer's asynchronous boundary and its progress / cancel contract
(rg_render_async, rg_poll, rg_wait, rg_set_progress_cb, rg_cancel), through
the C ABI (needs a B200).

The reference renders on worker threads, calls progressCallback from them
(rayrenderer.cpp:804-806) and polls cancelRequested per tile
(rayrenderer.h:427, rayrenderer.cpp:766).  Here waves are paced one behind
the device, so progress counts completed waves and a cancel ends the render
within about one wave.
"""
import threading
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def many_waves(rg, W=256, H=256, spp=256):
    """A render of many small waves: 16 Ki paths per wave, 1024 waves."""
    st = rg.RendererSettings(resolutionWidth=W, resolutionHeight=H, samples=spp, maxDepth=6, seed=5)
    st.pathsPerWave = 1 << 14
    return st


def test_async_render_matches_blocking_render_and_reports_progress(rg):
    sc = rg.Scene.builtin(2, 2, [20000])
    st = rg.RendererSettings(resolutionWidth=96, resolutionHeight=64, samples=32, maxDepth=6, seed=5)
    st.pathsPerWave = 1 << 14
    ref = rg.RayRenderer(st)
    ref.set_scene(sc)
    ref.render()
    want = ref.get_hdr_result()
    ref.close()

    r = rg.RayRenderer(st)
    r.set_scene(sc)
    seen, threads = [], set()
    r.progressCallback = lambda p: (seen.append(p), threads.add(threading.get_ident()))
    job = r.render_async()
    polled = []
    while True:
        done, pr = job.poll()
        polled.append(pr)
        if done:
            break
        time.sleep(0.002)
    assert job.wait(1000.0)
    job.close()
    np.testing.assert_array_equal(r.get_hdr_result(), want)
    # progress: from one host thread that is not the caller's, non-decreasing, ending at 1
    assert len(seen) >= 3 and seen[-1] == 1.0
    assert all(b >= a for a, b in zip(seen, seen[1:]))
    assert threads and threading.get_ident() not in threads and len(threads) == 1
    assert all(b >= a for a, b in zip(polled, polled[1:])) and polled[-1] == 1.0
    r.close()
    sc.close()


def test_one_render_in_flight_per_handle(rg):
    sc = rg.Scene.builtin(1, 1)
    r = rg.RayRenderer(many_waves(rg))
    r.set_scene(sc)
    job = r.render_async()
    with pytest.raises(rg.RayGenError) as e:
        r.render_async()
    assert e.value.code == rg.RG_ERR_BUSY
    # the blocking entry point and the scene / settings updates refuse too
    assert r._lib.rg_render(r._h) == rg.RG_ERR_BUSY
    assert r._lib.rg_set_scene(r._h, sc.ptr) == rg.RG_ERR_BUSY
    r.cancel()
    with pytest.raises(rg.RayGenError):
        job.wait()
    job.close()
    r.close()
    sc.close()


def test_cancel_mid_render_then_render_again(rg):
    sc = rg.Scene.builtin(2, 2, [20000])
    st = many_waves(rg)
    r = rg.RayRenderer(st)
    r.set_scene(sc)
    job = r.render_async()
    # wait until a few waves have completed, then cancel
    t0 = time.time()
    while job.poll()[1] < 0.02 and time.time() - t0 < 60:
        time.sleep(0.001)
    pr_at_cancel = job.poll()[1]
    assert 0.0 < pr_at_cancel < 0.5
    t_cancel = time.time()
    r.cancel()
    with pytest.raises(rg.RayGenError) as e:
        job.wait(60000.0)
    assert e.value.code == rg.RG_ERR_CANCELLED
    job.close()
    cancel_s = time.time() - t_cancel
    # a wave of 16 Ki paths takes well under 50 ms; the render stopped long before its end
    assert cancel_s < 2.0
    # the handle renders again, and the result equals a fresh renderer's
    small = rg.RendererSettings(resolutionWidth=64, resolutionHeight=48, samples=16, maxDepth=6, seed=9)
    r.settings = small
    r.render()
    got = r.get_hdr_result()
    f = rg.RayRenderer(small)
    f.set_scene(sc)
    f.render()
    np.testing.assert_array_equal(got, f.get_hdr_result())
    f.close()
    r.close()
    sc.close()


def test_blocking_render_cancelled_from_another_thread(rg):
    sc = rg.Scene.builtin(1, 1)
    r = rg.RayRenderer(many_waves(rg))
    r.set_scene(sc)
    fired = []

    def cancel_after_progress(p):
        if p > 0.01 and not fired:
            fired.append(p)
            threading.Thread(target=r.cancel).start()

    r.progressCallback = cancel_after_progress
    with pytest.raises(rg.RayGenError) as e:
        r.render()
    assert e.value.code == rg.RG_ERR_CANCELLED and fired
    r.progressCallback = None
    r.settings = rg.RendererSettings(resolutionWidth=32, resolutionHeight=32, samples=4, maxDepth=5, seed=1)
    r.render()
    assert np.isfinite(r.get_hdr_result()).all()
    r.close()
    sc.close()
