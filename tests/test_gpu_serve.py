"""Batched / served rendering through the job server (needs a B200).

A job's image must not depend on the mix it was rendered in: the path RNG is
keyed by (job seed, pixel, sample).  Only the order of the per-pixel float
accumulation can differ between mixes, so images agree to 1e-4 relative.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _scenes(rg, n, seed0=100):
    out = []
    for k in range(n):
        out.append(rg.Scene.builtin(4, seed0 + k, [2000 + 3000 * k, 1 + k % 5]))
    return out


def test_server_job_matches_single_renderer(rg):
    sc = rg.Scene.builtin(1, 1)
    srv = rg.RenderServer(max_resident_jobs=8)
    j = srv.submit(sc, 64, 48, 32, max_depth=5, seed=3)
    srv.wait(j)
    a = srv.result(j)
    r = rg.RayRenderer(rg.RendererSettings(resolutionWidth=64, resolutionHeight=48, samples=32, maxDepth=5, seed=3))
    r.set_scene(sc)
    r.render()
    b = r.get_hdr_result()
    np.testing.assert_allclose(a, b, rtol=1e-4, atol=1e-6)
    srv.close()


def test_result_is_independent_of_the_mix(rg):
    scenes = _scenes(rg, 6)
    alone = rg.RenderServer(max_resident_jobs=4)
    j = alone.submit(scenes[0], 80, 60, 24, max_depth=6, seed=7)
    alone.wait(j)
    ref = alone.result(j)
    alone.close()
    mix = rg.RenderServer(max_resident_jobs=16, paths_per_wave=1 << 16)
    ids = []
    for k, sc in enumerate(scenes):
        if k == 0:
            ids.append(mix.submit(sc, 80, 60, 24, max_depth=6, seed=7))
        else:
            ids.append(mix.submit(sc, 80 + 16 * k, 60 + 8 * k, 8 + 4 * k, max_depth=4 + k, seed=50 + k))
    for jid in ids:
        mix.wait(jid)
    got = mix.result(ids[0])
    np.testing.assert_allclose(got, ref, rtol=1e-4, atol=1e-6)
    st = mix.stats()
    assert st["jobs_done"] == len(scenes) and st["resident_peak"] >= 2 and st["waves"] > 1
    mix.close()


def test_wave_fill_gives_the_same_images(rg):
    """Filling each wave from as few jobs as possible changes which jobs share a
    wave, not the images."""
    scenes = _scenes(rg, 5, seed0=300)
    out = {}
    for fill in (0, 1):
        srv = rg.RenderServer(max_resident_jobs=8, paths_per_wave=1 << 15, wave_fill=fill)
        ids = [srv.submit(sc, 72 + 8 * k, 40 + 8 * k, 6 + 3 * k, max_depth=5, seed=90 + k) for k, sc in enumerate(scenes)]
        for jid in ids:
            srv.wait(jid)
        out[fill] = [srv.result(jid) for jid in ids]
        assert srv.stats()["waves"] > len(scenes)
        srv.close()
    for a, b in zip(out[0], out[1]):
        np.testing.assert_allclose(a, b, rtol=1e-4, atol=1e-6)


def test_admission_respects_the_budget(rg):
    """Each job reserves its admission estimate (about 66-70 MB here, most of it
    for the BVH build) until it is resident, then holds its measured footprint
    (a few MB): with a 75 MB budget no two jobs are admitted at once, at most
    two are resident together, and the budget is never exceeded."""
    scenes = _scenes(rg, 4, seed0=200)
    budget_gb = 0.07
    srv = rg.RenderServer(hbm_budget_gb=budget_gb, max_resident_jobs=8)
    ids = [srv.submit(sc, 48, 48, 8, max_depth=4, seed=k) for k, sc in enumerate(scenes)]
    for jid in ids:
        srv.wait(jid)
    st = srv.stats()
    assert st["jobs_done"] == 4 and 1 <= st["resident_peak"] <= 2
    assert 0 < st["bytes_peak"] <= budget_gb * (1 << 30)
    assert st["p99_ms"] >= st["p50_ms"] > 0
    for jid in ids:
        assert np.isfinite(srv.result(jid)).all()
    srv.close()


def test_progressive_snapshot(rg):
    sc = rg.Scene.builtin(2, 3, [20000])
    srv = rg.RenderServer(max_resident_jobs=2, paths_per_wave=1 << 15)
    j = srv.submit(sc, 256, 144, 64, max_depth=6, seed=1)
    snap = srv.snapshot(j)
    assert snap.shape == (144, 256, 4) and np.isfinite(snap).all()
    srv.wait(j)
    final = srv.result(j)
    assert final[..., :3].mean() > 0
    srv.close()


def test_autotuner_config_is_valid_and_keeps_results(rg):
    scenes = _scenes(rg, 4, seed0=300)
    probe = [(sc, 48, 48, 4, 5, 10 + k) for k, sc in enumerate(scenes)]
    t = rg.RenderServer.autotune(probe, max_resident_jobs=8)
    assert t["paths_per_wave"] in {1 << p for p in range(20, 27)}  # the autotuner's candidates, 1 Mi .. 64 Mi
    assert t["shade_blocks_per_sm"] in {0, 2, 4, 8, 16} and t["trace_blocks_per_sm"] in {0, 2, 4, 6}
    assert t["probe_ms"] > 0
    out = []
    for kw in ({}, {k: t[k] for k in ("paths_per_wave", "shade_blocks_per_sm", "trace_blocks_per_sm")}):
        srv = rg.RenderServer(max_resident_jobs=8, **kw)
        j = srv.submit(scenes[0], 64, 48, 8, max_depth=5, seed=3)
        srv.wait(j)
        out.append(srv.result(j))
        srv.close()
    # the path RNG is keyed by (seed, pixel, sample): wave size and launch widths do not change the image
    np.testing.assert_allclose(out[0], out[1], rtol=1e-4, atol=1e-6)


def test_job_larger_than_the_budget_is_refused(rg):
    small = rg.Scene.builtin(1, 1)
    big = rg.Scene.builtin(4, 5, [1000000, 4])  # about 0.5 GB to admit
    srv = rg.RenderServer(hbm_budget_gb=0.2, max_resident_jobs=4)
    with pytest.raises(rg.RayGenError) as e:
        srv.submit(big, 64, 64, 4, max_depth=4, seed=1)
    assert e.value.code == rg.RG_ERR_OUT_OF_MEMORY
    j = srv.submit(small, 32, 32, 4, max_depth=4, seed=1)  # the server goes on serving
    srv.wait(j)
    assert np.isfinite(srv.result(j)).all()
    srv.close()


def test_cancel_queued_and_resident_jobs_frees_their_slots(rg):
    """rg_server_cancel: a resident job is dropped between waves (its slot and
    memory are freed, waiters see RG_ERR_CANCELLED), a queued job leaves the
    queue, and the other jobs complete with the images they have alone."""
    sc = rg.Scene.builtin(2, 3, [20000])
    small = rg.Scene.builtin(1, 1)
    srv = rg.RenderServer(max_resident_jobs=1, paths_per_wave=1 << 14)
    long_job = srv.submit(sc, 256, 256, 256, max_depth=8, seed=1)   # many waves of 16 Ki paths
    queued = srv.submit(small, 32, 32, 8, max_depth=5, seed=2)      # waits for the only slot
    after = srv.submit(small, 40, 30, 8, max_depth=5, seed=3)
    srv.snapshot(long_job)                                         # resident and rendering
    assert srv.status(long_job)["state"] == rg.RG_JOB_RESIDENT
    assert srv.status(queued)["state"] == rg.RG_JOB_QUEUED
    assert srv.cancel(queued) == rg.RG_OK
    assert srv.cancel(long_job) == rg.RG_OK
    for jid in (long_job, queued):
        with pytest.raises(rg.RayGenError) as e:
            srv.wait(jid, 60000.0)
        assert e.value.code == rg.RG_ERR_CANCELLED
        st = srv.status(jid)
        assert st["state"] == rg.RG_JOB_FAILED and st["error"] == rg.RG_ERR_CANCELLED
    assert srv.status(long_job)["samples_issued"] < 256 * 256 * 256
    srv.wait(after)  # the freed slot admits the next job
    assert srv.cancel(after) == rg.RG_ERR_BUSY  # finished: nothing left to cancel
    got = srv.result(after)
    r = rg.RayRenderer(rg.RendererSettings(resolutionWidth=40, resolutionHeight=30, samples=8, maxDepth=5, seed=3))
    r.set_scene(small)
    r.render()
    np.testing.assert_allclose(got, r.get_hdr_result(), rtol=1e-4, atol=1e-6)
    r.close()
    srv.close()


def test_resident_scene_is_built_once_and_renders_like_an_uploaded_one(rg):
    """rg_server_add_scene keeps the BVH and tables on the device: jobs on it
    skip the upload and build, render the image an uploaded scene gives, count
    the scene once against the budget, and the scene outlives its removal until
    its last job ends."""
    sc = rg.Scene.builtin(2, 6, [20000])
    srv = rg.RenderServer(max_resident_jobs=8)
    j0 = srv.submit(sc, 96, 64, 16, max_depth=6, seed=4)  # uploaded with the job
    srv.wait(j0)
    want = srv.result(j0)
    sid = srv.add_scene(sc)
    bytes_scene = srv.stats()["bytes_peak"]
    assert bytes_scene > 0
    ids = [srv.submit(sid, 96, 64, 16, max_depth=6, seed=4) for _ in range(3)]
    ids.append(srv.submit(sid, 64, 48, 8, max_depth=5, seed=9))
    srv.remove_scene(sid)  # jobs still queued on it keep it alive
    for j in ids:
        srv.wait(j)
    for j in ids[:3]:
        np.testing.assert_allclose(srv.result(j), want, rtol=1e-4, atol=1e-6)
    assert np.isfinite(srv.result(ids[3])).all()
    with pytest.raises(rg.RayGenError) as e:  # the id is gone
        srv.submit(sid, 32, 32, 4)
    assert e.value.code == rg.RG_ERR_INVALID_ARGUMENT
    srv.close()
