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


def test_admission_respects_the_budget(rg):
    scenes = _scenes(rg, 4, seed0=200)
    srv = rg.RenderServer(hbm_budget_gb=0.05, max_resident_jobs=8)
    ids = [srv.submit(sc, 48, 48, 8, max_depth=4, seed=k) for k, sc in enumerate(scenes)]
    for jid in ids:
        srv.wait(jid)
    st = srv.stats()
    assert st["jobs_done"] == 4 and st["resident_peak"] == 1
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
