"""HDR bloom and image output on the device (needs a B200): rg_bloom against
the oracle's restatement of RayRenderer::applyPostProcess
(rayrenderer.cpp:598-696), the render pipeline with post-processing on,
reapplyPostProcess, and the CLI's JPEG output.

The bloom kernels round every product on its own in the reference's loop
order, as the oracle does, so results agree to float rounding of the final
add (1e-5 relative); a bloom curve other than 1 goes through powf (1e-4).
"""
import os
import subprocess

import numpy as np
import pytest

import scenes
from test_gpu_parity import render_gpu
from test_image_io import hdr_with_spots

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "raygen-renderer_b200", "raygen")


@pytest.mark.parametrize("params,tol", [
    (dict(), 1e-5),
    (dict(threshold=0.5, strength=2.0, radius=0.05, size_aspect=0.3), 1e-5),
    (dict(threshold=0.0, radius=0.01, size_aspect=0.02), 1e-5),   # 1-3 pixel glow buffer
    (dict(radius=0.001), 1e-5),                                   # sigma below 0.5: no blur
    (dict(curve=2.5, threshold=2.0), 1e-4),
])
def test_bloom_matches_oracle(rg, orc, params, tol):
    img = hdr_with_spots(90, 160, seed=3)
    got = rg.bloom(img, **params)
    ref = orc.bloom(img, **params)
    np.testing.assert_allclose(got, ref, rtol=tol, atol=1e-6)


def test_render_with_post_process(rg, orc):
    sc = rg.Scene.builtin(1, 1)
    kw = dict(maxDepth=5, seed=4, bloomThreshold=0.8, bloomStrength=1.5)
    plain = render_gpu(rg, sc, 96, 64, 16, **kw)
    base = plain.get_hdr_result()
    plain.close()
    r = render_gpu(rg, sc, 96, 64, 16, enableRenderingPostProcess=True, **kw)
    bloomed = r.get_hdr_result()
    ref = orc.bloom(base, threshold=0.8, strength=1.5)
    np.testing.assert_allclose(bloomed, ref, rtol=1e-5, atol=1e-6)
    assert (bloomed[..., :3] - base[..., :3]).max() > 1e-3  # the light quad blooms
    np.testing.assert_allclose(r.get_render_result(), rg.tonemap(bloomed), rtol=1e-5, atol=1e-6)
    # reapplyPostProcess: new strength from the same pre-bloom image
    r.settings.bloomStrength = 3.0
    r.reapply_post_process()
    np.testing.assert_allclose(r.get_hdr_result(), orc.bloom(base, threshold=0.8, strength=3.0), rtol=1e-5,
                               atol=1e-6)
    r.settings.enableRenderingPostProcess = False
    r.reapply_post_process()
    np.testing.assert_array_equal(r.get_hdr_result(), base)
    r.close()


def test_cli_jpeg_output_with_bloom(tmp_path):
    Image = pytest.importorskip("PIL.Image")
    out = str(tmp_path / "room.jpg")
    res = subprocess.run([CLI, "render", "builtin:1", "-r", "80,60", "-s", "8", "-enpp", "true", "--max-depth", "5",
                          "-o", out], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stdout + res.stderr
    im = Image.open(out)
    assert im.format == "JPEG" and im.size == (80, 60)
    a = np.asarray(im.convert("RGB")).astype(np.float64)
    assert 5 < a.mean() < 250
