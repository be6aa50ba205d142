"""A render handle rebuilds its scene in place: rg_set_scene hands the previous
scene's device buffers and the BVH build's working arrays to the new scene
(they only grow; a scene with less than half the previous one's triangles
starts from fresh buffers).  A chain of scene changes on one handle must give
the same BVH and bit-identical images as a fresh handle per scene, across
growth, no growth, shrinking, textures and an environment map coming and going
(needs a B200)."""
import numpy as np
import pytest

from test_gpu_envmap import CAMERA, SPHERES, sky_scene

pytestmark = pytest.mark.gpu


def _settings(rg, width):
    return rg.RendererSettings(resolutionWidth=48, resolutionHeight=32, samples=8, maxDepth=5, seed=3,
                               bvhWidth=width)


def _render(r, sc):
    r.set_scene(sc)
    r.render()
    return r.get_hdr_result().copy(), r.stats()["bvh_nodes"]


@pytest.mark.parametrize("width", [8, 2])
def test_scene_chain_matches_fresh_handles(rg, tmp_path, width):
    sky = sky_scene(rg, tmp_path, SPHERES, CAMERA, intensity=0.8)
    chain = [rg.Scene.builtin(2, 3, [20000]), sky, rg.Scene.builtin(2, 5, [3000]), rg.Scene.builtin(2, 6, [2500]),
             rg.Scene.builtin(1, 1, None), sky, rg.Scene.builtin(2, 7, [1500])]
    tris = [sc.desc.num_triangles for sc in chain]
    adopted = [2 * b >= a for a, b in zip(tris, tris[1:])]
    # the chain takes over buffers that grow, that do not, and starts fresh
    assert any(adopted) and not all(adopted)
    assert any(b > a and ok for a, b, ok in zip(tris, tris[1:], adopted))
    assert any(b <= a and ok for a, b, ok in zip(tris, tris[1:], adopted))
    r = rg.RayRenderer(_settings(rg, width))
    try:
        for k, sc in enumerate(chain):
            img, nodes = _render(r, sc)
            fresh = rg.RayRenderer(_settings(rg, width))
            try:
                ref, ref_nodes = _render(fresh, sc)
            finally:
                fresh.close()
            assert nodes == ref_nodes, f"scene {k}: BVH node count"
            assert np.isfinite(img).all() and img[..., :3].max() > 0, f"scene {k}: empty image"
            np.testing.assert_array_equal(img, ref, err_msg=f"scene {k} ({tris[k]} triangles)")
    finally:
        r.close()
