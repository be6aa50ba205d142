"""Equirectangular environment lighting on the device vs the CPU oracle
(needs a B200): eye and path misses, environment NEE from diffuse, glossy and
medium vertices (shadow queue C), the simple shaders' misses, and the server's
multi-job path.  Tolerances as test_gpu_parity (Monte-Carlo z-scores)."""
import json

import numpy as np
import pytest

import scenes
from test_gpu_parity import check_z, image_parity, render_gpu

pytestmark = pytest.mark.gpu


def sky_scene(rg, tmp_path, objects, camera, intensity=1.0, rotation=0.0, medium=None, img=None, name="sky.json"):
    scenes.write_hdr(tmp_path / "sky.hdr", scenes.sky_image(128, 64, seed=11) if img is None else img)
    doc = {"mainCamera": camera, "envmap": {"texture": "sky.hdr", "intensity": intensity, "rotation": rotation}}
    if medium:
        doc["medium"] = medium
    doc.update(objects)
    (tmp_path / name).write_text(json.dumps(doc))
    return rg.Scene.from_json(str(tmp_path / name))


SPHERES = {
    "floor": {"location": [0, -1, 0], "scale": [40, 1, 40], "mesh": {"type": "plane"}, "mat": {"color": [0.6, 0.6, 0.6]}},
    "diffuse": {"location": [-2.2, 0, 0], "mesh": {"type": "sphere", "radius": 0.9, "stacks": 20, "slices": 40},
                "mat": {"color": [0.9, 0.35, 0.25]}},
    "glass": {"location": [0, 0, 0], "mesh": {"type": "sphere", "radius": 0.9, "stacks": 20, "slices": 40},
              "mat": {"refraction": 1, "refractionRatio": 1.5, "roughness": 0}},
    "metal": {"location": [2.2, 0, 0], "mesh": {"type": "sphere", "radius": 0.9, "stacks": 20, "slices": 40},
              "mat": {"color": [0.9, 0.9, 0.95], "glossy": 1, "metallic": 1, "roughness": 0.3}},
    "mixed": {"location": [0, 0.3, -2.5], "scale": [1.2, 1.2, 1.2], "mesh": {"type": "cube"},
              "mat": {"color": [0.3, 0.6, 0.9], "glossy": 0.5, "roughness": 0.15}},
}
CAMERA = {"location": [0, 1.0, 6.0], "angle": [-8, 0, 0], "fieldOfView": 50}


def test_env_white_furnace_on_device(rg, tmp_path):
    img = np.full((8, 16, 3), 0.8, np.float32)
    L = float(scenes.rgbe_decode(scenes.rgbe_encode(img))[0, 0, 0])  # 0.8 as stored: 204/256
    objects = {"floor": {"scale": [1000, 1, 1000], "mesh": {"type": "plane"}, "mat": {"color": [0.5, 0.5, 0.5]}}}
    cam = {"location": [0, 1, 0], "angle": [-90, 0, 0], "fieldOfView": 40}
    sc = sky_scene(rg, tmp_path, objects, cam, img=img)
    r = render_gpu(rg, sc, 64, 64, 64, maxDepth=8, seed=2)
    m = r.get_hdr_result()[..., :3]
    r.close()
    assert m.mean() == pytest.approx(0.5 * L, rel=0.005)


def test_env_image_parity(rg, orc, tmp_path):
    sc = sky_scene(rg, tmp_path, SPHERES, CAMERA, intensity=1.3, rotation=35)
    z, g, m, stats = image_parity(rg, orc, sc, 64, 40, 128, maxDepth=8, rrDepth=3, seed=6)
    check_z(z, g, m, "environment-lit spheres", tail=0.01)
    assert stats["shadow_rays"] > 0


def test_env_medium_image_parity(rg, orc, tmp_path):
    medium = {"sigma_a": [0.01, 0.01, 0.01], "sigma_s": [0.05, 0.05, 0.05], "g": 0.4}
    sc = sky_scene(rg, tmp_path, SPHERES, CAMERA, medium=medium, name="fog.json")
    z, g, m, _ = image_parity(rg, orc, sc, 48, 30, 128, maxDepth=8, rrDepth=3, seed=7)
    check_z(z, g, m, "environment + global medium", tail=0.01)


@pytest.mark.parametrize("shader", [2, 0])
def test_env_simple_shaders(rg, orc, tmp_path, shader):
    sc = sky_scene(rg, tmp_path, SPHERES, CAMERA, rotation=-60)
    z, g, m, _ = image_parity(rg, orc, sc, 48, 30, 16, maxDepth=5, seed=3, shaderProvider=shader)
    check_z(z, g, m, f"shader {shader} with environment", tail=0.01)


def test_env_server_matches_renderer(rg, tmp_path):
    sc = sky_scene(rg, tmp_path, SPHERES, CAMERA, intensity=0.8)
    srv = rg.RenderServer(max_resident_jobs=4)
    j = srv.submit(sc, 64, 40, 16, max_depth=6, seed=4)
    srv.wait(j)
    a = srv.result(j)
    srv.close()
    r = render_gpu(rg, sc, 64, 40, 16, maxDepth=6, seed=4)
    b = r.get_hdr_result()
    r.close()
    np.testing.assert_allclose(a, b, rtol=1e-4, atol=1e-6)


def _cube(tmp_path, colours, sun=None, size=16):
    from test_envmap import cube_dir
    return cube_dir(tmp_path, colours=colours, size=size, sun=sun)


def test_cubemap_white_furnace_on_device(rg, tmp_path):
    _cube(tmp_path, [(204, 204, 204)] * 6)
    doc = {"mainCamera": {"location": [0, 1, 0], "angle": [-90, 0, 0], "fieldOfView": 40},
           "envmap": {"cubemap": "cube", "ext": "png"},
           "floor": {"scale": [1000, 1, 1000], "mesh": {"type": "plane"}, "mat": {"color": [0.5, 0.5, 0.5]}}}
    (tmp_path / "f.json").write_text(json.dumps(doc))
    r = render_gpu(rg, rg.Scene.from_json(str(tmp_path / "f.json")), 64, 64, 64, maxDepth=8, seed=2)
    m = r.get_hdr_result()[..., :3]
    r.close()
    L = ((204 / 255 + 0.055) / 1.055) ** 2.4
    assert m.mean() == pytest.approx(0.5 * L, rel=0.005)


def test_cubemap_image_parity(rg, orc, tmp_path):
    from test_envmap import FACE_COLOURS
    _cube(tmp_path, FACE_COLOURS, sun=(2, 5, 9))
    doc = {"mainCamera": CAMERA, "envmap": {"cubemap": "cube", "ext": "png", "intensity": 1.2, "rotation": 40}}
    doc.update(SPHERES)
    (tmp_path / "cube.json").write_text(json.dumps(doc))
    sc = rg.Scene.from_json(str(tmp_path / "cube.json"))
    assert sc.desc.envmap_cube == 1
    z, g, m, stats = image_parity(rg, orc, sc, 64, 40, 128, maxDepth=8, rrDepth=3, seed=6)
    check_z(z, g, m, "cubemap-lit spheres", tail=0.01)
