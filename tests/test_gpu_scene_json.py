"""Scenes loaded from the reference JSON schema, rendered on the device and
checked against the CPU oracle; the `raygen render <scene.json>` command line
on the same file (needs a B200)."""
import json
import os
import subprocess

import numpy as np
import pytest

import scenes
from test_gpu_parity import check_z, image_parity, render_gpu

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "raygen-renderer_b200", "raygen")

# primitives, a mesh-less emitter (point light), a glass sphere holding a
# medium, a global medium, a named material and a multi-axis rotation
MIXED = json.dumps({
    "mainCamera": {"location": [0, 1.2, 5], "angle": [-10, 0, 0], "fieldOfView": 55},
    "medium": {"sigma_a": [0.01, 0.01, 0.01], "sigma_s": [0.03, 0.03, 0.03], "g": 0.2},
    "_materials": {"metal": {"color": "#d0a060", "glossy": 1, "metallic": 1, "roughness": 0.25}},
    "floor": {"location": [0, -1, 0], "scale": [12, 1, 12], "mesh": {"type": "plane"}},
    "bulb": {"location": [0, 3, 1], "mat": {"emission": 20, "color": [1, 0.9, 0.8]}},
    "panel": {"location": [-2, 2.5, -1], "angle": [150, 0, 20], "scale": [1.5, 1, 1.5],
              "mesh": {"type": "plane"}, "mat": {"emission": 6}},
    "ball": {"location": [-0.9, 0, 0], "mesh": {"type": "sphere", "radius": 0.9, "stacks": 24, "slices": 48},
             "mat": {"refraction": 1, "refractionRatio": 1.5, "roughness": 0},
             "medium": {"sigma_a": [0.6, 0.2, 0.05], "sigma_s": [0.2, 0.2, 0.2]}},
    "cone": {"location": [1.1, -0.2, 0], "angle": [-90, 30, 0], "scale": [1.2, 1.2, 1.6],
             "mesh": {"type": "cone", "radiusStart": 0.6, "radiusEnd": 0.1, "slices": 40}, "mat": "metal"},
})


def scene_file(tmp_path, text, name):
    p = tmp_path / name
    p.write_text(text)
    return str(p)


def test_json_room_image_parity(rg, orc, tmp_path):
    sc = rg.Scene.from_json(scene_file(tmp_path, scenes.JSON_ROOM, "room.json"))
    z, g, m, stats = image_parity(rg, orc, sc, 64, 48, 64, maxDepth=6, rrDepth=3, seed=3)
    check_z(z, g, m, "json room")
    assert stats["kernel_launches"] > 0


def test_json_mixed_features_image_parity(rg, orc, tmp_path):
    sc = rg.Scene.from_json(scene_file(tmp_path, MIXED, "mixed.json"))
    d = sc.desc
    assert d.num_point_lights == 1 and d.num_media == 2 and d.global_medium == 0
    z, g, m, _ = image_parity(rg, orc, sc, 48, 36, 128, maxDepth=8, rrDepth=3, seed=5)
    check_z(z, g, m, "json primitives + point light + media", tail=0.01)


def read_pfm(path):
    with open(path, "rb") as f:
        assert f.readline().strip() == b"PF"
        w, h = map(int, f.readline().split())
        scale = float(f.readline())
        data = np.frombuffer(f.read(), dtype="<f4" if scale < 0 else ">f4")
    return data.reshape(h, w, 3)[::-1]


def test_cli_renders_json_scene(rg, tmp_path):
    path = scene_file(tmp_path, scenes.JSON_ROOM, "room.json")
    out = str(tmp_path / "room.pfm")
    res = subprocess.run([CLI, "render", path, "-r", "64,48", "-s", "16", "--max-depth", "6", "--seed", "7",
                          "-o", out], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stdout + res.stderr
    img = read_pfm(out)
    # the same settings through the library: identical image (the tracer is deterministic)
    r = render_gpu(rg, rg.Scene.from_json(path), 64, 48, 16, maxDepth=6, seed=7)
    ref = r.get_hdr_result()[..., :3]
    r.close()
    assert img.shape == ref.shape
    np.testing.assert_allclose(img, ref, rtol=0, atol=0)
    assert img.mean() > 0.01


def test_json_textured_materials_image_parity(rg, orc, tmp_path):
    """'tex' textures from a JPEG (4:2:0, restart intervals) and a PNG, sampled
    with the sRGB decode (Texture::sample, texture.cpp:210-241)."""
    import image_codecs as ic
    y, x = np.mgrid[0:64, 0:96]
    checker = np.where(((x // 12) + (y // 12)) % 2 == 0, 220, 40)
    img = np.stack([checker, 0.6 * checker + 40, 255 - checker], axis=-1).astype(np.float64)
    ic.encode_jpeg(str(tmp_path / "wood.jpg"), img, sampling=((2, 2), (1, 1), (1, 1)), restart=4)
    stripes = np.stack([np.where((x // 8) % 2 == 0, 250, 20)[:32, :32]] * 3, axis=-1)
    ic.write_png(str(tmp_path / "stripes.png"), stripes.astype(np.int64), 2, 8)
    doc = {
        "mainCamera": {"location": [0, 1.5, 5], "angle": [-15, 0, 0], "fieldOfView": 50},
        "lamp": {"location": [0, 4, 0], "angle": [180, 0, 0], "scale": [2, 1, 2], "mesh": {"type": "plane"},
                 "mat": {"color": [1, 1, 1], "emission": 8}},
        "floor": {"location": [0, -1, 0], "scale": [8, 1, 8], "mesh": {"type": "plane"},
                  "mat": {"tex": "wood.jpg", "texTiling": [2, 2]}},
        "box": {"location": [0.8, -0.3, 0], "angle": [0, 30, 0], "scale": [1.2, 1.4, 1.2], "mesh": {"type": "cube"},
                "mat": {"tex": "stripes.png", "color": [0.9, 0.8, 0.7]}},
        "ball": {"location": [-1.3, -0.2, 0.5], "mesh": {"type": "sphere", "radius": 0.8, "stacks": 16, "slices": 32},
                 "mat": {"tex": "wood.jpg", "glossy": 1, "roughness": 0.3}},
    }
    (tmp_path / "tex.json").write_text(json.dumps(doc))
    sc = rg.Scene.from_json(str(tmp_path / "tex.json"))
    assert sc.desc.num_textures == 2
    z, g, m, stats = image_parity(rg, orc, sc, 64, 40, 64, maxDepth=6, rrDepth=3, seed=3)
    check_z(z, g, m, "textured JSON scene", tail=0.01)
    # the textures really are sampled: the same scene without them renders differently
    doc2 = json.loads(json.dumps(doc))
    for k in ("floor", "box", "ball"):
        doc2[k]["mat"].pop("tex")
    (tmp_path / "flat.json").write_text(json.dumps(doc2))
    r = render_gpu(rg, rg.Scene.from_json(str(tmp_path / "flat.json")), 64, 40, 64, maxDepth=6, rrDepth=3, seed=3)
    flat = r.get_hdr_result()[..., :3]
    r.close()
    assert np.abs(flat - g).mean() > 0.02 * max(g.mean(), 1e-3)
