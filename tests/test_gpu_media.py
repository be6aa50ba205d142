"""Procedural participating media on the device vs the CPU oracle (needs a
B200): the camera-space medium fields (density, cone / path emission, index of
refraction, heat-haze bending) through rg_medium_eval / rg_medium_bend, and
image parity of JSON scenes with an fBm cloud (delta tracking), a jet flame
(cone emission, volume-light NEE from diffuse and glossy vertices and from
scatter events), a turbulent absorbing flame, a path-tube emitter, a heat-haze
volume in front of an environment map and a constant-glow volume light.
Tolerances as test_gpu_parity (Monte-Carlo z-scores)."""
import json

import numpy as np
import pytest

import scenes
from test_gpu_parity import check_z, image_parity, render_gpu

pytestmark = pytest.mark.gpu

CAMERA = {"location": [0, 1.0, 6.0], "angle": [-8, 0, 0], "fieldOfView": 45}
ROOM = {
    "floor": {"location": [0, -1, 0], "scale": [20, 1, 20], "mesh": {"type": "plane"}, "mat": {"color": [0.6, 0.6, 0.6]}},
    "back": {"location": [0, 0, -4], "angle": [90, 0, 0], "scale": [20, 1, 20], "mesh": {"type": "plane"},
             "mat": {"color": [0.5, 0.5, 0.55]}},
    "ball": {"location": [-2.0, -0.3, 0.5], "mesh": {"type": "sphere", "radius": 0.7, "stacks": 16, "slices": 32},
             "mat": {"color": [0.9, 0.9, 0.95], "glossy": 1, "metallic": 1, "roughness": 0.35}},
}
LAMP = {"lamp": {"location": [0, 4, 0], "angle": [180, 0, 0], "scale": [2, 1, 2], "mesh": {"type": "plane"},
                 "mat": {"color": [1, 1, 1], "emission": 6}}}
FLAME = {"emissionMode": "cone", "coneOrigin": [0.6, 0.0, 0.0], "coneAxis": [-1, 0, 0], "coneLength": 1.6,
         "coneRadius": 0.35, "coneInner": [4, 6, 12], "coneOuter": [10, 3, 0.4], "coneIntensity": 25.0,
         "conePeakAxial": 0.18, "conePeakSharpness": 4.0, "coneEmissionSamples": 8}


def json_scene(rg, tmp_path, objects, name, medium=None, envmap=False):
    doc = {"mainCamera": CAMERA}
    if envmap:
        scenes.write_hdr(tmp_path / "sky.hdr", scenes.sky_image(128, 64, seed=5))
        doc["envmap"] = {"texture": "sky.hdr", "intensity": 1.0}
    if medium:
        doc["medium"] = medium
    doc.update(objects)
    (tmp_path / name).write_text(json.dumps(doc))
    return rg.Scene.from_json(str(tmp_path / name))


def box(location, scale, medium, **mat):
    return {"location": location, "scale": scale, "mesh": {"type": "cube"},
            "mat": dict({"transparency": 1.0}, **mat), "medium": medium}


def field_scene(rg, tmp_path):
    media = {
        "cloud": box([0, 0.5, 0], [2.4, 1.6, 2.4],
                     {"sigma_a": [0.05] * 3, "sigma_s": [2.0] * 3, "densityField": "fbm", "noiseFrequency": 1.6,
                      "noiseOctaves": 4, "noiseAmplitude": 1.4, "noiseBias": -0.25, "noiseOffset": [0.2, 0, 0]}),
        "flame": box([1.5, 0.4, 0], [1.6, 0.8, 0.8], dict(FLAME, coneFollowObject=True, densityField="fbm",
                                                          noiseFrequency=4.0, noiseAmplitude=1.6, noiseBias=-0.3)),
        "tube": box([0, 0, 1], [2, 2, 2], {"emissionMode": "path", "pathIntensity": 3.0, "pathFalloffPower": 1.5,
                                           "pathPoints": [{"p": [-0.8, -0.5, 1], "radius": 0.3, "t": 0},
                                                          {"p": [0, 0.2, 1.2], "radius": 0.2, "t": 0.5},
                                                          {"p": [0.7, 0.6, 0.8], "radius": 0.05, "t": 1}]}),
        "haze": box([0, 0, 0], [3, 2, 1], {"heatHaze": True, "iorAmplitude": 0.02, "iorFrequency": 1.2,
                                           "iorOctaves": 3, "iorMarchSteps": 12, "iorFalloff": 0.5}),
    }
    return json_scene(rg, tmp_path, media, "fields.json")


def test_medium_fields_match_the_oracle(rg, orc, tmp_path):
    sc = field_scene(rg, tmp_path)
    r = rg.RayRenderer(rg.RendererSettings(resolutionWidth=8, resolutionHeight=8, samples=1))
    r.set_scene(sc)
    o = orc.OracleScene(sc.ptr)
    d = sc.desc
    rng = np.random.default_rng(9)
    pts = (rng.uniform(-3, 3, (20000, 3)) + np.array([0, -0.5, -6])).astype(np.float32)  # camera space
    for mi in range(d.num_media):
        g, c = r.medium_eval(mi, pts), o.medium_eval(mi, pts)
        np.testing.assert_array_equal(g[:, 0], c[:, 0])  # density: exact
        np.testing.assert_array_equal(g[:, 4], c[:, 4])  # index of refraction: exact
        np.testing.assert_allclose(g[:, 1:4], c[:, 1:4], rtol=2e-6, atol=1e-7)  # expf / powf may differ by an ulp
    haze = max(range(d.num_media), key=lambda i: d.media[i].heat_haze)
    dirs = rng.normal(size=(3000, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    rays = np.concatenate([pts[:3000], dirs, rng.uniform(0.2, 3.0, (3000, 1))], axis=1).astype(np.float32)
    gb, cb = r.medium_bend(haze, rays), o.medium_bend(haze, rays)
    np.testing.assert_array_equal(gb, cb)
    assert np.abs(gb[:, 3:] - rays[:, 3:6]).max() > 1e-4  # the rays were bent
    r.close()


def test_fbm_cloud_image_parity(rg, orc, tmp_path):
    objs = dict(ROOM, **LAMP)
    objs["cloud"] = box([0, 0.6, 0], [2.4, 1.6, 2.4],
                        {"sigma_a": [0.05] * 3, "sigma_s": [2.5] * 3, "g": 0.6, "densityField": "fbm",
                         "noiseFrequency": 1.6, "noiseOctaves": 4, "noiseAmplitude": 1.4, "noiseBias": -0.25})
    sc = json_scene(rg, tmp_path, objs, "cloud.json")
    z, g, m, stats = image_parity(rg, orc, sc, 48, 32, 96, maxDepth=8, rrDepth=3, seed=4)
    check_z(z, g, m, "fBm cloud", tail=0.01)


def test_jet_flame_image_parity(rg, orc, tmp_path):
    """Cone emission seen through a transparent box, lighting the floor, the back
    wall and a glossy ball through volume-light NEE; a thin global fog adds
    scatter-vertex NEE toward the flame."""
    objs = dict(ROOM)
    objs["flame"] = box([0.6, 0.0, 0.0], [1.8, 0.9, 0.9], FLAME)
    fog = {"sigma_a": [0.01] * 3, "sigma_s": [0.04] * 3, "g": 0.3}
    sc = json_scene(rg, tmp_path, objs, "flame.json", medium=fog)
    z, g, m, stats = image_parity(rg, orc, sc, 48, 32, 96, maxDepth=6, rrDepth=3, seed=5)
    check_z(z, g, m, "jet flame", tail=0.01)
    assert g.mean() > 1e-3


def test_turbulent_absorbing_flame_image_parity(rg, orc, tmp_path):
    objs = dict(ROOM, **LAMP)
    flame = dict(FLAME, sigma_a=[0.3, 0.3, 0.3], densityField="fbm", noiseFrequency=4.0, noiseOctaves=4,
                 noiseGain=0.55, noiseLacunarity=2.1, noiseAmplitude=1.6, noiseBias=-0.3, coneEmissionSamples=12)
    objs["flame"] = box([0.6, 0.0, 0.0], [1.8, 0.9, 0.9], flame)
    sc = json_scene(rg, tmp_path, objs, "turbulent.json")
    z, g, m, stats = image_parity(rg, orc, sc, 48, 32, 96, maxDepth=6, rrDepth=3, seed=6)
    check_z(z, g, m, "turbulent absorbing flame", tail=0.01)


def test_path_tube_image_parity(rg, orc, tmp_path):
    objs = dict(ROOM, **LAMP)
    objs["vapour"] = box([0, 0.3, 0], [3, 2, 2],
                         {"emissionMode": "path", "pathIntensity": 4.0, "pathFalloffPower": 1.5,
                          "pathEmissionSamples": 8, "pathFollowObject": True,
                          "pathPoints": [{"p": [-0.45, -0.3, 0], "radius": 0.3, "t": 0},
                                         {"p": [0, 0.1, 0.1], "radius": 0.2, "t": 0.5},
                                         {"p": [0.4, 0.35, -0.1], "radius": 0.05, "t": 1}]})
    sc = json_scene(rg, tmp_path, objs, "tube.json")
    z, g, m, stats = image_parity(rg, orc, sc, 48, 32, 96, maxDepth=6, rrDepth=3, seed=7)
    check_z(z, g, m, "path tube", tail=0.01)


def test_heat_haze_image_parity(rg, orc, tmp_path):
    objs = dict(ROOM)
    objs.pop("back")
    objs["exhaust"] = box([0, 0.5, 1.5], [4, 2.5, 1.5],
                          {"heatHaze": True, "iorAmplitude": 0.03, "iorFrequency": 1.2, "iorOctaves": 3,
                           "iorMarchSteps": 12, "iorOffset": [0.1, 0.2, 0.3]})
    sc = json_scene(rg, tmp_path, objs, "haze.json", envmap=True)
    z, g, m, stats = image_parity(rg, orc, sc, 48, 32, 64, maxDepth=6, rrDepth=3, seed=8)
    check_z(z, g, m, "heat haze", tail=0.01)


def test_constant_glow_volume_light_and_heterogeneous_fog(rg, orc, tmp_path):
    """A constant-emission interior medium is a volume light anchored at its
    object's location (rayrenderer.cpp:2091-2100); the global fog has an fBm
    density (delta tracking on every segment)."""
    objs = dict(ROOM, **LAMP)
    objs["glow"] = box([1.2, -0.2, 0], [1, 1, 1], {"emission": [0.8, 0.5, 0.2], "sigma_a": [0.2] * 3})
    fog = {"sigma_a": [0.01] * 3, "sigma_s": [0.08] * 3, "g": 0.2, "densityField": "fbm", "noiseFrequency": 0.8,
           "noiseAmplitude": 1.2, "noiseBias": -0.1}
    sc = json_scene(rg, tmp_path, objs, "glow.json", medium=fog)
    z, g, m, stats = image_parity(rg, orc, sc, 48, 32, 96, maxDepth=6, rrDepth=3, seed=9)
    check_z(z, g, m, "constant glow + fBm fog", tail=0.01)


def test_media_scene_in_the_server_matches_the_renderer(rg, tmp_path):
    objs = dict(ROOM, **LAMP)
    objs["flame"] = box([0.6, 0.0, 0.0], [1.8, 0.9, 0.9], dict(FLAME, densityField="fbm", noiseAmplitude=1.4,
                                                                 noiseBias=-0.2, sigma_s=[0.5] * 3))
    sc = json_scene(rg, tmp_path, objs, "server.json")
    plain = rg.Scene.builtin(1, 1)
    srv = rg.RenderServer(max_resident_jobs=4)
    j = srv.submit(sc, 48, 32, 32, max_depth=5, seed=3)  # waves holding it take the procedural-media kernels
    k = srv.submit(plain, 40, 30, 16, max_depth=5, seed=4)
    srv.wait(j)
    srv.wait(k)
    a, ap = srv.result(j), srv.result(k)
    srv.close()
    for scene, (w, h, spp, seed), got in ((sc, (48, 32, 32, 3), a), (plain, (40, 30, 16, 4), ap)):
        r = render_gpu(rg, scene, w, h, spp, maxDepth=5, seed=seed)
        b = r.get_hdr_result()
        r.close()
        np.testing.assert_allclose(got, b, rtol=1e-4, atol=1e-6)
        assert b[..., :3].mean() > 0
