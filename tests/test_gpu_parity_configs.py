"""Device vs CPU oracle on the benchmarked configurations and on the lobe,
camera and light branches that the smaller parity scenes do not take (needs a
B200).

* the 4,014,124-triangle benchmark scene: 50,000-ray closest / any-hit batches
  (all four occluder predicates) and a reduced-resolution image of the
  benchmark job (96 x 54, 64 spp, depth 8);
* the media + adaptive + A-Trous configuration as configured (fog sigma_t
  0.05, albedo 0.8, g 0.3; per-pixel adaptive 16 -> 256 spp at 0.02;
  5-level A-Trous on FP16 guides), at 64 x 36;
* anisotropic GGX (bsdf.cpp:233-249), rough dielectrics (:429-431, :496-498),
  chromatic dispersion (:394-420), the thin lens with a disk and with aperture
  blades (rayrenderer.cpp:862-934), spot and point lights (:2205-2260).

Tolerances as in test_gpu_parity.py (per-pixel |z| against the Monte-Carlo
error: mean |z| < 1, few channels beyond 4 sigma, image means within 1%).
"""
import json

import numpy as np
import pytest

import scenes
from test_gpu_parity import check_z, image_parity, render_gpu

pytestmark = pytest.mark.gpu

HEAVY = (2, 1, [1003520])


def test_benchmark_scene_ray_batches(rg, orc):
    sc = rg.Scene.builtin(*HEAVY)
    assert sc.desc.num_triangles == 4014124
    r = rg.RayRenderer(rg.RendererSettings(resolutionWidth=8, resolutionHeight=8, samples=1))
    r.set_scene(sc)
    o = orc.OracleScene(sc.ptr)
    rays = scenes.random_rays(((-9.5, -4.9, -19.5), (9.5, 4.9, -0.5)), 50000, 21)
    tg, pg = r.trace_closest(rays)
    to, po = o.closest(rays)
    same = pg == po
    assert same.mean() > 0.999, same.mean()
    hit = same & (po >= 0)
    assert hit.mean() > 0.95
    np.testing.assert_allclose(tg[hit, 0], to[hit, 0], rtol=1e-5, atol=2e-6)
    tmax = np.random.default_rng(3).uniform(0.05, 25.0, len(rays)).astype(np.float32)
    for pred in (0, 1, 2, 3):
        a = r.trace_any(rays, tmax, pred)
        b = o.any(rays, tmax, pred)
        assert (a == b).mean() > 0.999, pred
    assert r.stats()["device_error"] == 0
    o.close()
    r.close()
    sc.close()


def test_benchmark_job_image(rg, orc):
    sc = rg.Scene.builtin(*HEAVY)
    z, g, m, stats = image_parity(rg, orc, sc, 96, 54, 64, maxDepth=8, rrDepth=3, seed=1)
    check_z(z, g, m, "benchmark job 96x54", tail=0.01)
    assert stats["device_error"] == 0
    sc.close()


def test_media_adaptive_atrous_configuration(rg, orc):
    """Fog (sigma_t 0.05, albedo 0.8, g 0.3) over the benchmark geometry, per-pixel
    adaptive sampling 16 -> 256 spp at relative variance 0.02, then the 5-level
    A-Trous on FP16 guides: sample counts, the noisy image and the denoised image."""
    sc = rg.Scene.builtin(3, 1, [1003520])
    med = sc.desc.media[sc.desc.global_medium]
    assert np.allclose([med.sigma_a[0] + med.sigma_s[0], med.sigma_s[0] / (med.sigma_a[0] + med.sigma_s[0]), med.g],
                       [0.05, 0.8, 0.3], atol=1e-6)
    W, H = 64, 36
    kw = dict(maxDepth=8, rrDepth=3, seed=1, enableAdaptiveSampling=True, adaptiveBaseSamples=16,
              adaptiveThreshold=0.02, adaptiveMode=1)
    o = orc.OracleScene(sc.ptr)
    ref = o.render(W, H, 256, max_depth=8, rr_depth=3, seed=1, adaptive=True, adaptive_base=16, adaptive_mode=1,
                   adaptive_threshold=0.02)
    r = render_gpu(rg, sc, W, H, 256, **kw)
    cg = r.get_sample_counts()
    assert cg.min() >= 16 and cg.max() <= 256
    assert (cg == ref["n"]).mean() > 0.97
    assert abs(cg.sum() - ref["n"].sum()) / ref["n"].sum() < 0.03
    # noisy image: where both sides took the same samples, per-pixel z against the MC error
    g = r.get_hdr_result()[..., :3].astype(np.float64)
    n = ref["n"][..., None].astype(np.float64)
    m = ref["sum"] / n
    se = np.sqrt(2.0 * np.maximum(ref["sumsq"] / n - m * m, 0.0) / n)
    z = np.abs(g - m) / np.maximum(se, 1e-6)
    z[(se < 1e-6) & (np.abs(g - m) < 1e-4)] = 0.0
    same = (cg == ref["n"])
    check_z(z[same], g[same], m[same], "C3 noisy, adaptive", tail=0.01)
    r.close()
    # denoised: the device's 5-level A-Trous (FP16 guides) against the oracle's FP32 one
    r = render_gpu(rg, sc, W, H, 256, enableDenoise=True, **kw)
    gd = r.get_hdr_result()[..., :3].astype(np.float64)
    refd = o.render(W, H, 256, max_depth=8, rr_depth=3, seed=1, adaptive=True, adaptive_base=16, adaptive_mode=1,
                    adaptive_threshold=0.02, denoise=True)
    md = refd["hdr"][..., :3].astype(np.float64)
    assert abs(gd.mean() - md.mean()) / md.mean() < 0.01
    # each denoised pixel is a weighted mean of noisy neighbours that agree within the MC error
    assert (np.abs(gd - md) > 4.0 * se + 1e-3 * md.max()).mean() < 0.01
    assert r.stats()["device_error"] == 0
    r.close()
    o.close()
    sc.close()


LAMP = {"location": [0, 3.95, -1], "angle": [180, 0, 0], "scale": [3, 1, 2], "mesh": {"type": "plane"},
        "mat": {"color": [1, 0.95, 0.9], "emission": 6}}
ROOM = {
    "floor": {"location": [0, -1, -1], "scale": [10, 1, 10], "mesh": {"type": "plane"}, "mat": {"color": "#bbbbbb"}},
    "back": {"location": [0, 1.5, -4], "angle": [90, 0, 0], "scale": [10, 1, 6], "mesh": {"type": "plane"},
             "mat": {"color": [0.3, 0.5, 0.7]}},
    "left": {"location": [-4, 1.5, -1], "angle": [0, 0, -90], "scale": [6, 1, 10], "mesh": {"type": "plane"},
             "mat": {"color": [0.7, 0.25, 0.2]}},
}
SPHERE = {"type": "sphere", "radius": 0.75, "stacks": 24, "slices": 48}

BRANCH_SCENES = {
    # anisotropic GGX: alpha_x / alpha_y split and the rotated tangent frame
    "anisotropic_ggx": {
        "mainCamera": {"location": [0, 0.8, 4], "angle": [-10, 0, 0], "fieldOfView": 55},
        "lamp": LAMP, **ROOM,
        "a": {"location": [-1.7, -0.25, -1], "mesh": SPHERE,
              "mat": {"color": "#e0c090", "glossy": 1, "metallic": 1, "roughness": 0.45, "anisotropy": 0.8}},
        "b": {"location": [0, -0.25, -1.3], "mesh": SPHERE,
              "mat": {"color": "#c0c8e0", "glossy": 1, "metallic": 1, "roughness": 0.6, "anisotropy": -0.6,
                      "anisoRotation": 45}},
        "c": {"location": [1.7, -0.25, -1], "mesh": SPHERE,
              "mat": {"color": "#d04030", "glossy": 1, "metallic": 0.3, "roughness": 0.35, "anisotropy": 0.5,
                      "anisoRotation": -30}},
    },
    # rough dielectrics: the hemisphere jitter of the reflected and refracted directions
    "rough_dielectric": {
        "mainCamera": {"location": [0, 0.8, 4], "angle": [-10, 0, 0], "fieldOfView": 55},
        "lamp": LAMP, **ROOM,
        "a": {"location": [-1.7, -0.25, -1], "mesh": SPHERE,
              "mat": {"refraction": 1, "refractionRatio": 1.5, "roughness": 0.15}},
        "b": {"location": [0, -0.25, -1.3], "mesh": SPHERE,
              "mat": {"refraction": 1, "refractionRatio": 1.33, "roughness": 0.45, "color": [0.9, 1, 0.9]}},
        "c": {"location": [1.7, -0.25, -1], "mesh": {"type": "cube"}, "scale": [1.2, 1.2, 1.2],
              "mat": {"refraction": 1, "refractionRatio": 1.7, "roughness": 0.3}},
    },
    # chromatic dispersion: one RGB channel per path, tripled
    "dispersion": {
        "mainCamera": {"location": [0, 0.8, 4], "angle": [-10, 0, 0], "fieldOfView": 55},
        "lamp": LAMP, **ROOM,
        "a": {"location": [-1.0, -0.25, -1], "mesh": SPHERE,
              "mat": {"refraction": 1, "refractionRatio": 1.6, "chromaDispersion": 0.08}},
        "b": {"location": [1.0, -0.25, -1.2], "mesh": SPHERE,
              "mat": {"refraction": 1, "refractionRatio": 1.5, "chromaDispersion": 0.04, "roughness": 0.1}},
    },
    # thin lens with a six-blade aperture, a spot light (a cone of about 37 degrees
    # through the reference's degree/radian spotRange arithmetic) and a point light
    "thin_lens_blades_spot": {
        "mainCamera": {"location": [0, 0.8, 4], "angle": [-10, 0, 0], "fieldOfView": 55, "depthOfField": 5.2,
                       "aperture": 3.0, "apertureBlades": 6, "apertureRotation": 15},
        **ROOM,
        "spot": {"location": [-0.8, 3.0, -1.0], "mat": {"emission": 40, "spotRange": 0.2351, "color": [1, 0.9, 0.7]}},
        "bulb": {"location": [1.8, 2.0, 0.5], "mat": {"emission": 8, "color": [0.7, 0.8, 1]}},
        "near": {"location": [-1.2, -0.25, 1.0], "mesh": SPHERE, "mat": {"glossy": 1, "roughness": 0.2, "metallic": 1}},
        "far": {"location": [1.2, -0.25, -2.5], "mesh": SPHERE, "mat": {"color": "#ffffff"}},
    },
    # thin lens with the concentric disk (no blades)
    "thin_lens_disk": {
        "mainCamera": {"location": [0, 0.8, 4], "angle": [-10, 0, 0], "fieldOfView": 55, "depthOfField": 3.0,
                       "aperture": 2.0},
        "lamp": LAMP, **ROOM,
        "near": {"location": [-1.0, -0.25, 1.0], "mesh": SPHERE, "mat": {"color": "#e0e0a0"}},
        "far": {"location": [1.2, -0.25, -2.5], "mesh": SPHERE, "mat": {"glossy": 1, "roughness": 0.3}},
    },
}


@pytest.mark.parametrize("name", list(BRANCH_SCENES))
def test_branch_image_parity(rg, orc, tmp_path, name):
    p = tmp_path / f"{name}.json"
    p.write_text(json.dumps(BRANCH_SCENES[name]))
    sc = rg.Scene.from_json(str(p))
    z, g, m, stats = image_parity(rg, orc, sc, 48, 36, 128, maxDepth=8, rrDepth=3, seed=7)
    check_z(z, g, m, name, tail=0.01)
    assert g.mean() > 0.01, "the scene renders black: the branch is not exercised"
    assert stats["device_error"] == 0
    sc.close()


@pytest.mark.parametrize("roughness,anisotropy,tilt", scenes.FURNACE_CASES)
def test_ggx_white_furnace_on_device(rg, orc, roughness, anisotropy, tilt):
    """The GGX furnace known answer (directional albedo by quadrature) on the
    device, and the same image against the oracle."""
    sc = scenes.furnace_scene(rg, roughness, anisotropy, tilt)
    r = render_gpu(rg, sc, 32, 32, 256, maxDepth=8, rrDepth=3, seed=3, fireflyClamp=0.0)
    mean = float(r.get_hdr_result()[..., :3].mean())
    r.close()
    expected = scenes.furnace_expected(roughness, anisotropy, tilt)
    assert abs(mean - expected) < 0.01 * expected, (mean, expected)
    z, g, m, _ = image_parity(rg, orc, sc, 32, 32, 64, maxDepth=8, rrDepth=3, seed=3, fireflyClamp=0.0)
    check_z(z, g, m, f"furnace r={roughness} aniso={anisotropy} tilt={tilt}")
    sc.close()
