"""Procedural participating media on the CPU: the oracle's fields against a
from-scratch numpy restatement (fBm density, cone and path emission, heat-haze
bending), analytic known answers (delta-tracking transmittance through an fBm
absorber, the stratified cone emission integral, the equiangular volume-light
estimator), the volume-light occluder class, and the loader's medium schema.

Follows medium.cpp:18-525 (HomogeneousMedium), rayrenderer.cpp:1596-1864
(tracePath), :2067-2203 (sampleVolumeLightForNEE), :180-206 (emissive-volume
registration) and sceneloader.cpp:202-334 (readMedium).  No GPU needed.
"""
import json
import math

import numpy as np
import pytest

import media_numpy as mn
import scenes

FBM = dict(noise_frequency=1.6, noise_octaves=4, noise_gain=0.5, noise_lacunarity=2.0, noise_amplitude=1.4,
           noise_bias=-0.25, noise_offset=[0.3, -0.2, 0.1])


def with_media(rg, media, global_medium=-1, volume_objects=(), far=True, parts=()):
    """Scene of `parts` (plus one far triangle behind the camera so the BVH is not
    empty) and mesh-less objects whose interior media are `volume_objects`
    (medium index, location)."""
    parts = list(parts)
    if far:
        fp, fn = scenes.quad_z(60.0, 0.5, +1)
        parts.append((fp, fn, scenes.material(rg, (0.5, 0.5, 0.5)), -1))
    pos, nrm, tri_mesh, mesh_obj, objs, mats = [], [], [], [], [], []
    for k, (p, n, m, med) in enumerate(parts):
        pos.append(p)
        nrm.append(n)
        tri_mesh += [k] * len(p)
        mesh_obj.append(k)
        o = rg.rg_object()
        o.material = k
        o.interior_medium = med
        objs.append(o)
        mats.append(m)
    for med, loc in volume_objects:
        o = rg.rg_object()
        o.material = 0
        o.interior_medium = med
        o.location[:] = list(loc)
        objs.append(o)
    return rg.Scene.from_arrays(np.concatenate(pos), np.concatenate(nrm), tri_mesh, mesh_obj, objs, mats,
                                scenes.camera(rg, fov=0.5), media=media, global_medium=global_medium)


def test_medium_defaults(rg):
    m = rg.medium()
    assert m.density == 1.0 and m.emission_mode == 0 and m.density_field == 0 and m.heat_haze == 0
    assert list(m.cone_axis) == [0.0, 0.0, -1.0] and m.cone_length == 1.0 and m.cone_radius == pytest.approx(0.3)
    assert m.cone_intensity == 50.0 and m.cone_emission_samples == 4 and m.cone_peak_axial == pytest.approx(0.15)
    assert m.cone_peak_sharpness == 5.0 and m.path_intensity == 1.0 and m.path_falloff_power == 2.0
    assert m.path_emission_samples == 6 and m.noise_frequency == 1.0 and m.noise_octaves == 4
    assert m.ior_amplitude == pytest.approx(0.005) and m.ior_frequency == 4.0 and m.ior_octaves == 3
    assert m.ior_march_steps == 16 and m.num_path_points == 0


def test_density_field_matches_numpy_bit_for_bit(rg, orc):
    m = rg.medium(sigma_a=[0.05] * 3, sigma_s=[3.0] * 3, density_field=rg.RG_DENSITY_FBM, **FBM)
    o = orc.OracleScene(with_media(rg, [m], global_medium=0).ptr)
    pts = np.random.default_rng(1).uniform(-6, 6, (5000, 3)).astype(np.float32)
    got = o.medium_eval(0, pts)
    want = mn.density(pts, 1.6, 4, 0.5, 2.0, 1.4, -0.25, (0.3, -0.2, 0.1))
    np.testing.assert_array_equal(got[:, 0], want)
    assert (want == 0).any() and want.max() > 0.6  # the bias carves empty pockets
    # constant emission is scaled by the density field too (medium.cpp:305-309)
    g = rg.medium(sigma_e=[0.5, 0.25, 0.0], density_field=rg.RG_DENSITY_FBM, **FBM)
    o2 = orc.OracleScene(with_media(rg, [g], global_medium=0).ptr)
    e = o2.medium_eval(0, pts)
    np.testing.assert_allclose(e[:, 1:4], want[:, None] * np.array([0.5, 0.25, 0.0], np.float32), rtol=1e-6)


def test_cone_emission_matches_numpy(rg, orc):
    axis = np.array([0.3, 0.1, -1.0], np.float32)
    m = rg.medium(emission_mode=rg.RG_EMISSION_CONE, cone_origin=[0.2, 0.1, -3.0], cone_axis=list(axis),
                  cone_length=1.6, cone_radius=0.35, cone_inner=[4, 6, 12], cone_outer=[10, 3, 0.4],
                  cone_intensity=25.0, cone_peak_axial=0.18, cone_peak_sharpness=4.0, density=1.5)
    o = orc.OracleScene(with_media(rg, [m], global_medium=0).ptr)
    a = axis / np.sqrt((axis * axis).sum())
    rng = np.random.default_rng(2)
    s = rng.uniform(-0.1, 1.1, 4000)
    q = rng.normal(size=(4000, 3)) * 0.25
    pts = (np.array([0.2, 0.1, -3.0]) + np.outer(s * 1.6, a) + q).astype(np.float32)
    got = o.medium_eval(0, pts)[:, 1:4]
    want = mn.cone_emission(pts, [0.2, 0.1, -3.0], a, 1.6, 0.35, [4, 6, 12], [10, 3, 0.4], 25.0, 0.18, 4.0, 1.5)
    np.testing.assert_allclose(got, want, rtol=2e-5, atol=2e-5)
    assert (want > 0).any() and (want == 0).any()


def test_path_emission_matches_numpy(rg, orc):
    pts_ctrl = [((0.0, 0.0, -2.0), 0.3, 0.0), ((0.5, 0.2, -2.5), 0.2, 0.4), ((0.8, 0.6, -3.2), 0.05, 1.0)]
    m = rg.medium(emission_mode=rg.RG_EMISSION_PATH, path_points=pts_ctrl, path_inner=[0.6, 0.7, 1.0],
                  path_outer=[0.3, 0.4, 0.6], path_intensity=3.0, path_falloff_power=1.5)
    o = orc.OracleScene(with_media(rg, [m], global_medium=0).ptr)
    rng = np.random.default_rng(3)
    pts = (np.array([0.4, 0.3, -2.6]) + rng.normal(size=(4000, 3)) * 0.4).astype(np.float32)
    got = o.medium_eval(0, pts)[:, 1:4]
    want = mn.path_emission(pts, pts_ctrl, [0.6, 0.7, 1.0], [0.3, 0.4, 0.6], 3.0, 1.5)
    np.testing.assert_allclose(got, want, rtol=1e-4, atol=1e-5)
    assert (want > 0).any() and (want == 0).any()


def test_heat_haze_bend_matches_numpy(rg, orc):
    m = rg.medium(heat_haze=1, ior_amplitude=0.012, ior_frequency=1.2, ior_octaves=3, ior_gain=0.5,
                  ior_lacunarity=2.0, ior_march_steps=12)
    o = orc.OracleScene(with_media(rg, [m], global_medium=0).ptr)
    rng = np.random.default_rng(4)
    n = 300
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.concatenate([rng.uniform(-2, 2, (n, 3)), d, rng.uniform(0.5, 4.0, (n, 1))], axis=1).astype(np.float32)
    got = o.medium_bend(0, rays)
    want = mn.bend(rays, 0.012, 1.2, 3, 0.5, 2.0, 12)
    np.testing.assert_allclose(got, want, rtol=0, atol=2e-6)
    # unit directions, and a visible deflection that grows with the amplitude
    assert np.allclose(np.linalg.norm(got[:, 3:], axis=1), 1.0, atol=1e-6)
    ang = np.arccos(np.clip((got[:, 3:] * rays[:, 3:6]).sum(axis=1), -1, 1))
    assert ang.mean() > 1e-4
    ior = o.medium_eval(0, rays[:, :3])[:, 4]
    np.testing.assert_array_equal(ior, mn.ior(rays[:, :3], 0.012, 1.2, 3, 0.5, 2.0))
    assert np.all(np.abs(ior - 1.0) <= 0.012 + 1e-7)


def test_heat_haze_off_is_a_straight_march(rg, orc):
    m = rg.medium(sigma_a=[0.1] * 3, heat_haze=1, ior_amplitude=0.0)  # isHeatHaze needs amplitude > 0
    o = orc.OracleScene(with_media(rg, [m], global_medium=0).ptr)
    rays = np.array([[0, 0, 0, 0, 0, -1, 3.0], [1, 2, 3, 0.6, 0.8, 0, 2.0]], np.float32)
    out = o.medium_bend(0, rays)
    np.testing.assert_allclose(out[:, :3], rays[:, :3] + rays[:, 3:6] * rays[:, 6:7], rtol=1e-6)
    np.testing.assert_array_equal(out[:, 3:], rays[:, 3:6])


def test_delta_tracking_transmittance_through_fbm_absorber(rg, orc):
    """A pure absorber with an fBm density: the eye ray reaches the emitter with
    probability exp(-sigma_t * integral of the density) (delta tracking is exact)."""
    le, dist = 2.0, 5.0
    m = rg.medium(sigma_a=[0.3] * 3, density_field=rg.RG_DENSITY_FBM, noise_frequency=0.7, noise_octaves=3,
                  noise_gain=0.5, noise_lacunarity=2.0, noise_amplitude=1.2, noise_bias=-0.1)
    lp, ln = scenes.quad_z(-dist, 50.0, +1)
    sc = with_media(rg, [m], global_medium=0, parts=[(lp, ln, scenes.material(rg, (1, 1, 1), emission=le), -1)])
    o = orc.OracleScene(sc.ptr)
    s = np.linspace(0.0, dist, 40001)
    pts = np.stack([np.zeros_like(s), np.zeros_like(s), -s], axis=1).astype(np.float32)
    dens = o.medium_eval(0, pts)[:, 0].astype(np.float64)
    tau = 0.3 * np.trapezoid(dens, s)
    T = math.exp(-tau)
    assert 0.1 < T < 0.9
    assert dens.min() < 0.5 * dens.max()  # the field really varies along the ray
    spp = 16384
    out = o.render(1, 1, spp, max_depth=4, firefly_clamp=0.0, antialias=False)
    mean = float(out["sum"][0, 0, 0] / out["n"][0, 0])
    se = le * math.sqrt(T * (1 - T) / spp)
    assert abs(mean - le * T) < 4 * se, (mean, le * T, se)


def test_cone_emission_integral_along_the_eye_ray(rg, orc):
    """A purely emissive cone seen along its axis: the stratified estimator
    converges to the line integral of sigma_e (no extinction)."""
    m = rg.medium(emission_mode=rg.RG_EMISSION_CONE, cone_origin=[0, 0, -2.0], cone_axis=[0, 0, -1],
                  cone_length=3.0, cone_radius=0.6, cone_inner=[1, 1.2, 1.8], cone_outer=[1.2, 0.4, 0.05],
                  cone_intensity=2.0, cone_peak_axial=0.3, cone_peak_sharpness=3.0, cone_emission_samples=8)
    o = orc.OracleScene(with_media(rg, [m], global_medium=0).ptr)
    s = np.linspace(0.0, 100.0, 200001)
    pts = np.stack([np.zeros_like(s), np.zeros_like(s), -s], axis=1).astype(np.float32)
    e = o.medium_eval(0, pts)[:, 1:4].astype(np.float64)
    want = np.trapezoid(e, s, axis=0)
    spp = 32768
    out = o.render(1, 1, spp, max_depth=4, firefly_clamp=0.0, antialias=False)
    n = out["n"][0, 0]
    mean = out["sum"][0, 0] / n
    se = np.sqrt(np.maximum(out["sumsq"][0, 0] / n - mean * mean, 0) / n)
    assert np.all(np.abs(mean - want) < 4 * se + 1e-6), (mean, want, se)


@pytest.mark.parametrize("count", [1, 2])
def test_equiangular_volume_light_estimator(rg, orc, count):
    """E[Le / pdf] of volume-light NEE is the sum over the volumes of the line
    integral of sigma_e / r^2 along each cone axis, divided by count^2: the
    reference folds the pick probability into the pdf as a factor `count`
    instead of 1 / count (rayrenderer.cpp:2190-2193), kept as written."""
    m = rg.medium(emission_mode=rg.RG_EMISSION_CONE, cone_origin=[0.0, 0.0, -3.0], cone_axis=[1, 0, 0],
                  cone_length=2.0, cone_radius=0.4, cone_intensity=5.0, cone_peak_axial=0.4,
                  cone_peak_sharpness=2.0)
    sc = with_media(rg, [m], volume_objects=[(0, (0, 0, 0))] * count)
    o = orc.OracleScene(sc.ptr)
    assert o.num_volume_lights() == count
    hit = np.array([0.7, 1.2, -2.5], np.float32)
    d, pdf, le, ok = o.volume_nee(hit, [0, -1, 0], 40000, seed=7)
    assert ok.mean() > 0.95
    est = np.where(ok[:, None], le / np.maximum(pdf, 1e-30)[:, None], 0.0)
    s = np.linspace(0.0, 2.0, 40001)
    axis_pts = np.stack([s, np.zeros_like(s), np.full_like(s, -3.0)], axis=1).astype(np.float32)
    sig = o.medium_eval(0, axis_pts)[:, 1:4].astype(np.float64)
    r2 = ((axis_pts.astype(np.float64) - hit) ** 2).sum(axis=1)
    want = count * np.trapezoid(sig / r2[:, None], s, axis=0) / count ** 2  # `count` identical volumes
    mean = est.mean(axis=0)
    se = est.std(axis=0) / math.sqrt(len(est))
    assert np.all(np.abs(mean - want) < 4 * se + 1e-6), (mean, want, se)
    # directions point at the axis and are unit vectors
    assert np.allclose(np.linalg.norm(d[ok], axis=1), 1.0, atol=1e-5)


def test_volume_light_occluder_class(rg, orc):
    """Refractive surfaces let volume-light shadow rays through (rayrenderer.cpp:2167-2171)
    but stop environment / point-light rays (:2211-2215); opaque ones stop both."""
    def quad(z, **kw):
        p, n = scenes.quad_z(z, 1.0, +1)
        return (p, n, scenes.material(rg, (0.8, 0.8, 0.8), **kw), -1)
    rays = np.array([[0, 0, 0, 0, 0, -2]], np.float32)
    for kw, blocks_point, blocks_volume in ((dict(refraction=0.5), True, False), (dict(), True, True),
                                            (dict(emission=2.0), False, False), (dict(transparency=0.5), False, False)):
        sc = scenes.build(rg, [quad(-1.0, **kw)], scenes.camera(rg))
        o = orc.OracleScene(sc.ptr)
        assert o.any(rays, np.array([0.99999], np.float32), rg.PRED_POINT)[0] == blocks_point, kw
        assert o.any(rays, np.array([0.99999], np.float32), rg.PRED_VOLUME)[0] == blocks_volume, kw


# ---------------------------------------------------------------- loader
def load(rg, tmp_path, doc):
    p = tmp_path / "media.json"
    p.write_text(json.dumps(doc))
    return rg.Scene.from_json(str(p))


def test_loader_reads_the_medium_schema(rg, tmp_path):
    doc = {
        "mainCamera": {"location": [0, 0, 5], "fieldOfView": 40},
        "medium": {"sigma_a": [0.02, 0.02, 0.02], "sigma_s": [0.1, 0.1, 0.1], "densityField": "fbm",
                   "noiseFrequency": 2.5, "noiseOctaves": 5, "noiseGain": 0.6, "noiseLacunarity": 2.2,
                   "noiseAmplitude": 1.3, "noiseBias": -0.2, "noiseOffset": [1, 2, 3]},
        "flame": {"location": [1.5, 0.4, 0], "mesh": {"type": "cube"}, "mat": {"transparency": 1.0},
                  "medium": {"emissionMode": "cone", "coneFollowObject": True, "coneOrigin": [0.5, 0, 0],
                             "coneAxis": [-2, 0, 0], "coneLength": 1.6, "coneRadius": 0.35,
                             "coneInner": [4, 6, 12], "coneOuter": [10, 3, 0.4], "coneIntensity": 30,
                             "conePeakAxial": 0.18, "conePeakSharpness": 4, "coneEmissionSamples": 8}},
        "tube": {"mesh": {"type": "cube"}, "mat": {"transparency": 1.0},
                 "medium": {"emissionMode": "path", "pathIntensity": 2.0, "pathFalloffPower": 1.5,
                            "pathEmissionSamples": 9,
                            "pathPoints": [{"p": [0, 0, 0], "radius": 0.2, "t": 0}, {"p": [1, 0, 0]},
                                           7, {"p": [2, 1, 0], "radius": 0.05, "t": 1}]}},
        "haze": {"mesh": {"type": "cube"}, "mat": {"transparency": 1.0},
                 "medium": {"heatHaze": True, "iorAmplitude": 0.02, "iorFrequency": 1.2, "iorOctaves": 3,
                            "iorMarchSteps": 12, "iorFalloff": -0.5}},
        "dead": {"mesh": {"type": "cube"}, "medium": {"sigma_a": [0, 0, 0]}},
        "ghost": {"visible": False, "location": [0, 3, 0], "mesh": {"type": "cube"},
                  "medium": {"emissionMode": "cone", "coneIntensity": 10},
                  "child": {"mesh": {"type": "plane"}}},
        "glow": {"location": [0, -1, 0], "medium": {"emission": [0.5, 0.2, 0.1]}},
        "floor": {"mesh": {"type": "plane"}},
    }
    sc = load(rg, tmp_path, doc)
    d = sc.desc
    media = [d.media[i] for i in range(d.num_media)]
    g = media[d.global_medium]
    assert g.density_field == rg.RG_DENSITY_FBM and g.noise_octaves == 5
    assert g.noise_frequency == pytest.approx(2.5) and g.noise_bias == pytest.approx(-0.2)
    assert list(g.noise_offset) == [1, 2, 3] and g.emission_mode == 0
    objs = [d.objects[i] for i in range(d.num_objects)]
    meshes_of = {}
    for mi in range(d.num_meshes):
        meshes_of.setdefault(d.mesh_object[mi], []).append(mi)
    # flame, tube, haze, dead (no medium: inactive), ghost (mesh-less volume), glow (mesh-less volume), floor
    assert len(objs) == 7
    flame, tube, haze, dead, ghost, glow, floor = objs
    assert dead.interior_medium == -1 and floor.interior_medium == -1
    assert 4 not in meshes_of and 5 not in meshes_of and len(meshes_of) == 5
    fm = media[flame.interior_medium]
    assert fm.emission_mode == rg.RG_EMISSION_CONE and fm.cone_emission_samples == 8
    np.testing.assert_allclose(list(fm.cone_origin), [2.0, 0.4, 0.0], atol=1e-6)  # follows the object
    np.testing.assert_allclose(list(fm.cone_axis), [-2.0, 0.0, 0.0], atol=1e-6)
    assert fm.cone_intensity == 30 and fm.cone_peak_axial == pytest.approx(0.18)
    tm = media[tube.interior_medium]
    assert tm.emission_mode == rg.RG_EMISSION_PATH and tm.num_path_points == 3 and tm.path_emission_samples == 9
    pts = [(list(tm.path_points[i].p), tm.path_points[i].radius, tm.path_points[i].t) for i in range(3)]
    assert pts[1][0] == [1, 0, 0] and pts[1][1] == pytest.approx(0.1) and pts[1][2] == 0  # PathSample defaults
    assert pts[2][1] == pytest.approx(0.05) and pts[2][2] == 1
    hm = media[haze.interior_medium]
    assert hm.heat_haze == 1 and hm.ior_march_steps == 12 and hm.ior_falloff == pytest.approx(-0.5)
    assert hm.ior_gain == pytest.approx(0.5)  # default
    gm = media[ghost.interior_medium]
    assert gm.emission_mode == rg.RG_EMISSION_CONE and list(ghost.location) == [0, 3, 0]
    lm = media[glow.interior_medium]
    assert list(lm.sigma_e) == pytest.approx([0.5, 0.2, 0.1]) and list(glow.location) == [0, -1, 0]


def test_inactive_medium_keeps_the_previous_one(rg, tmp_path):
    """readMedium returns NULL for an inactive medium and the object keeps what it had."""
    doc = {"box": {"mesh": {"type": "cube"}, "medium": {"sigma_a": [0.5, 0.5, 0.5]}}}
    text = json.dumps(doc)[:-2] + ', "medium": {"sigma_s": [0, 0, 0]}}}'
    p = tmp_path / "keep.json"
    p.write_text(text)
    d = rg.Scene.from_json(str(p)).desc
    assert d.objects[0].interior_medium >= 0
    assert list(d.media[d.objects[0].interior_medium].sigma_a) == pytest.approx([0.5, 0.5, 0.5])
