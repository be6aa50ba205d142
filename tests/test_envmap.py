"""Environment maps on the host and in the oracle: Radiance .hdr / PFM readers,
the scene-JSON "envmap" key, and the oracle's equirectangular lookup,
importance sampler and NEE (no GPU).

Reference: decodeRadianceHDR (texture.cpp:74-151), sceneloader.cpp:700-748,
Scene::buildEnvmapCDF (scene.cpp:414-463), sampleEnvironment /
sampleEnvmapDirection / envmapDirectionPdf / traceEnvmapLight
(rayrenderer.cpp:1299-1573).
"""
import json

import numpy as np
import pytest

import scenes


def env_scene(rg, tmp_path, img, intensity=1.0, rotation=0.0, objects=None, camera=None, name="env.json",
              fmt="hdr"):
    if fmt == "hdr":
        ref = scenes.write_hdr(tmp_path / "sky.hdr", img)
    else:
        scenes.write_pfm(tmp_path / "sky.pfm", img)
        ref = np.asarray(img, np.float32)
    doc = {"mainCamera": camera or {"location": [0, 1, 4], "fieldOfView": 60},
           "envmap": {"texture": f"sky.{fmt}", "intensity": intensity, "rotation": rotation}}
    doc.update(objects or {})
    (tmp_path / name).write_text(json.dumps(doc))
    return rg.Scene.from_json(str(tmp_path / name)), ref


def texture_array(sc, i):
    t = sc.desc.textures[i]
    return np.ctypeslib.as_array(t.rgba, shape=(t.height, t.width, 4)).copy()


def test_rgbe_reader_rle_and_flat(rg, tmp_path):
    img = scenes.sky_image(77, 19, seed=3)  # odd width: RLE runs and literals of all lengths
    img[2, 5:40] = 0.0  # long zero runs
    for rle in (True, False):
        ref = scenes.write_hdr(tmp_path / "a.hdr", img, rle=rle)
        (tmp_path / "a.json").write_text(json.dumps({"envmap": "a.hdr"}))
        sc = rg.Scene.from_json(str(tmp_path / "a.json"))
        d = sc.desc
        assert d.has_envmap == 1 and d.num_textures == 1 and d.textures[0].is_hdr == 1
        got = texture_array(sc, 0)
        np.testing.assert_array_equal(got[..., :3], ref)
        assert np.all(got[..., 3] == 1.0)


def test_rgbe_reader_rejects_malformed(rg, tmp_path):
    scenes.write_hdr(tmp_path / "b.hdr", scenes.sky_image(16, 8))
    data = (tmp_path / "b.hdr").read_bytes()
    (tmp_path / "t.hdr").write_bytes(data[: len(data) - 40])
    (tmp_path / "t.json").write_text(json.dumps({"envmap": "t.hdr"}))
    with pytest.raises(rg.RayGenError, match="malformed Radiance") as e:
        rg.Scene.from_json(str(tmp_path / "t.json"))
    assert e.value.code == rg.RG_ERR_PARSE


def test_pfm_reader(rg, tmp_path):
    img = scenes.sky_image(9, 5, seed=4)
    sc, ref = env_scene(rg, tmp_path, img, fmt="pfm")
    np.testing.assert_array_equal(texture_array(sc, 0)[..., :3], ref)


def test_envmap_json_keys(rg, tmp_path):
    img = scenes.sky_image(16, 8)
    sc, _ = env_scene(rg, tmp_path, img, intensity=1.5, rotation=30)
    d = sc.desc
    assert d.has_envmap == 1 and d.envmap_texture == 0
    assert d.envmap_intensity == pytest.approx(1.5) and d.envmap_rotation == pytest.approx(30)
    # a path string; a missing file leaves the scene without an environment (as the reference)
    (tmp_path / "s.json").write_text(json.dumps({"envmap": "sky.hdr", "f": {"mesh": {"type": "plane"}}}))
    assert rg.Scene.from_json(str(tmp_path / "s.json")).desc.has_envmap == 1
    (tmp_path / "m.json").write_text(json.dumps({"envmap": {"texture": "nothere.hdr"}, "f": {"mesh": {"type": "plane"}}}))
    d = rg.Scene.from_json(str(tmp_path / "m.json")).desc
    assert d.has_envmap == 0 and d.num_triangles == 2
    # a cubemap with missing faces gives no cubemap (all six or none, scene.cpp:348)
    (tmp_path / "c.json").write_text(json.dumps({"envmap": {"cubemap": "../cube", "ext": "jpg"}}))
    assert rg.Scene.from_json(str(tmp_path / "c.json")).desc.envmap_cube == 0


def random_dirs(n, seed):
    rng = np.random.default_rng(seed)
    d = rng.standard_normal((n, 3))
    return (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)


def lookup_np(img, dirs, intensity, rotation):
    """Numpy restatement of sampleEnvironment's lat-long lookup (rayrenderer.cpp:1299-1348)."""
    H, W = img.shape[:2]
    d = dirs / np.linalg.norm(dirs, axis=1, keepdims=True)
    yaw = np.deg2rad(rotation)
    rx = d[:, 0] * np.cos(yaw) - d[:, 2] * np.sin(yaw)
    rz = d[:, 0] * np.sin(yaw) + d[:, 2] * np.cos(yaw)
    u = 0.5 + np.arctan2(rz, rx) / (2 * np.pi)
    v = 0.5 - np.arcsin(np.clip(d[:, 1], -1, 1)) / np.pi
    fu, fv = u - np.floor(u), v - np.floor(v)
    x = np.clip((fu * W).astype(int), 0, W - 1)
    y = np.clip((fv * H).astype(int), 0, H - 1)
    return img[y, x, :3] * intensity


@pytest.mark.parametrize("rotation", [0.0, 37.0, -120.0])
def test_env_lookup_matches_formula(rg, orc, tmp_path, rotation):
    img = scenes.sky_image(64, 32, seed=5)
    sc, ref = env_scene(rg, tmp_path, img, intensity=1.7, rotation=rotation)
    o = orc.OracleScene(sc.ptr)
    dirs = random_dirs(20000, 6)
    rgb, _ = o.env_eval(dirs)
    exp = lookup_np(ref, dirs, 1.7, rotation)
    close = np.all(np.abs(rgb - exp) <= 1e-5 * (1 + np.abs(exp)), axis=1)
    assert close.mean() > 0.995  # texel-boundary directions may round to the neighbour


def sphere_grid(nt=400, nph=800):
    th = (np.arange(nt) + 0.5) / nt * np.pi
    ph = (np.arange(nph) + 0.5) / nph * 2 * np.pi
    T, P = np.meshgrid(th, ph, indexing="ij")
    dirs = np.stack([np.sin(T) * np.cos(P), np.cos(T), np.sin(T) * np.sin(P)], axis=-1).reshape(-1, 3)
    dw = (np.sin(T) * (np.pi / nt) * (2 * np.pi / nph)).reshape(-1)
    return dirs.astype(np.float32), dw


def test_env_pdf_is_normalised(rg, orc, tmp_path):
    sc, _ = env_scene(rg, tmp_path, scenes.sky_image(64, 32, seed=7), rotation=25)
    o = orc.OracleScene(sc.ptr)
    dirs, dw = sphere_grid()
    _, pdf = o.env_eval(dirs)
    assert (pdf * dw).sum() == pytest.approx(1.0, rel=0.01)


def test_env_sample_pdf_consistency_and_distribution(rg, orc, tmp_path):
    img = scenes.sky_image(16, 8, sun=(0.3, 0.3), sun_radius=0.08, sun_level=20.0, seed=8)
    sc, ref = env_scene(rg, tmp_path, img)
    o = orc.OracleScene(sc.ptr)
    rng = np.random.default_rng(9)
    n = 200000
    dirs, pdf = o.env_sample(rng.random((n, 2)).astype(np.float32))
    assert np.allclose(np.linalg.norm(dirs, axis=1), 1.0, atol=1e-5)
    _, pdf2 = o.env_eval(dirs)
    agree = np.abs(pdf - pdf2) <= 1e-3 * pdf
    assert agree.mean() > 0.99
    # texel frequencies follow luminance x sin(theta) (the CDF's weights)
    H, W = ref.shape[:2]
    u = 0.5 + np.arctan2(dirs[:, 2], dirs[:, 0]) / (2 * np.pi)
    v = 0.5 - np.arcsin(np.clip(dirs[:, 1], -1, 1)) / np.pi
    x = np.clip((u * W).astype(int), 0, W - 1)
    y = np.clip((v * H).astype(int), 0, H - 1)
    counts = np.bincount(y * W + x, minlength=W * H).reshape(H, W)
    lum = np.maximum(0, 0.2126 * ref[..., 0] + 0.7152 * ref[..., 1] + 0.0722 * ref[..., 2])
    w = lum * np.sin(np.pi * (np.arange(H) + 0.5) / H)[:, None]
    p = w / w.sum()
    expected = p * n
    big = expected > 50
    z = (counts[big] - expected[big]) / np.sqrt(expected[big])
    assert np.abs(z).max() < 6.0


def test_oracle_white_furnace_floor(rg, orc, tmp_path):
    """Diffuse floor (albedo 0.5) under a uniform environment L, seen from
    straight above: every pixel converges to albedo x L (the environment NEE and
    the BSDF-sampled miss share the estimate through MIS)."""
    img = np.full((8, 16, 3), 0.8, np.float32)
    objects = {"floor": {"scale": [1000, 1, 1000], "mesh": {"type": "plane"}, "mat": {"color": [0.5, 0.5, 0.5]}}}
    cam = {"location": [0, 1, 0], "angle": [-90, 0, 0], "fieldOfView": 40}
    sc, ref = env_scene(rg, tmp_path, img, objects=objects, camera=cam)
    expected = 0.5 * float(ref[0, 0, 0])  # L as stored in RGBE: 204/256
    r = orc.OracleScene(sc.ptr).render(32, 32, 64, max_depth=8, seed=3)
    m = r["hdr"][..., :3]
    assert m.mean() == pytest.approx(expected, rel=0.005)
    assert np.abs(m.mean(axis=(0, 1)) - expected).max() < 0.005


def test_oracle_eye_miss_sees_environment(rg, orc, tmp_path):
    img = np.full((8, 16, 3), 0.3, np.float32)
    sc, ref = env_scene(rg, tmp_path, img, intensity=2.0)  # ref: the RGBE-quantised texels
    for shader in (5, 2, 0):
        r = orc.OracleScene(sc.ptr).render(16, 16, 4, shader=shader, seed=1)
        np.testing.assert_allclose(r["hdr"][..., :3], np.broadcast_to(ref[0, 0] * 2.0, (16, 16, 3)), rtol=1e-6)


# ---------------------------------------------------------------- cubemaps
FACE_COLOURS = [(230, 40, 40), (40, 230, 40), (40, 40, 230), (230, 230, 40), (40, 230, 230), (230, 40, 230)]


def cube_dir(tmp_path, colours=FACE_COLOURS, size=8, ext="png", sun=None):
    """Six PNG faces px nx py ny pz nz, each one flat colour (optionally a bright texel on one face)."""
    import image_codecs as ic
    d = tmp_path / "cube"
    d.mkdir(exist_ok=True)
    for k, name in enumerate(("px", "nx", "py", "ny", "pz", "nz")):
        img = np.tile(np.array(colours[k], np.int64), (size, size, 1))
        if sun is not None and sun[0] == k:
            img[sun[1], sun[2]] = (255, 255, 255)
        ic.write_png(str(d / f"{name}.{ext}"), img, 2, 8)
    return d


def test_cubemap_loads_and_looks_up_faces(rg, orc, tmp_path):
    cube_dir(tmp_path)
    doc = {"envmap": {"cubemap": "cube", "ext": "png", "intensity": 2.0}, "f": {"mesh": {"type": "plane"}}}
    (tmp_path / "cube.json").write_text(json.dumps(doc))
    sc = rg.Scene.from_json(str(tmp_path / "cube.json"))
    d = sc.desc
    assert d.envmap_cube == 1 and d.has_envmap == 0 and d.num_textures == 6
    assert len(set(d.envmap_cube_faces)) == 6
    o = orc.OracleScene(sc.ptr)
    dirs = np.array([[1, 0.1, 0.2], [-1, 0.2, -0.1], [0.1, 1, 0.3], [0.2, -1, 0.1], [0.1, 0.2, 1], [0.3, 0.1, -1]],
                    np.float32)  # camera at the origin with zero angles: view = world
    rgb, pdf = o.env_eval(dirs)
    srgb = lambda c: np.where(c <= 0.04045, c / 12.92, ((c + 0.055) / 1.055) ** 2.4)
    want = 2.0 * srgb(np.array(FACE_COLOURS) / 255.0)
    np.testing.assert_allclose(rgb, want, rtol=1e-5)
    assert np.all(pdf > 0)


def test_cubemap_pdf_normalises_and_matches_its_sampler(rg, orc, tmp_path):
    cube_dir(tmp_path, sun=(2, 3, 5))
    doc = {"envmap": {"cubemap": "cube", "ext": "png", "rotation": 25}, "f": {"mesh": {"type": "plane"}}}
    (tmp_path / "cube.json").write_text(json.dumps(doc))
    sc = rg.Scene.from_json(str(tmp_path / "cube.json"))  # keeps the description alive
    o = orc.OracleScene(sc.ptr)
    # integral of the pdf over the sphere (uniform directions)
    _, pdf = o.env_eval(random_dirs(400000, 3))
    assert pdf.mean() * 4 * np.pi == pytest.approx(1.0, rel=0.02)
    # directions drawn by the sampler carry the pdf that the lookup reports
    u = np.random.default_rng(4).random((20000, 2)).astype(np.float32)
    dirs, spdf = o.env_sample(u)
    _, lpdf = o.env_eval(dirs)
    ok = spdf > 0
    assert ok.mean() > 0.99
    assert np.mean(np.isclose(spdf[ok], lpdf[ok], rtol=1e-4)) > 0.99  # texel-boundary ties aside
    # per region of the sphere, the share of samples equals the pdf's mass there
    region = lambda v: np.argmax(np.abs(v), axis=1) * 2 + (np.take_along_axis(v, np.argmax(np.abs(v), axis=1)[:, None], 1)[:, 0] < 0)
    uni = random_dirs(400000, 5)
    _, updf = o.env_eval(uni)
    for r in range(6):
        mass = 4 * np.pi * np.mean(updf * (region(uni) == r))
        assert np.mean(region(dirs) == r) == pytest.approx(mass, abs=0.01)


def test_cubemap_white_furnace_in_the_oracle(rg, orc, tmp_path):
    cube_dir(tmp_path, colours=[(204, 204, 204)] * 6)
    doc = {"mainCamera": {"location": [0, 1, 0], "angle": [-90, 0, 0], "fieldOfView": 40},
           "envmap": {"cubemap": "cube", "ext": "png"},
           "floor": {"scale": [1000, 1, 1000], "mesh": {"type": "plane"}, "mat": {"color": [0.5, 0.5, 0.5]}}}
    (tmp_path / "f.json").write_text(json.dumps(doc))
    sc = rg.Scene.from_json(str(tmp_path / "f.json"))
    out = orc.OracleScene(sc.ptr).render(8, 8, 64, max_depth=8, seed=2)
    L = ((204 / 255 + 0.055) / 1.055) ** 2.4
    mean = out["sum"].sum(axis=(0, 1)) / out["n"].sum()
    assert np.allclose(mean, 0.5 * L, rtol=0.02), (mean, 0.5 * L)
