"""C-ABI surface checks that need no GPU: exports, defaults, procedural scenes, errors."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "raygen_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(rg_[a-z_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol(rg):
    lib = rg.load_library()
    names = header_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_settings_defaults_match_reference(rg):
    s = rg.default_settings_c()
    # RendererSettings defaults (rayrenderer.h:98-153, linux build)
    assert (s.resolution_width, s.resolution_height, s.samples, s.threads, s.shader_provider) == (800, 600, 100, 1, 5)
    assert s.enable_antialias == 1 and s.enable_color_sampling == 1 and s.enable_denoise == 0
    assert s.denoise_levels == 5 and abs(s.denoise_sigma_color - 0.4) < 1e-7 and s.denoise_sigma_normal == 128.0
    assert abs(s.firefly_clamp - 10.0) < 1e-7 and s.adaptive_base_samples == 4
    assert abs(s.adaptive_threshold - 0.02) < 1e-7
    assert s.max_depth == 32 and s.rr_depth == 3 and s.seed == 1
    assert np.allclose(list(s.back_color), [0.2, 0.19, 0.18, 0.0])
    py = rg.RendererSettings().to_c()
    for f, _ in rg.rg_settings._fields_:
        a, b = getattr(s, f), getattr(py, f)
        if not isinstance(a, (int, float)):
            a, b = list(a), list(b)
        assert np.allclose(a, b), f


def test_cube_room_scene(rg):
    sc = rg.Scene.builtin(1, 1)
    d = sc.desc
    assert d.num_triangles == 36 and d.num_objects == 6 and d.num_meshes == 6
    pos, nrm, tm = sc.arrays()
    assert pos.shape == (36, 9)
    assert np.allclose(np.linalg.norm(nrm.reshape(-1, 3), axis=1), 1.0, atol=1e-6)
    mats = [d.materials[i] for i in range(d.num_materials)]
    assert sum(1 for m in mats if m.emission > 0) == 1
    assert abs(d.camera.field_of_view - 40.0) < 1e-6
    sc.close()


def test_heavy_scene_counts(rg):
    sc = rg.Scene.builtin(2, 7, [2000])
    d = sc.desc
    f = round((2000 / 20) ** 0.5)
    assert d.num_triangles == 4 * 20 * f * f + 12 + 32
    emitters = sum(1 for i in range(d.num_materials) if d.materials[i].emission > 0)
    assert emitters == 16
    pos, _, _ = sc.arrays()
    assert np.isfinite(pos).all()
    sc.close()


def test_sphere_mesh_is_watertight(rg):
    """Every edge of the displaced geodesic sphere is shared by exactly two triangles."""
    sc = rg.Scene.builtin(4, 3, [500, 1])
    pos, _, tm = sc.arrays()
    sphere = pos[tm == tm.max()].reshape(-1, 3, 3)
    keys = {}
    for t in sphere:
        for a, b in ((0, 1), (1, 2), (2, 0)):
            e = tuple(sorted((tuple(t[a]), tuple(t[b]))))
            keys[e] = keys.get(e, 0) + 1
    assert set(keys.values()) == {2}
    sc.close()


def test_invalid_builtin_kind(rg):
    with pytest.raises(rg.RayGenError) as e:
        rg.Scene.builtin(99, 1)
    assert e.value.code == rg.RG_ERR_INVALID_ARGUMENT


def test_scene_free_rejects_unknown_pointer(rg):
    lib = rg.load_library()
    d = rg.rg_scene_desc()
    assert lib.rg_scene_free(C.pointer(d)) == rg.RG_ERR_INVALID_ARGUMENT


def test_null_arguments_are_rejected(rg):
    lib = rg.load_library()
    assert lib.rg_create(None, None) == rg.RG_ERR_INVALID_ARGUMENT
    assert lib.rg_render(None) == rg.RG_ERR_INVALID_ARGUMENT
    assert lib.rg_set_scene(None, None) == rg.RG_ERR_INVALID_ARGUMENT
    assert lib.rg_destroy(None) == rg.RG_ERR_INVALID_ARGUMENT


def test_version_string(rg):
    assert "raygen" in rg.version()
