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


def test_noalloc_address_cache_is_keyed_by_context(rg):
    """The no-allocation A-Trous entry point caches its working array's device
    address per CUDA context id (a reset or a second context on the same
    device loads the module at another address).  The cache logic runs here
    on fake ids, with no CUDA call."""
    lib = rg.load_library()
    f = lib.rg_noalloc_cache_probe
    f.restype = C.c_int32
    f.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]
    # ctx 7 (device 0), a reset gives ctx 9 on the same device, back to 7 is a hit;
    # then 70 distinct contexts overflow the 64-entry table, which drops the oldest
    ids = [7, 7, 9, 9, 7] + list(range(100, 170)) + [7, 169]
    ids = np.array(ids, np.uint64)
    n = len(ids)
    resolved = np.zeros(n, np.int32)
    slot = np.zeros(n, np.int32)
    assert f(ids.ctypes.data, n, resolved.ctypes.data, slot.ctypes.data) == 0
    assert list(resolved[:5]) == [1, 0, 1, 0, 0]
    assert list(slot[:5]) == [1, 1, 2, 2, 1]
    assert resolved[5:75].all()  # every new context resolves once
    assert resolved[75] == 1 and slot[75] == 73  # ctx 7 was evicted; resolves afresh
    assert resolved[76] == 0 and slot[76] == slot[74]  # the newest entry is still cached
    assert f(None, -1, None, None) == rg.RG_ERR_INVALID_ARGUMENT


@pytest.mark.parametrize("kind,iparams", [(1, None), (2, [2000]), (4, [3000, 5])])
def test_cpu_scene_generator_matches_the_library(rg, orc, kind, iparams):
    """The CPU timing arm builds its scenes with oracle/libscenegen.so (the
    same generator source, host-compiled); the arrays must equal the library's."""
    import oracle
    a = rg.Scene.builtin(kind, 3, iparams)
    b = oracle.CpuScene(kind, 3, iparams)
    db = C.cast(C.c_void_p(b.ptr), C.POINTER(rg.rg_scene_desc)).contents
    da = a.desc
    n = da.num_triangles
    assert db.num_triangles == n == b.num_triangles()
    for f, w in (("positions", 9), ("normals", 9)):
        x = np.ctypeslib.as_array(getattr(da, f), shape=(n, w))
        y = np.ctypeslib.as_array(getattr(db, f), shape=(n, w))
        assert np.array_equal(x.view(np.uint32), y.view(np.uint32)), f
    assert np.array_equal(np.ctypeslib.as_array(da.tri_mesh, shape=(n,)), np.ctypeslib.as_array(db.tri_mesh, shape=(n,)))
    assert da.num_materials == db.num_materials and da.num_objects == db.num_objects
    for i in range(da.num_materials):
        assert bytes(da.materials[i]) == bytes(db.materials[i])
    assert bytes(da.camera) == bytes(db.camera)
    a.close()
    b.close()
