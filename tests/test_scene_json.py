"""Scene JSON loader (rg_load_scene_json) on the host: schema, primitives,
transforms, materials, media, .obj/.mtl and .mesh readers.

Follows the reference loader: sceneloader.cpp:101-883 (keys, material and
medium readers, named-material scopes), polygons.cpp:13-288 (primitives),
rayrenderer.cpp:237-363 (transform stack, mesh-less lights), objreader.cpp
(OBJ), meshloader.cpp (binary .mesh).  No GPU needed.
"""
import json
import struct

import numpy as np
import pytest

from scenes import JSON_ROOM as CUBE_ROOM


def load(rg, tmp_path, text, name="scene.json"):
    p = tmp_path / name
    p.write_text(text)
    return rg.Scene.from_json(str(p))


def tri_arrays(sc):
    pos, nrm, tm = sc.arrays()[:3]
    return np.asarray(pos).reshape(-1, 3, 3), np.asarray(nrm).reshape(-1, 3, 3), np.asarray(tm)


def mesh_object(sc):
    d = sc.desc
    return np.array([d.mesh_object[i] for i in range(d.num_meshes)])


def material_of_triangles(sc):
    d = sc.desc
    _, _, tm = tri_arrays(sc)
    mo = mesh_object(sc)
    return np.array([d.objects[mo[m]].material for m in tm])


def test_cube_room_schema(rg, tmp_path):
    sc = load(rg, tmp_path, CUBE_ROOM)
    d = sc.desc
    # 6 planes x 2 + cube 12 triangles, one object (and one mesh) per JSON object, DFS file order
    assert d.num_triangles == 24 and d.num_objects == 7 and d.num_meshes == 7
    assert list(d.camera.location) == pytest.approx([0, 0.5, 6])
    assert list(d.camera.angle) == pytest.approx([-5, 0, 0])
    assert d.camera.field_of_view == pytest.approx(60) and d.camera.exposure == pytest.approx(1.5)
    pos, nrm, tm = tri_arrays(sc)
    assert list(tm) == [0, 0, 1, 1, 2, 2, 3, 3, 4, 4, 5, 5] + [6] * 12
    # every wall normal points into the room (towards the origin)
    for m in range(6):
        c = pos[tm == m].reshape(-1, 3).mean(0)
        n = nrm[tm == m].reshape(-1, 3).mean(0)
        assert np.dot(n, -c) > 0, f"mesh {m} faces outward"
    # plane extents: scale 6 -> +-3 ; lamp at y=2.9 facing down
    floor = pos[tm == 1].reshape(-1, 3)
    assert floor[:, 0].min() == pytest.approx(-3) and floor[:, 2].max() == pytest.approx(3)
    assert np.allclose(floor[:, 1], -3)
    lamp = nrm[tm == 0].reshape(-1, 3)
    assert np.allclose(lamp, [0, -1, 0], atol=1e-6)
    # left wall at x=-3 with normal +x (angle z=-90 maps +Y to +X)
    assert np.allclose(pos[tm == 3].reshape(-1, 3)[:, 0], -3, atol=1e-5)
    assert np.allclose(nrm[tm == 3].reshape(-1, 3), [1, 0, 0], atol=1e-6)
    # back wall (angle x=90 maps +Y to +Z)
    assert np.allclose(nrm[tm == 5].reshape(-1, 3), [0, 0, 1], atol=1e-6)


def test_materials_and_colours(rg, tmp_path):
    sc = load(rg, tmp_path, CUBE_ROOM)
    d = sc.desc
    mats = [d.materials[d.objects[o].material] for o in range(d.num_objects)]
    lamp, floor, _, left, right, back, box = mats
    assert lamp.emission == pytest.approx(8) and list(lamp.color) == pytest.approx([1, 1, 240 / 255])
    # named material from _materials, defaults elsewhere (material.h:27-52)
    assert list(floor.color) == pytest.approx([0xcc / 255, 0xbb / 255, 0xaa / 255]) and floor.diffuse == pytest.approx(0.9)
    assert floor.roughness == pytest.approx(0.5) and floor.refraction_ratio == pytest.approx(1.45)
    assert list(back.color) == list(floor.color)
    assert list(left.color) == pytest.approx([1, 0x55 / 255, 0x55 / 255]) and left.diffuse == pytest.approx(0.8)
    assert list(right.color) == pytest.approx([0.3, 1.0, 0.3])
    assert box.glossy == pytest.approx(0.3) and box.roughness == pytest.approx(0.2)


def test_colour_string_forms(rg, tmp_path):
    def colour(s):
        sc = load(rg, tmp_path, json.dumps({"o": {"mesh": {"type": "plane"}, "mat": {"color": s}}}))
        return list(sc.desc.materials[0].color)

    assert colour("#102030") == pytest.approx([0x10 / 255, 0x20 / 255, 0x30 / 255])
    assert colour("102030") == pytest.approx([0x10 / 255, 0x20 / 255, 0x30 / 255])
    assert colour("#10203040") == pytest.approx([0x10 / 255, 0x20 / 255, 0x30 / 255])
    # 3-digit form: the hex value times two, read as a packed 0xRRGGBB word
    v = 0xABC * 2
    assert colour("#abc") == pytest.approx([(v >> 16 & 255) / 255, (v >> 8 & 255) / 255, (v & 255) / 255])
    assert colour("#1") == pytest.approx([0.8, 0.8, 0.8])  # shorter than 3 -> default kept


def test_named_material_scopes(rg, tmp_path):
    text = json.dumps({
        "_materials": {"m": {"color": [1, 0, 0]}},
        "a": {"_materials": {"m": {"color": [0, 1, 0]}},
              "inner": {"mesh": {"type": "plane"}, "mat": "m"}},
        "b": {"mesh": {"type": "plane"}, "mat": "m"},
        "c": {"mesh": {"type": "plane"}, "mat": "missing"},
    })
    sc = load(rg, tmp_path, text)
    d = sc.desc
    cols = [list(d.materials[d.objects[o].material].color) for o in range(d.num_objects)]
    assert cols == [pytest.approx([0, 1, 0]), pytest.approx([1, 0, 0]), pytest.approx([0.8, 0.8, 0.8])]


def test_hierarchy_transform_and_visibility(rg, tmp_path):
    text = json.dumps({
        "parent": {"location": [10, 0, 0], "angle": [0, 90, 0], "scale": [2, 2, 2],
                   "mesh": {"type": "plane"},
                   "child": {"location": [1, 0, 0], "mesh": {"type": "plane"}},
                   "hidden": {"visible": False, "mesh": {"type": "cube"},
                              "grandchild": {"mesh": {"type": "cube"}}}},
    })
    sc = load(rg, tmp_path, text)
    pos, _, tm = tri_arrays(sc)
    assert sc.desc.num_triangles == 4  # the invisible subtree is skipped
    child = pos[tm == 1].reshape(-1, 3)
    # child origin (1,0,0) -> scale 2 -> rotate y 90 (x -> -z) -> translate 10: centre (10, 0, -2)
    assert child.mean(0) == pytest.approx([10, 0, -2], abs=1e-5)
    assert np.ptp(child[:, 0]) == pytest.approx(2, abs=1e-5)


def test_point_light_from_meshless_emitter(rg, tmp_path):
    text = json.dumps({
        "lamp": {"location": [1, 2, 3], "mat": {"emission": 5, "color": [1, 0.5, 0.25]}},
        "floor": {"mesh": {"type": "plane"}},
        "dark": {"location": [0, 1, 0]},
    })
    sc = load(rg, tmp_path, text)
    d = sc.desc
    assert d.num_point_lights == 1 and d.num_triangles == 2
    pl = d.point_lights[0]
    assert list(pl.position) == pytest.approx([1, 2, 3])
    assert list(pl.normal) == pytest.approx([0, 1, 0])
    m = d.materials[pl.material]
    assert m.emission == pytest.approx(5) and list(m.color) == pytest.approx([1, 0.5, 0.25])


def test_media_global_and_interior(rg, tmp_path):
    text = json.dumps({
        "medium": {"sigma_a": [0.01, 0.02, 0.03], "sigma_s": {"x": 0.1, "y": 0.2, "z": 0.3}, "g": 0.4},
        "water": {"mesh": {"type": "cube"},
                  "medium": {"sigma_a": [0.5, 0.1, 0.05], "emission": [0.1, 0, 0], "density": 2}},
    })
    sc = load(rg, tmp_path, text)
    d = sc.desc
    assert d.num_media == 2 and d.global_medium == 0
    g = d.media[0]
    assert list(g.sigma_a) == pytest.approx([0.01, 0.02, 0.03]) and list(g.sigma_s) == pytest.approx([0.1, 0.2, 0.3])
    assert g.g == pytest.approx(0.4) and g.density == pytest.approx(1.0)
    assert d.objects[0].interior_medium == 1
    w = d.media[1]
    assert list(w.sigma_e) == pytest.approx([0.1, 0, 0]) and w.density == pytest.approx(2)


@pytest.mark.parametrize("kind,params,ntri", [
    ("plane", {}, 2), ("cube", {}, 12),
    ("sphere", {}, 16 * 32 * 2), ("sphere", {"stacks": 4, "slices": 6, "radius": 2}, 4 * 6 * 2),
    ("cone", {}, 32 * 4), ("cone", {"radiusEnd": 0, "slices": 8}, 8 * 3),
])
def test_primitive_meshes(rg, tmp_path, kind, params, ntri):
    sc = load(rg, tmp_path, json.dumps({"o": {"mesh": dict(type=kind, **params)}}))
    pos, nrm, _ = tri_arrays(sc)
    assert sc.desc.num_triangles == ntri
    assert np.allclose(np.linalg.norm(nrm, axis=2), 1.0, atol=1e-5)
    if kind == "sphere":
        r = params.get("radius", 1)
        assert np.allclose(np.linalg.norm(pos, axis=2), r, atol=1e-5)
        # smooth normals are radial
        assert np.allclose(nrm * r, pos, atol=1e-4)
    if kind == "cube":
        assert np.allclose(np.abs(pos).max(), 0.5)


def test_obj_reader(rg, tmp_path):
    (tmp_path / "m.mtl").write_text("newmtl red\nKd 0.9 0.1 0.1\nTf 0.5 0.5 0.5\nnewmtl blue\nKd 0.1 0.1 0.9\n")
    (tmp_path / "m.obj").write_text(
        "# test\nmtllib m.mtl\n"
        "v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nvt 0 0\nvt 1 0\nvt 1 1\nvt 0 1\nvn 0 0 1\n"
        "o quad\nusemtl red\nf 1/1/1 2/2/1 3/3/1 4/4/1\n"
        "g second part\nusemtl blue\nf -4 -2 -1\n"
        "o third\nusemtl override\nf 1 2 3\n"
        "o nomtl\nf 1 3 4\n")
    text = json.dumps({"_materials": {"override": {"color": [0, 1, 0], "glossy": 1}},
                       "model": {"location": [0, 0, -1], "mat": {"color": [0.2, 0.3, 0.4]}, "mesh": "m.obj"}})
    sc = load(rg, tmp_path, text)
    d = sc.desc
    pos, nrm, tm = tri_arrays(sc)
    assert d.num_triangles == 5 and d.num_objects == 4
    # quad fan (v0, v1, v2), (v0, v2, v3), moved by the parent transform
    assert pos[0].tolist() == [[0, 0, -1], [1, 0, -1], [1, 1, -1]]
    assert pos[1].tolist() == [[0, 0, -1], [1, 1, -1], [0, 1, -1]]
    assert np.allclose(nrm[0], [0, 0, 1])
    uv = np.ctypeslib.as_array(d.uvs, shape=(d.num_triangles, 6)).reshape(-1, 3, 2)
    assert uv[0].tolist() == [[0, 1], [1, 1], [1, 0]]  # v flipped on read
    mats = [d.materials[d.objects[o].material] for o in range(d.num_objects)]
    # .mtl defaults: Kd -> colour, Tf -> transparency 1 - mean(Tf), other fields at Material defaults
    assert list(mats[0].color) == pytest.approx([0.9, 0.1, 0.1]) and mats[0].transparency == pytest.approx(0.5)
    assert mats[0].diffuse == pytest.approx(0.8)
    # transparency carries over between .mtl entries (not reset by newmtl)
    assert list(mats[1].color) == pytest.approx([0.1, 0.1, 0.9]) and mats[1].transparency == pytest.approx(0.5)
    # scene _materials override by the usemtl name
    assert list(mats[2].color) == pytest.approx([0, 1, 0]) and mats[2].glossy == pytest.approx(1)
    # no usemtl -> the loading object's material as it stands when "mesh" is read
    assert list(mats[3].color) == pytest.approx([0.2, 0.3, 0.4])
    late = json.dumps({"model": {"mesh": "m.obj", "mat": {"color": [0.2, 0.3, 0.4]}}})
    d2 = load(rg, tmp_path, late, "late.json").desc
    assert list(d2.materials[d2.objects[3].material].color) == pytest.approx([0.8, 0.8, 0.8])
    # face without normals -> face normal
    assert np.allclose(nrm[4], [0, 0, 1])


def test_obj_missing_file_adds_no_geometry(rg, tmp_path):
    sc = load(rg, tmp_path, json.dumps({"a": {"mesh": "nothere.obj"}, "b": {"mesh": {"type": "plane"}}}))
    assert sc.desc.num_triangles == 2


def write_mesh(path, verts, normals=None, uvs=None, indexes=None, ver=0x0105):
    flags = 0x8
    if normals is not None:
        flags |= 0x2
    if uvs is not None:
        flags |= 0x4
    vc = len(verts)
    ic = 0 if indexes is None else len(indexes)
    body = np.asarray(verts, np.float32).tobytes()
    if normals is not None:
        body += np.asarray(normals, np.float32).tobytes()
    if uvs is not None:
        body += np.asarray(uvs, np.float32).tobytes()
    if indexes is not None:
        body += np.asarray(indexes, np.uint32).tobytes()
    header_len = 128
    head = struct.pack("<IHHI", 0x6873656D, ver, flags, header_len) + struct.pack("<5I", vc, 1, ic, 0, 0)
    path.write_bytes(head + b"\0" * (header_len - len(head)) + body)


def test_mesh_file_reader(rg, tmp_path):
    v = [[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]]
    n = [[0, 0, 1]] * 4
    write_mesh(tmp_path / "quad.mesh", v, n, uvs=[[0, 0], [1, 0], [1, 1], [0, 1]], indexes=[0, 1, 2, 0, 2, 3])
    write_mesh(tmp_path / "soup.mesh", [v[0], v[1], v[2]])
    sc = load(rg, tmp_path, json.dumps({"a": {"mesh": ["quad.mesh", "soup.mesh"], "scale": [2, 2, 2]}}))
    d = sc.desc
    assert d.num_triangles == 3 and d.num_meshes == 2 and d.num_objects == 1
    pos, nrm, tm = tri_arrays(sc)
    assert list(tm) == [0, 0, 1]
    assert pos[1].tolist() == [[0, 0, 0], [2, 2, 0], [0, 2, 0]]
    assert np.allclose(nrm, [0, 0, 1])  # given normals, then the face normal of the soup
    # truncated file -> a clear error
    (tmp_path / "bad.mesh").write_bytes((tmp_path / "quad.mesh").read_bytes()[:150])
    with pytest.raises(RuntimeError, match="malformed .mesh"):
        load(rg, tmp_path, json.dumps({"a": {"mesh": "bad.mesh"}}), "bad.json")


def test_errors(rg, tmp_path):
    with pytest.raises(rg.RayGenError, match="parse error") as e:
        load(rg, tmp_path, '{ "a": { "mesh": [1, 2 } }', "broken.json")
    assert e.value.code == rg.RG_ERR_PARSE
    with pytest.raises(rg.RayGenError) as e:
        rg.Scene.from_json(str(tmp_path / "does_not_exist.json"))
    assert e.value.code == rg.RG_ERR_IO
    with pytest.raises(rg.RayGenError, match="toba") as e:
        load(rg, tmp_path, json.dumps({"w": {"_bundle": "x.toba"}}), "bundle.json")
    assert e.value.code == rg.RG_ERR_UNSUPPORTED
    # an unterminated root object is closed at the end of the input
    sc = load(rg, tmp_path, '{ "a": { "mesh": { "type": "plane" } }\n// }\n', "open.json")
    assert sc.desc.num_triangles == 2


def test_branch_scenes_take_their_branches(rg, tmp_path):
    """The scenes of the device branch-parity tests (test_gpu_parity_configs.py)
    load with the materials, lights and camera those tests rely on (no GPU)."""
    from test_gpu_parity_configs import BRANCH_SCENES
    for name, doc in BRANCH_SCENES.items():
        p = tmp_path / f"{name}.json"
        p.write_text(json.dumps(doc))
        d = rg.Scene.from_json(str(p)).desc
        mats = [d.materials[i] for i in range(d.num_materials)]
        cam = d.camera
        if name == "anisotropic_ggx":
            assert sum(abs(mm.anisotropy) > 0.4 for mm in mats) == 3 and any(mm.aniso_rotation != 0 for mm in mats)
        if name == "rough_dielectric":
            assert sum(mm.refraction > 0.5 and mm.roughness > 0.1 for mm in mats) == 3
        if name == "dispersion":
            assert sum(mm.chroma_dispersion > 0 for mm in mats) == 2
        if name.startswith("thin_lens"):
            assert cam.depth_of_field > 0 and cam.aperture > 0
            assert cam.aperture_blades == (6 if "blades" in name else 0)
        if name == "thin_lens_blades_spot":
            assert d.num_point_lights == 2
            assert sum(mm.spot_range > 0 for mm in mats) == 1
