#!/usr/bin/env python3
"""Golden vectors from the reference renderer's OWN code.

The reference's hot-path sources (src/raygen/bvh.cpp, raycommon.cpp,
medium.cpp, bsdf.cpp of the RayGen checkout) are compiled unchanged into
oracle/_ref/libraygen_ref.so by `make -C oracle ref` (REFERENCE_ROOT names the
checkout; see oracle/Makefile and oracle/ref_harness.cpp).  This script runs
them on seeded inputs and writes the results next to itself:

  ref_rays.npz      closest-hit (TriangleBVH::intersectClosest, bvh.cpp:233-285)
                    and any-hit (intersectAny, bvh.h:63-101) of seeded view-space
                    ray batches on three scenes: the cube room (36 triangles), a
                    98,044-triangle sphere scene and the 4,014,124-triangle
                    heavy-geometry benchmark scene.  The scenes are regenerated
                    by the tests from their seeds; a SHA-256 of the flattened
                    view-space triangles pins that they are the same scenes.
  ref_sampling.npz  Halton / Cranley-Patterson values (raycommon.cpp:35-92),
                    cosineWeightedDirection, ldsPointInTriangle, and the GGX /
                    dielectric helpers of bsdf.cpp (sampleGGXVNDF, smithG1,
                    fresnelSchlick, refract, buildTangentFrame) on seeded inputs.
  ref_media.npz     HomogeneousMedium (medium.cpp) on five parameter sets:
                    transmittance, free-flight and phase sampling, phase pdf,
                    density / emission / index fields and heat-haze bending.

Only this script (run where the reference checkout exists) touches
oracle/_ref; the tests read the .npz files.  Run:  python tests/golden/make_ref_golden.py
"""
from __future__ import annotations

import ctypes as C
import hashlib
import os
import subprocess
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import oracle  # noqa: E402  (the oracle front end: scenes and flattening)
import ref_cases  # noqa: E402  (the seeded inputs, shared with the tests)

REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libraygen_ref.so")


def load_ref() -> C.CDLL:
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref"], check=True)
    lib = C.CDLL(REF_LIB)
    vp = C.c_void_p
    lib.ref_scene_create.restype = vp
    lib.ref_scene_create.argtypes = [vp, vp, C.c_int32]
    lib.ref_scene_destroy.argtypes = [vp]
    lib.ref_bvh_nodes.restype = C.c_int32
    lib.ref_bvh_nodes.argtypes = [vp]
    lib.ref_closest.argtypes = [vp, vp, C.c_int32, vp, vp]
    lib.ref_any.argtypes = [vp, vp, vp, C.c_int32, vp]
    lib.ref_lds.restype = C.c_float
    lib.ref_lds.argtypes = [C.c_int32] * 4
    lib.ref_cosine_direction.argtypes = [C.c_int32] * 4 + [vp, vp]
    lib.ref_point_in_triangle.argtypes = [C.c_int32] * 4 + [vp, vp]
    lib.ref_bsdf_probe.argtypes = [C.c_int32, vp, C.c_int32, vp]
    lib.ref_medium_create.restype = vp
    lib.ref_medium_create.argtypes = [vp]
    lib.ref_medium_destroy.argtypes = [vp]
    lib.ref_medium_probe.argtypes = [vp, C.c_int32, vp, C.c_int32, vp]
    return lib


def ray_goldens(ref) -> dict:
    out = {}
    for key, (kind, seed, params, nrays) in ref_cases.RAY_SCENES.items():
        t0 = time.time()
        sc = oracle.CpuScene(kind, seed, params)
        pos, nrm = oracle.view_triangles(sc.ptr)
        n = len(pos)
        h = ref.ref_scene_create(pos.ctypes.data, nrm.ctypes.data, n)
        rays, tmax = ref_cases.ray_batch(key, pos, nrays)
        tuv = np.zeros((nrays, 3), np.float32)
        prim = np.zeros(nrays, np.int32)
        ref.ref_closest(h, rays.ctypes.data, nrays, tuv.ctypes.data, prim.ctypes.data)
        hit = np.zeros(nrays, np.uint8)
        ref.ref_any(h, rays.ctypes.data, tmax.ctypes.data, nrays, hit.ctypes.data)
        out[f"{key}_tri_sha256"] = np.frombuffer(hashlib.sha256(pos.tobytes() + nrm.tobytes()).digest(), np.uint8)
        out[f"{key}_num_triangles"] = np.int64(n)
        out[f"{key}_rays"] = rays
        out[f"{key}_tmax"] = tmax
        out[f"{key}_prim"] = prim
        out[f"{key}_tuv"] = tuv
        out[f"{key}_any"] = hit
        print(f"{key}: {n} triangles, {ref.ref_bvh_nodes(h)} reference BVH nodes, {nrays} rays, "
              f"{(prim >= 0).mean():.3f} hit, {hit.mean():.3f} occluded ({time.time() - t0:.1f} s)")
        ref.ref_scene_destroy(h)
        sc.close()
    return out


def sampling_goldens(ref) -> dict:
    out = {}
    lds_in = ref_cases.lds_inputs()
    out["lds_in"] = lds_in
    out["lds_out"] = np.array([ref.ref_lds(*map(int, r)) for r in lds_in], np.float32)
    cos_in = ref_cases.cosine_inputs()
    o = np.zeros((len(cos_in), 3), np.float32)
    for i, r in enumerate(cos_in):
        nrm = np.ascontiguousarray(r[4:7], np.float32)
        ref.ref_cosine_direction(int(r[0]), int(r[1]), int(r[2]), int(r[3]), nrm.ctypes.data, o[i].ctypes.data)
    out["cosine_in"], out["cosine_out"] = cos_in, o
    tri_in = ref_cases.triangle_point_inputs()
    o = np.zeros((len(tri_in), 3), np.float32)
    for i, r in enumerate(tri_in):
        t9 = np.ascontiguousarray(r[4:13], np.float32)
        ref.ref_point_in_triangle(int(r[0]), int(r[1]), int(r[2]), int(r[3]), t9.ctypes.data, o[i].ctypes.data)
    out["tripoint_in"], out["tripoint_out"] = tri_in, o
    for which, name in enumerate(ref_cases.BSDF_PROBES):
        x = ref_cases.bsdf_inputs(which)
        y = np.zeros((len(x), ref_cases.BSDF_OUT_WIDTH[which]), np.float32)
        ref.ref_bsdf_probe(which, x.ctypes.data, len(x), y.ctypes.data)
        out[f"{name}_in"], out[f"{name}_out"] = x, y
    return out


def media_goldens(ref) -> dict:
    out = {}
    for name, params in ref_cases.MEDIA.items():
        vec = ref_cases.medium_vector(params)
        m = ref.ref_medium_create(vec.ctypes.data)
        out[f"{name}_params"] = vec
        for which, probe in enumerate(ref_cases.MEDIUM_PROBES):
            x = ref_cases.medium_inputs(which, name)
            if x is None:
                continue
            y = np.zeros((len(x), ref_cases.MEDIUM_OUT_WIDTH[which]), np.float32)
            ref.ref_medium_probe(m, which, x.ctypes.data, len(x), y.ctypes.data)
            out[f"{name}_{probe}_in"], out[f"{name}_{probe}_out"] = x, y
        ref.ref_medium_destroy(m)
    return out


def main():
    ref = load_ref()
    np.savez_compressed(os.path.join(HERE, "ref_sampling.npz"), **sampling_goldens(ref))
    np.savez_compressed(os.path.join(HERE, "ref_media.npz"), **media_goldens(ref))
    np.savez_compressed(os.path.join(HERE, "ref_rays.npz"), **ray_goldens(ref))
    for f in ("ref_sampling.npz", "ref_media.npz", "ref_rays.npz"):
        print(f, os.path.getsize(os.path.join(HERE, f)), "bytes")


if __name__ == "__main__":
    main()
