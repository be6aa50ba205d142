"""TEST INFRASTRUCTURE ONLY: ctypes front end of the CPU oracle (rg_oracle.cpp).

Loaded by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline /
reference arm; never by the product path.  The oracle restates RayGen's
shader-5 renderer on the CPU (see the header of rg_oracle.cpp for the
reference files it follows and the documented deviations).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


class orc_settings(C.Structure):
    _fields_ = [
        ("width", C.c_int32), ("height", C.c_int32), ("spp", C.c_int32), ("shader", C.c_int32),
        ("antialias", C.c_int32), ("color_sampling", C.c_int32), ("denoise", C.c_int32),
        ("denoise_levels", C.c_int32),
        ("sigma_color", C.c_float), ("sigma_normal", C.c_float), ("sigma_depth", C.c_float),
        ("denoise_intensity", C.c_float), ("firefly_clamp", C.c_float),
        ("adaptive", C.c_int32), ("adaptive_base", C.c_int32), ("adaptive_mode", C.c_int32),
        ("adaptive_threshold", C.c_float),
        ("world_color", C.c_float * 3), ("back_color", C.c_float * 4),
        ("seed", C.c_uint32), ("max_depth", C.c_int32), ("rr_depth", C.c_int32),
        ("light_pick_fix", C.c_int32), ("threads", C.c_int32), ("mix_tree", C.c_int32),
    ]


_libs = {}


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def load(fast: bool = False) -> C.CDLL:
    name = "liboracle_fast.so" if fast else "liboracle.so"
    if name in _libs:
        return _libs[name]
    path = os.path.join(HERE, name)
    if not os.path.exists(path):
        build()
    lib = C.CDLL(path)
    P = C.POINTER
    f = P(C.c_float)
    lib.orc_scene_create.restype = C.c_void_p
    lib.orc_scene_create.argtypes = [C.c_void_p, C.c_int32]
    lib.orc_scene_destroy.argtypes = [C.c_void_p]
    lib.orc_bvh_nodes.restype = C.c_int32
    lib.orc_bvh_nodes.argtypes = [C.c_void_p]
    for nm in ("orc_closest", "orc_closest_brute"):
        getattr(lib, nm).argtypes = [C.c_void_p, f, C.c_int32, f, P(C.c_int32)]
    lib.orc_any.argtypes = [C.c_void_p, f, f, C.c_int32, C.c_int32, P(C.c_uint8)]
    lib.orc_render.restype = C.c_int32
    lib.orc_render.argtypes = [C.c_void_p, P(orc_settings), P(C.c_double), P(C.c_double), P(C.c_int32), f, f, f, f, f]
    lib.orc_denoise.argtypes = [C.c_int32, C.c_int32, f, f, f, f, f, C.c_int32, C.c_float, C.c_float, C.c_float,
                                C.c_float, f]
    lib.orc_tonemap.argtypes = [C.c_int32, C.c_int32, f, f]
    lib.orc_lds.restype = C.c_float
    lib.orc_lds.argtypes = [C.c_uint32] * 5 + [C.c_int32]
    lib.orc_prng.restype = C.c_float
    lib.orc_prng.argtypes = [C.c_uint32] * 5 + [C.c_int32, C.c_int32]
    lib.orc_phase_pdf.restype = C.c_float
    lib.orc_phase_pdf.argtypes = [C.c_float, C.c_float]
    lib.orc_sample_phase.argtypes = [C.c_float, C.c_float, C.c_float, f]
    lib.orc_env_eval.argtypes = [C.c_void_p, f, C.c_int32, f, f]
    lib.orc_bloom.argtypes = [C.c_int32, C.c_int32, f] + [C.c_float] * 5
    lib.orc_env_sample.argtypes = [C.c_void_p, f, C.c_int32, f, f]
    lib.orc_medium_eval.argtypes = [C.c_void_p, C.c_int32, f, C.c_int32, f]
    lib.orc_medium_bend.argtypes = [C.c_void_p, C.c_int32, f, C.c_int32, f]
    lib.orc_volume_nee.argtypes = [C.c_void_p, f, f, C.c_int32, C.c_uint32, f, f, f, P(C.c_uint8)]
    lib.orc_num_volume_lights.restype = C.c_int32
    lib.orc_num_volume_lights.argtypes = [C.c_void_p]
    vp = C.c_void_p
    lib.orc_bsdf_probe.argtypes = [C.c_int32, vp, C.c_int32, vp]
    lib.orc_cosine_direction.argtypes = [C.c_int32] * 4 + [vp, vp]
    lib.orc_point_in_triangle.argtypes = [C.c_int32] * 4 + [vp, vp]
    lib.orc_view_triangles.argtypes = [vp, vp, vp]
    lib.orc_num_triangles.restype = C.c_int32
    lib.orc_num_triangles.argtypes = [vp]
    lib.orc_medium_probe.argtypes = [vp, C.c_int32, C.c_int32, vp, C.c_int32, vp]
    _libs[name] = lib
    return lib


# Output widths of the probes (the reference harness uses the same layouts).
BSDF_OUT_WIDTH = (3, 1, 1, 3, 6)
MEDIUM_OUT_WIDTH = (3, 1, 3, 1, 5, 6)


def bsdf_probe(which: int, x) -> np.ndarray:
    """sampleGGXVNDF / smithG1 / fresnelSchlick / refract / buildTangentFrame rows."""
    lib = load()
    x = np.ascontiguousarray(x, np.float32)
    y = np.zeros((len(x), BSDF_OUT_WIDTH[which]), np.float32)
    lib.orc_bsdf_probe(which, x.ctypes.data, len(x), y.ctypes.data)
    return y


def lds_probe(rows) -> np.ndarray:
    """LDS value of rows (x, y, sample, dim) with seed 1."""
    lib = load()
    return np.array([lib.orc_lds(int(r[0]), int(r[1]), 1 << 16, int(r[2]), 1, int(r[3])) for r in rows], np.float32)


def cosine_probe(rows) -> np.ndarray:
    """cosineWeightedDirection on LDS dims dim, dim+1 of rows (x, y, sample, dim, n xyz)."""
    lib = load()
    out = np.zeros((len(rows), 3), np.float32)
    for i, r in enumerate(rows):
        nrm = np.ascontiguousarray(r[4:7], np.float32)
        lib.orc_cosine_direction(int(r[0]), int(r[1]), int(r[2]), int(r[3]), nrm.ctypes.data, out[i].ctypes.data)
    return out


def triangle_point_probe(rows) -> np.ndarray:
    """ldsPointInTriangle on LDS dims dim, dim+1 of rows (x, y, sample, dim, triangle 9)."""
    lib = load()
    out = np.zeros((len(rows), 3), np.float32)
    for i, r in enumerate(rows):
        t9 = np.ascontiguousarray(r[4:13], np.float32)
        lib.orc_point_in_triangle(int(r[0]), int(r[1]), int(r[2]), int(r[3]), t9.ctypes.data, out[i].ctypes.data)
    return out


def view_triangles(desc_ptr):
    """The flattened view-space triangles (positions, vertex normals; n x 9 each)
    in the reference's DFS order, as the oracle flattens the scene."""
    o = OracleScene(desc_ptr)
    try:
        return o.view_triangles()
    finally:
        o.close()


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class CpuScene:
    """A seeded procedural scene (rg_scene_builtin's kinds) built on the CPU by
    libscenegen.so, for the CPU-only timing arm; `ptr` is an rg_scene_desc*."""

    def __init__(self, kind: int, seed: int = 1, iparams=None):
        path = os.path.join(HERE, "libscenegen.so")
        if not os.path.exists(path):
            build()
        self.lib = C.CDLL(path)
        self.lib.og_scene_builtin.restype = C.c_int32
        self.lib.og_scene_builtin.argtypes = [C.c_int32, C.c_uint32, C.POINTER(C.c_int32), C.c_int32,
                                              C.POINTER(C.c_void_p)]
        self.lib.og_scene_free.restype = C.c_int32
        self.lib.og_scene_free.argtypes = [C.c_void_p]
        ip = (C.c_int32 * max(1, len(iparams or [])))(*(iparams or [0]))
        out = C.c_void_p()
        rc = self.lib.og_scene_builtin(kind, seed, ip, len(iparams or []), C.byref(out))
        if rc != 0:
            raise RuntimeError(f"og_scene_builtin({kind}) failed: {rc}")
        self.ptr = out.value

    def num_triangles(self) -> int:
        # rg_scene_desc starts with int32 num_triangles
        return C.cast(self.ptr, C.POINTER(C.c_int32))[0]

    def close(self):
        if self.ptr:
            self.lib.og_scene_free(self.ptr)
            self.ptr = None


class OracleScene:
    """CPU restatement of the flattened scene + reference BVH (16 bins by default)."""

    def __init__(self, desc_ptr, bins: int = 16, fast: bool = False):
        self.lib = load(fast)
        self.h = self.lib.orc_scene_create(C.cast(desc_ptr, C.c_void_p), bins)

    def close(self):
        if self.h:
            self.lib.orc_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def view_triangles(self):
        n = self.lib.orc_num_triangles(self.h)
        pos = np.zeros((n, 9), np.float32)
        nrm = np.zeros((n, 9), np.float32)
        self.lib.orc_view_triangles(self.h, pos.ctypes.data, nrm.ctypes.data)
        return pos, nrm

    def medium_probe(self, m: int, which: int, x) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float32)
        y = np.zeros((len(x), MEDIUM_OUT_WIDTH[which]), np.float32)
        self.lib.orc_medium_probe(self.h, m, which, x.ctypes.data, len(x), y.ctypes.data)
        return y

    def bvh_nodes(self) -> int:
        return self.lib.orc_bvh_nodes(self.h)

    def closest(self, rays, brute: bool = False):
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 6)
        n = rays.shape[0]
        tuv = np.empty((n, 3), np.float32)
        prim = np.empty(n, np.int32)
        fn = self.lib.orc_closest_brute if brute else self.lib.orc_closest
        fn(self.h, _fp(rays), n, _fp(tuv), prim.ctypes.data_as(C.POINTER(C.c_int32)))
        return tuv, prim

    def any(self, rays, tmax, predicate: int = 0):
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 6)
        tmax = np.ascontiguousarray(tmax, np.float32).reshape(-1)
        n = rays.shape[0]
        out = np.empty(n, np.uint8)
        self.lib.orc_any(self.h, _fp(rays), _fp(tmax), n, predicate, out.ctypes.data_as(C.POINTER(C.c_uint8)))
        return out.astype(bool)

    def env_eval(self, dirs):
        """(radiance n x 3, pdf n) of the environment map for view-space directions n x 3."""
        d = np.ascontiguousarray(dirs, np.float32).reshape(-1, 3)
        rgb = np.zeros((d.shape[0], 3), np.float32)
        pdf = np.zeros(d.shape[0], np.float32)
        self.lib.orc_env_eval(self.h, _fp(d), d.shape[0], _fp(rgb), _fp(pdf))
        return rgb, pdf

    def medium_eval(self, medium, points):
        """Camera-space points n x 3 -> n x 5 (density, emission rgb, ior) of medium `medium`."""
        pts = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
        out = np.zeros((pts.shape[0], 5), np.float32)
        self.lib.orc_medium_eval(self.h, medium, _fp(pts), pts.shape[0], _fp(out))
        return out

    def medium_bend(self, medium, rays):
        """Rays n x 7 (origin, direction, length) -> bent rays n x 6."""
        r = np.ascontiguousarray(rays, np.float32).reshape(-1, 7)
        out = np.zeros((r.shape[0], 6), np.float32)
        self.lib.orc_medium_bend(self.h, medium, _fp(r), r.shape[0], _fp(out))
        return out

    def volume_nee(self, hit, normal, n, seed=1):
        """n volume-light NEE draws at a camera-space point: (dir n x 3, pdf n, Le n x 3, ok n)."""
        h = np.ascontiguousarray(hit, np.float32).reshape(3)
        nn = np.ascontiguousarray(normal, np.float32).reshape(3)
        d = np.zeros((n, 3), np.float32)
        pdf = np.zeros(n, np.float32)
        le = np.zeros((n, 3), np.float32)
        ok = np.zeros(n, np.uint8)
        self.lib.orc_volume_nee(self.h, _fp(h), _fp(nn), n, seed, _fp(d), _fp(pdf), _fp(le),
                                ok.ctypes.data_as(C.POINTER(C.c_uint8)))
        return d, pdf, le, ok.astype(bool)

    def num_volume_lights(self):
        return self.lib.orc_num_volume_lights(self.h)

    def env_sample(self, u):
        """Luminance-importance samples: u n x 2 in [0,1) -> (directions n x 3, pdf n)."""
        uu = np.ascontiguousarray(u, np.float32).reshape(-1, 2)
        d = np.zeros((uu.shape[0], 3), np.float32)
        pdf = np.zeros(uu.shape[0], np.float32)
        self.lib.orc_env_sample(self.h, _fp(uu), uu.shape[0], _fp(d), _fp(pdf))
        return d, pdf

    def render(self, width, height, spp, shader=5, seed=1, max_depth=32, rr_depth=3, threads=None,
               mix_tree=False, antialias=True, color_sampling=True, denoise=False, denoise_levels=5,
               sigma_color=0.4, sigma_normal=128.0, sigma_depth=0.1, denoise_intensity=1.0,
               firefly_clamp=10.0, adaptive=False, adaptive_base=4, adaptive_mode=1,
               adaptive_threshold=0.02, light_pick_fix=False, world_color=(0.1, 0.095, 0.09),
               back_color=(0.2, 0.19, 0.18, 0.0)):
        """Returns dict with sum/sumsq (H,W,3 float64), n (H,W), hdr/ldr (H,W,4) and guides."""
        s = orc_settings()
        s.width, s.height, s.spp, s.shader = width, height, spp, shader
        s.antialias, s.color_sampling, s.denoise, s.denoise_levels = int(antialias), int(color_sampling), int(denoise), denoise_levels
        s.sigma_color, s.sigma_normal, s.sigma_depth = sigma_color, sigma_normal, sigma_depth
        s.denoise_intensity, s.firefly_clamp = denoise_intensity, firefly_clamp
        s.adaptive, s.adaptive_base, s.adaptive_mode, s.adaptive_threshold = int(adaptive), adaptive_base, adaptive_mode, adaptive_threshold
        for i in range(3):
            s.world_color[i] = world_color[i]
        for i in range(4):
            s.back_color[i] = back_color[i]
        s.seed, s.max_depth, s.rr_depth = seed, max_depth, rr_depth
        s.light_pick_fix = int(light_pick_fix)
        s.threads = threads if threads else (os.cpu_count() or 1)
        s.mix_tree = int(mix_tree)
        n = width * height
        out = {
            "sum": np.zeros((height, width, 3), np.float64),
            "sumsq": np.zeros((height, width, 3), np.float64),
            "n": np.zeros((height, width), np.int32),
            "hdr": np.zeros((height, width, 4), np.float32),
            "ldr": np.zeros((height, width, 4), np.float32),
            "normal": np.zeros((height, width, 3), np.float32),
            "albedo": np.zeros((height, width, 3), np.float32),
            "depth": np.zeros((height, width), np.float32),
        }
        dp = C.POINTER(C.c_double)
        rc = self.lib.orc_render(self.h, C.byref(s), out["sum"].ctypes.data_as(dp), out["sumsq"].ctypes.data_as(dp),
                                 out["n"].ctypes.data_as(C.POINTER(C.c_int32)), _fp(out["hdr"]), _fp(out["ldr"]),
                                 _fp(out["normal"]), _fp(out["albedo"]), _fp(out["depth"]))
        if rc != 0:
            raise RuntimeError(f"oracle render failed: {rc}")
        del n
        return out


def denoise(color, normal, depth, albedo, albedo_alpha, levels=5, sigma_color=0.4, sigma_normal=128.0,
            sigma_depth=0.1, intensity=1.0):
    lib = load()
    color = np.ascontiguousarray(color, np.float32)
    h, w = color.shape[:2]
    a = [np.ascontiguousarray(x, np.float32) for x in (normal, depth, albedo, albedo_alpha)]
    out = np.empty((h, w, 3), np.float32)
    lib.orc_denoise(w, h, _fp(color), _fp(a[0]), _fp(a[1]), _fp(a[2]), _fp(a[3]), levels, sigma_color,
                    sigma_normal, sigma_depth, intensity, _fp(out))
    return out


def tonemap(hdr):
    lib = load()
    hdr = np.ascontiguousarray(hdr, np.float32)
    h, w = hdr.shape[:2]
    out = np.empty_like(hdr)
    lib.orc_tonemap(w, h, _fp(hdr), _fp(out))
    return out


def bloom(hdr, threshold=1.0, strength=1.0, radius=0.03, size_aspect=0.15, curve=1.0):
    """HDR bloom (RayRenderer::applyPostProcess) of an H x W x 4 image; returns a new array."""
    lib = load()
    out = np.ascontiguousarray(hdr, np.float32).copy()
    h, w = out.shape[:2]
    lib.orc_bloom(w, h, _fp(out), threshold, strength, radius, size_aspect, curve)
    return out


def lds(x, y, width, sample, seed, dim):
    return load().orc_lds(x, y, width, sample, seed, dim)


def prng(x, y, width, sample, seed, vertex, slot):
    return load().orc_prng(x, y, width, sample, seed, vertex, slot)
