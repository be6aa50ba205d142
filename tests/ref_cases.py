"""Seeded inputs of the reference golden vectors (tests/golden/ref_*.npz).

tests/golden/make_ref_golden.py feeds these to the reference's own code
(oracle/_ref) and stores inputs and outputs; the tests read the stored inputs
back and feed them to the oracle and to the device.  Nothing here calls a
library.
"""
from __future__ import annotations

import numpy as np

# name -> (builtin scene kind, seed, integer parameters, rays)
RAY_SCENES = {
    "cube_room": (1, 1, None, 8192),           # 36 triangles
    "spheres_98k": (2, 1, [25000], 8192),       # 4 x 24,500-triangle spheres: 98,044 triangles
    "heavy_4m": (2, 1, [1003520], 8192),        # the benchmark scene: 4,014,124 triangles
}

BSDF_PROBES = ("vndf", "smith", "schlick", "refract", "frame")
BSDF_OUT_WIDTH = (3, 1, 1, 3, 6)
MEDIUM_PROBES = ("transmittance", "freeflight", "phase_sample", "phase_pdf", "fields", "bend")
MEDIUM_OUT_WIDTH = (3, 1, 3, 1, 5, 6)


def _unit(rng, n):
    d = rng.normal(size=(n, 3))
    return (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)


def ray_batch(key: str, pos: np.ndarray, n: int):
    """View-space rays over the scene's bounds: half camera rays from the
    origin into the -z half space, half from random interior points in random
    directions; any-hit limits uniform over [0.02, 0.6] of the bounds' diagonal."""
    rng = np.random.default_rng(sum(map(ord, key)))
    p = pos.reshape(-1, 3)
    lo, hi = p.min(0), p.max(0)
    lo, hi = lo + 0.02 * (hi - lo), hi - 0.02 * (hi - lo)
    nc = n // 2
    o = np.zeros((n, 3), np.float32)
    o[nc:] = lo + (hi - lo) * rng.random((n - nc, 3))
    d = _unit(rng, n)
    d[:nc, 2] = -np.abs(d[:nc, 2]) - 0.5
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.concatenate([o, d], 1).astype(np.float32)
    diag = float(np.linalg.norm(hi - lo))
    tmax = (rng.uniform(0.02, 0.6, n) * diag).astype(np.float32)
    return rays, tmax


def lds_inputs(n=2048):
    rng = np.random.default_rng(101)
    return np.stack([rng.integers(0, 2048, n), rng.integers(0, 2048, n), rng.integers(0, 4096, n),
                     rng.integers(0, 16, n)], 1).astype(np.float32)


def cosine_inputs(n=1024):
    rng = np.random.default_rng(102)
    x = np.zeros((n, 7), np.float32)
    x[:, 0] = rng.integers(0, 2048, n)
    x[:, 1] = rng.integers(0, 2048, n)
    x[:, 2] = rng.integers(0, 1024, n)
    x[:, 3] = rng.integers(0, 15, n)  # dims dim, dim + 1 both below 16
    nrm = _unit(rng, n)
    nrm[: n // 8] = np.array([0, 1, 0], np.float32)  # axis-aligned normals take the other tangent branch
    nrm[n // 8: n // 4] = np.array([0, 0, -1], np.float32)
    x[:, 4:7] = nrm
    return x


def triangle_point_inputs(n=512):
    rng = np.random.default_rng(103)
    x = np.zeros((n, 13), np.float32)
    x[:, 0] = rng.integers(0, 2048, n)
    x[:, 1] = rng.integers(0, 2048, n)
    x[:, 2] = rng.integers(0, 1024, n)
    x[:, 3] = rng.integers(0, 15, n)
    x[:, 4:13] = rng.uniform(-5, 5, (n, 9))
    return x


def bsdf_inputs(which: int, n=2048):
    rng = np.random.default_rng(200 + which)
    if which == 0:  # sampleGGXVNDF: local view direction in the upper hemisphere
        v = _unit(rng, n)
        v[:, 2] = np.abs(v[:, 2]) + 1e-3
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        v[: n // 16] = np.array([0, 0, 1], np.float32)  # normal incidence: the degenerate frame branch
        a = np.exp(rng.uniform(np.log(1e-3), 0.0, (n, 2)))
        u = rng.random((n, 2))
        return np.concatenate([v, a, u], 1).astype(np.float32)
    if which == 1:  # smithG1, including w.z <= 0
        w = _unit(rng, n)
        w[:, 2] = np.where(rng.random(n) < 0.9, np.abs(w[:, 2]), -np.abs(w[:, 2]))
        a = np.exp(rng.uniform(np.log(1e-3), 0.0, (n, 2)))
        return np.concatenate([w, a], 1).astype(np.float32)
    if which == 2:  # fresnelSchlick
        return np.stack([rng.random(n), rng.uniform(1.0, 2.6, n)], 1).astype(np.float32)
    if which == 3:  # refract, both sides and total internal reflection
        d = _unit(rng, n)
        nn = _unit(rng, n)
        ior = rng.uniform(1.05, 2.4, (n, 1))
        return np.concatenate([d, nn, ior], 1).astype(np.float32)
    if which == 4:  # buildTangentFrame, including near +-y
        nn = _unit(rng, n)
        nn[: n // 8] = np.array([0, 1, 0], np.float32)
        nn[n // 8: n // 4] = np.array([0.01, -0.9999, 0.0], np.float32)
        return (nn / np.linalg.norm(nn, axis=1, keepdims=True)).astype(np.float32)
    raise ValueError(which)


# Reference defaults of HomogeneousMedium (medium.h), overridden per case; the
# keys are the C ABI's rg_medium field names.
MEDIUM_DEFAULTS = dict(
    sigma_a=(0, 0, 0), sigma_s=(0, 0, 0), g=0.0, density=1.0, density_field=0, noise_frequency=1.0,
    noise_octaves=4, noise_gain=0.5, noise_lacunarity=2.0, noise_amplitude=1.0, noise_bias=0.0,
    noise_offset=(0, 0, 0), emission_mode=0, sigma_e=(0, 0, 0), cone_origin=(0, 0, 0), cone_axis=(0, 0, -1),
    cone_length=1.0, cone_radius=0.3, cone_inner=(0.6, 0.7, 1.0), cone_outer=(1.0, 0.4, 0.05), cone_intensity=50.0,
    cone_peak_axial=0.15, cone_peak_sharpness=5.0, heat_haze=0, ior_amplitude=0.005, ior_frequency=4.0,
    ior_octaves=3, ior_gain=0.5, ior_lacunarity=2.0, ior_march_steps=16, ior_offset=(0, 0, 0), ior_falloff=0.0)

MEDIA = {
    # the media + adaptive workload's fog: sigma_t 0.05, albedo 0.8, g 0.3
    "fog_c3": dict(sigma_a=(0.01, 0.01, 0.01), sigma_s=(0.04, 0.04, 0.04), g=0.3),
    "coloured_back": dict(sigma_a=(0.02, 0.05, 0.1), sigma_s=(0.3, 0.2, 0.1), g=-0.6, density=1.5),
    "fbm": dict(sigma_a=(0.05, 0.05, 0.05), sigma_s=(0.4, 0.35, 0.3), g=0.5, density_field=1, noise_frequency=1.6,
                noise_octaves=4, noise_gain=0.5, noise_lacunarity=2.0, noise_amplitude=1.4, noise_bias=-0.25,
                noise_offset=(0.3, -0.2, 0.1)),
    "cone": dict(sigma_a=(0.01, 0.01, 0.01), sigma_s=(0.01, 0.01, 0.01), emission_mode=1, cone_origin=(0.0, -1.0, -5.0),
                 cone_axis=(0.0, 1.0, 0.2), cone_length=3.0, cone_radius=0.6, cone_intensity=20.0,
                 cone_peak_axial=0.2, cone_peak_sharpness=4.0),
    "haze": dict(sigma_a=(0.001, 0.001, 0.001), heat_haze=1, ior_amplitude=0.01, ior_frequency=3.0, ior_octaves=3,
                 ior_march_steps=16, ior_offset=(0.2, 0.1, -0.3), ior_falloff=0.5),
}


def medium_params(name: str) -> dict:
    p = dict(MEDIUM_DEFAULTS)
    p.update(MEDIA[name])
    return p


def medium_vector(params: dict) -> np.ndarray:
    """The reference harness's 50-float medium layout (oracle/ref_harness.cpp
    ref_medium_create)."""
    p = dict(MEDIUM_DEFAULTS)
    p.update(params)
    v = []
    for k in ("sigma_a", "sigma_s"):
        v += list(p[k])
    v += [p["g"], p["density"], p["density_field"], p["noise_frequency"], p["noise_octaves"], p["noise_gain"],
          p["noise_lacunarity"], p["noise_amplitude"], p["noise_bias"]]
    v += list(p["noise_offset"])
    v += [p["emission_mode"]] + list(p["sigma_e"]) + list(p["cone_origin"]) + list(p["cone_axis"])
    v += [p["cone_length"], p["cone_radius"]] + list(p["cone_inner"]) + list(p["cone_outer"])
    v += [p["cone_intensity"], p["cone_peak_axial"], p["cone_peak_sharpness"], p["heat_haze"], p["ior_amplitude"],
          p["ior_frequency"], p["ior_octaves"], p["ior_gain"], p["ior_lacunarity"], p["ior_march_steps"]]
    v += list(p["ior_offset"]) + [p["ior_falloff"]]
    assert len(v) == 50
    return np.array(v, np.float32)


def medium_inputs(which: int, name: str):
    rng = np.random.default_rng(300 + 10 * which + sum(map(ord, name)))
    if which == 0:
        return np.concatenate([[0.0, -1.0, 1e-4], rng.uniform(0, 60, 61)]).astype(np.float32)
    if which == 1:
        return np.concatenate([[0.0, 0.9999999, 1.0, 0.5], rng.random(124)]).astype(np.float32)
    if which == 2:
        wo = _unit(rng, 256)
        wo[:16] = np.array([1, 0, 0], np.float32)
        return np.concatenate([wo, rng.random((256, 2))], 1).astype(np.float32)
    if which == 3:
        return np.concatenate([_unit(rng, 256), _unit(rng, 256)], 1).astype(np.float32)
    if which == 4:
        p = rng.uniform((-3, -3, -9), (3, 3, -1), (512, 3))
        return p.astype(np.float32)
    if which == 5:
        if name != "haze":
            return None
        o = rng.uniform((-2, -2, -6), (2, 2, -2), (128, 3))
        d = _unit(rng, 128)
        length = rng.uniform(0.5, 6.0, (128, 1))
        return np.concatenate([o, d, length], 1).astype(np.float32)
    raise ValueError(which)
