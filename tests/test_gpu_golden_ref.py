"""The B200 kernels against golden vectors written by the REFERENCE's own code
(tests/golden/ref_*.npz; see tests/golden/make_ref_golden.py), through the C ABI.

Tolerances (the device contracts multiply-adds and uses its own sincosf /
acosf / expf / logf, so bit equality with the reference is not expected except
for the integer-hash Halton values):
* ray batches, including the 4,014,124-triangle benchmark scene: hit ids
  identical except exact ties and edge grazes (<= 0.1% of rays), t within 1e-5
  relative + 2e-6 absolute, barycentrics as a hit point within 1e-5 of the
  distance, any-hit flags identical on >= 99.9% of rays, no device error;
* Halton values bit for bit;
* G1, Fresnel, pdfs and points: 2e-5 relative + 2e-6 absolute; unit
  direction vectors 1e-5 absolute;
* media: density / emission / index fields and bending 2e-5 relative + 2e-6
  absolute; free-flight distances 2e-5 relative.
"""
import numpy as np
import pytest

import ref_cases
from test_golden_ref import check_barycentrics, check_rays, load, medium_scene

pytestmark = pytest.mark.gpu

TOL = dict(rtol=2e-5, atol=2e-6)
# unit vectors (sampled directions, frames): the device's sincosf / sqrt / FMA
# contraction differ from the reference's libm by a few ulp of the angle
DIR_TOL = dict(rtol=2e-5, atol=1e-5)


@pytest.mark.parametrize("width", [8, 2])
@pytest.mark.parametrize("key", list(ref_cases.RAY_SCENES))
def test_device_ray_batches_match_reference(rg, orc, key, width):
    if key == "heavy_4m" and width == 2:
        pytest.skip("the benchmark scene runs the 8-wide BVH")
    R = load("ref_rays.npz")
    kind, seed, params, _ = ref_cases.RAY_SCENES[key]
    sc = rg.Scene.builtin(kind, seed, params)
    r = rg.RayRenderer(rg.RendererSettings(resolutionWidth=8, resolutionHeight=8, samples=1, bvhWidth=width))
    r.set_scene(sc)
    rays = R[f"{key}_rays"]
    tuv, prim = r.trace_closest(rays)
    anyhit = r.trace_any(rays, R[f"{key}_tmax"], rg.PRED_ALL)
    hit = check_rays(key, R, tuv, prim, anyhit)
    o = orc.OracleScene(orc.CpuScene(kind, seed, params).ptr) if key != "heavy_4m" else None
    if o is not None:  # barycentrics need the flattened triangles (the oracle's, pinned by SHA-256)
        pos, _ = o.view_triangles()
        check_barycentrics(pos, rays, hit, prim, tuv, R[f"{key}_tuv"])
        o.close()
    assert r.stats()["device_error"] == 0
    r.close()
    sc.close()


def test_device_halton_values_match_reference(rg):
    S = load("ref_sampling.npz")
    got = rg.probe_sampling(rg.PROBE_LDS, S["lds_in"])[:, 0]
    np.testing.assert_array_equal(got, S["lds_out"])


def test_device_cosine_and_triangle_points_match_reference(rg):
    S = load("ref_sampling.npz")
    np.testing.assert_allclose(rg.probe_sampling(rg.PROBE_COSINE, S["cosine_in"]), S["cosine_out"], **TOL)
    np.testing.assert_allclose(rg.probe_sampling(rg.PROBE_TRIANGLE_POINT, S["tripoint_in"]), S["tripoint_out"],
                               rtol=2e-5, atol=2e-5)


@pytest.mark.parametrize("which,name", list(enumerate(ref_cases.BSDF_PROBES)))
def test_device_bsdf_helpers_match_reference(rg, which, name):
    S = load("ref_sampling.npz")
    got = rg.probe_sampling(which, S[f"{name}_in"])
    tol = DIR_TOL if name in ("vndf", "refract", "frame") else TOL
    np.testing.assert_allclose(got, S[f"{name}_out"], **tol, err_msg=name)


@pytest.mark.parametrize("name", list(ref_cases.MEDIA))
def test_device_media_match_reference(rg, name):
    M = load("ref_media.npz")
    p = ref_cases.medium_params(name)
    g = p["g"]
    # sigma_t hero channel as prepare() forms it (medium.cpp:19-28), in float32
    d = np.float32(max(0.0, p["density"]))
    st = np.array(p["sigma_a"], np.float32) * d + np.array(p["sigma_s"], np.float32) * d
    hero = np.float32((st[0] + st[1] + st[2]) * np.float32(1.0 / 3.0))
    # Henyey-Greenstein sampling and pdf, free flight (the kernel's own helpers)
    x = M[f"{name}_phase_sample_in"]
    rows = np.concatenate([x[:, :3], np.full((len(x), 1), g, np.float32), x[:, 3:5]], 1)
    np.testing.assert_allclose(rg.probe_sampling(rg.PROBE_PHASE_SAMPLE, rows), M[f"{name}_phase_sample_out"], **TOL)
    x = M[f"{name}_phase_pdf_in"]
    rows = np.concatenate([x, np.full((len(x), 1), g, np.float32)], 1)
    np.testing.assert_allclose(rg.probe_sampling(rg.PROBE_PHASE_PDF, rows)[:, 0], M[f"{name}_phase_pdf_out"][:, 0],
                               **TOL)
    x = M[f"{name}_freeflight_in"]
    rows = np.stack([np.full(len(x), hero, np.float32), x], 1)
    np.testing.assert_allclose(rg.probe_sampling(rg.PROBE_FREE_FLIGHT, rows)[:, 0], M[f"{name}_freeflight_out"][:, 0],
                               rtol=2e-5)
    # the medium's fields and heat-haze bending, on the device copy of the scene's medium
    sc = medium_scene(rg, name)
    r = rg.RayRenderer(rg.RendererSettings(resolutionWidth=8, resolutionHeight=8, samples=1))
    r.set_scene(sc)
    np.testing.assert_allclose(r.medium_eval(0, M[f"{name}_fields_in"]), M[f"{name}_fields_out"], **TOL)
    if f"{name}_bend_in" in M:
        np.testing.assert_allclose(r.medium_bend(0, M[f"{name}_bend_in"]), M[f"{name}_bend_out"], rtol=2e-5, atol=2e-5)
    r.close()
    sc.close()
