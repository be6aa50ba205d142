"""The CPU oracle against golden vectors written by the REFERENCE's own code.

tests/golden/ref_*.npz come from the reference renderer's hot-path sources
(bvh.cpp, raycommon.cpp, medium.cpp, bsdf.cpp) compiled unchanged into
oracle/_ref and run by tests/golden/make_ref_golden.py.  These tests pin the
oracle (and, in test_gpu_golden_ref.py, the device) to them.

Tolerances:
* ray batches: hit triangle ids identical except exact ties (coplanar
  triangles at the same distance: t agrees within 1e-5 relative; any number)
  and edge grazes (the nearer of the two hits lies within 1e-5 of its
  triangle's edge in barycentrics, where rounding decides inside or outside;
  at most 0.1% of rays); t within 1e-5 relative + 2e-6 absolute
  (view-space coordinates reach 20, where floats are 2e-6 apart, so a hit a
  hundredth of a unit from the ray origin carries that absolute error); barycentrics as a
  hit point: |sum(dw_i v_i)| <= 1e-5 x the distance from the ray origin to the
  triangle (u and v alone are ill-conditioned for small, far triangles); any-hit
  flags identical except on 0.1% of rays;
* Halton values, GGX / dielectric helpers and the point on a triangle: bit
  for bit (the oracle evaluates them in the reference's order, without fused
  multiply-adds);
* cosine-weighted directions: 1e-6 absolute (the reference evaluates its
  trigonometry in double precision);
* media: transmittance, free flight, phase sampling and pdf, density /
  emission / index fields and heat-haze bending within 1e-5 relative + 1e-6
  absolute.
"""
import hashlib
import os

import numpy as np
import pytest

import ref_cases
import scenes

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")


def load(name):
    return np.load(os.path.join(GOLD, name))


def tie(tuv, prim, rtuv, rprim):
    """Two different closest hits at the same distance (coplanar triangles)."""
    return prim >= 0 and rprim >= 0 and abs(tuv[0] - rtuv[0]) <= 1e-5 * abs(rtuv[0]) + 2e-6


def edge_graze(tuv, prim, rtuv, rprim, eps=1e-5):
    """The nearer of two different closest hits sits on an edge of its triangle
    (a graze that the other side's rounding rejected)."""
    near = tuv if (rprim < 0 or (prim >= 0 and tuv[0] < rtuv[0])) else rtuv
    u, v = float(near[1]), float(near[2])
    return min(u, v, 1.0 - u - v) <= eps


def check_rays(key, R, tuv, prim, anyhit=None):
    """Compare one ray batch with the reference's results: every different hit id
    is an exact tie (any number: the cube room's boxes stand on its floor) or an
    edge graze (at most 0.1% of the rays)."""
    rays, rprim, rtuv = R[f"{key}_rays"], R[f"{key}_prim"], R[f"{key}_tuv"]
    same = prim == rprim
    grazes = 0
    for i in np.nonzero(~same)[0]:
        if tie(tuv[i], prim[i], rtuv[i], rprim[i]):
            continue
        assert edge_graze(tuv[i], prim[i], rtuv[i], rprim[i]), \
            f"{key} ray {i}: id {prim[i]} t {tuv[i, 0]} against the reference's {rprim[i]} t {rtuv[i, 0]}"
        grazes += 1
    assert grazes <= 0.001 * len(prim), f"{key}: {grazes} edge grazes"
    hit = same & (rprim >= 0)
    np.testing.assert_allclose(tuv[hit, 0], rtuv[hit, 0], rtol=1e-5, atol=2e-6)
    if anyhit is not None:
        assert (anyhit == R[f"{key}_any"].astype(bool)).mean() >= 0.999
    return hit


def check_barycentrics(pos, rays, hit, prim, tuv, rtuv):
    tri = pos[prim[hit]].reshape(-1, 3, 3)
    e1, e2 = tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0]
    du = (tuv[hit, 1] - rtuv[hit, 1])[:, None]
    dv = (tuv[hit, 2] - rtuv[hit, 2])[:, None]
    dp = np.linalg.norm(e1 * du + e2 * dv, axis=1)
    dist = np.linalg.norm(rays[hit, :3] - tri[:, 0], axis=1) + np.linalg.norm(e1, axis=1)
    assert np.all(dp <= 1e-5 * dist), float((dp / dist).max())


@pytest.mark.parametrize("key", list(ref_cases.RAY_SCENES))
def test_oracle_ray_batches_match_reference(orc, key):
    R = load("ref_rays.npz")
    kind, seed, params, _ = ref_cases.RAY_SCENES[key]
    sc = orc.CpuScene(kind, seed, params)
    o = orc.OracleScene(sc.ptr)
    pos, nrm = o.view_triangles()
    # the same flattened scene the reference traced
    assert len(pos) == int(R[f"{key}_num_triangles"])
    assert hashlib.sha256(pos.tobytes() + nrm.tobytes()).digest() == R[f"{key}_tri_sha256"].tobytes()
    rays = R[f"{key}_rays"]
    tuv, prim = o.closest(rays)
    anyhit = o.any(rays, R[f"{key}_tmax"], 3)  # every triangle occludes, as in the reference harness
    hit = check_rays(key, R, tuv, prim, anyhit)
    check_barycentrics(pos, rays, hit, prim, tuv, R[f"{key}_tuv"])
    o.close()
    sc.close()


def test_oracle_halton_values_match_reference(orc):
    S = load("ref_sampling.npz")
    np.testing.assert_array_equal(orc.lds_probe(S["lds_in"]), S["lds_out"])


def test_oracle_cosine_and_triangle_points_match_reference(orc):
    S = load("ref_sampling.npz")
    np.testing.assert_allclose(orc.cosine_probe(S["cosine_in"]), S["cosine_out"], rtol=0, atol=1e-6)
    np.testing.assert_array_equal(orc.triangle_point_probe(S["tripoint_in"]), S["tripoint_out"])


@pytest.mark.parametrize("which,name", list(enumerate(ref_cases.BSDF_PROBES)))
def test_oracle_bsdf_helpers_match_reference(orc, which, name):
    S = load("ref_sampling.npz")
    np.testing.assert_array_equal(orc.bsdf_probe(which, S[f"{name}_in"]), S[f"{name}_out"])


def medium_scene(rg, name):
    """One far triangle behind the camera and the named medium as the global medium."""
    med = rg.medium(**ref_cases.medium_params(name))
    fp, fn = scenes.quad_z(60.0, 0.5, +1)
    return scenes.build(rg, [(fp, fn, scenes.material(rg), -1)], scenes.camera(rg), media=[med], global_medium=0)


@pytest.mark.parametrize("name", list(ref_cases.MEDIA))
def test_oracle_media_match_reference(rg, orc, name):
    M = load("ref_media.npz")
    np.testing.assert_array_equal(ref_cases.medium_vector(ref_cases.medium_params(name)), M[f"{name}_params"])
    sc = medium_scene(rg, name)
    o = orc.OracleScene(sc.ptr)
    for which, probe in enumerate(ref_cases.MEDIUM_PROBES):
        key = f"{name}_{probe}_in"
        if key not in M:
            continue
        got = o.medium_probe(0, which, M[key])
        np.testing.assert_allclose(got, M[f"{name}_{probe}_out"], rtol=1e-5, atol=1e-6, err_msg=f"{name} {probe}")
    o.close()
    sc.close()


def test_goldens_cover_the_reference_inputs():
    """The stored inputs are the seeded ones of ref_cases (nothing hand-edited)."""
    S = load("ref_sampling.npz")
    np.testing.assert_array_equal(S["lds_in"], ref_cases.lds_inputs())
    np.testing.assert_array_equal(S["cosine_in"], ref_cases.cosine_inputs())
    for which, name in enumerate(ref_cases.BSDF_PROBES):
        np.testing.assert_array_equal(S[f"{name}_in"], ref_cases.bsdf_inputs(which))
    M = load("ref_media.npz")
    for name in ref_cases.MEDIA:
        np.testing.assert_array_equal(M[f"{name}_fields_in"], ref_cases.medium_inputs(4, name))
