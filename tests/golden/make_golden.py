"""Generates tests/golden/oracle_golden.npz from the CPU oracle.

The reference ships no golden vectors (no tests at all), so these fixtures pin
the oracle against itself: LDS / counter-RNG values, cube-room ray-batch hits
and a small cube-room render.  Regenerate only on a deliberate oracle change:

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))


def golden_inputs():
    rng = np.random.default_rng(1234)
    keys = np.stack([rng.integers(0, 256, 64), rng.integers(0, 256, 64), rng.integers(0, 4096, 64),
                     rng.integers(0, 20, 64)], axis=1)
    import scenes
    rays = scenes.random_rays(((-5, -5, -23), (5, 5, -14)), 2048, 77)
    return keys, rays


def compute(rg, oracle):
    keys, rays = golden_inputs()
    lds = np.array([oracle.lds(int(x), int(y), 256, int(s), 1, int(d)) for x, y, s, d in keys], np.float32)
    prng = np.array([oracle.prng(int(x), int(y), 256, int(s), 1, int(d) % 8, int(d) % 19) for x, y, s, d in keys],
                    np.float32)
    sc = rg.Scene.builtin(1, 1)
    o = oracle.OracleScene(sc.ptr)
    tuv, prim = o.closest(rays)
    img = o.render(16, 16, 16, max_depth=5, seed=1, threads=1)
    return dict(keys=keys, rays=rays, lds=lds, prng=prng, tuv=tuv, prim=prim, img_sum=img["sum"])


if __name__ == "__main__":
    from __graft_entry__ import load_package
    import oracle
    out = compute(load_package(), oracle)
    np.savez_compressed(os.path.join(HERE, "oracle_golden.npz"), **out)
    print({k: v.shape for k, v in out.items()})
