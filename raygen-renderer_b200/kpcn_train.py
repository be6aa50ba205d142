"""Training data and training loop of the learned denoiser.

Pairs are rendered by the tracer itself: a low-spp render (the network's input:
noisy radiance plus the albedo / normal / depth guides) and a high-spp render of
the same job (the target).  Scenes are the seeded procedural batch jobs
(heterogeneous triangle counts, emitters and materials) and the cube room.

    python -m raygen_b200.kpcn_train --out weights.bin   (from the package's parent)

or through `train(...)` from Python.
"""
import argparse
import time

import numpy as np


def render_set(rg, scene, width, height, spp_list, spp_hi, seed, max_depth=6):
    """-> [(noisy RGBA, normal, albedo, depth, reference RGBA, spp) for spp in spp_list]:
    one job rendered at each input spp, all against one spp_hi reference."""
    st = rg.RendererSettings(resolutionWidth=width, resolutionHeight=height, samples=spp_hi, maxDepth=max_depth,
                             seed=seed + 7919)
    r = rg.RayRenderer(st)
    r.set_scene(scene)
    r.render()
    ref = r.get_hdr_result()
    r.settings.enableDenoise = True
    r.settings.denoiseIntensity = 0.0  # the denoiser pass leaves the radiance as rendered
    out = []
    for i, spp in enumerate(spp_list):
        r.settings.samples = int(spp)
        r.settings.seed = seed + 104729 * i
        r.render()
        noisy = r.get_hdr_result()
        normal, albedo, depth = r.get_aovs()
        out.append((noisy, normal, albedo, depth, ref, float(spp)))
    r.close()
    return out


def render_pair(rg, scene, width, height, spp_lo, spp_hi, seed, max_depth=6):
    """-> (noisy RGBA, normal, albedo, depth, reference RGBA, spp_lo) for one job."""
    return render_set(rg, scene, width, height, [spp_lo], spp_hi, seed, max_depth)[0]


def input_spp(k, spp_lo, spp_lo_max, per_scene=1):
    """The input spp of training scene k: `per_scene` distinct powers of two in
    [spp_lo, spp_lo_max], drawn uniformly over the exponents from a generator seeded by k."""
    levels = [spp_lo << i for i in range(64) if spp_lo << i <= max(spp_lo, spp_lo_max)]
    rng = np.random.default_rng(7000 + k)
    return sorted(int(x) for x in rng.choice(levels, size=min(per_scene, len(levels)), replace=False))


def scene_for(rg, k, generator="narrow"):
    """Seeded procedural job k.
    narrow: batch-job scenes of 2k-40k triangles with 1-8 emitters; every 8th the cube room.
    config4: the heterogeneous job mix's scenes -- triangles log-uniform 1e3-3e5 (2e6 in the
      mix; capped for rendering time), emitters 1-64; every 8th the cube room and every 8th the
      heavy-sphere scene (metal / dielectric spheres, 4 x 25k triangles)."""
    if k % 8 == 7:
        return rg.Scene.builtin(1, 1 + k)
    rng = np.random.default_rng(1000 + k)
    if generator == "config4":
        if k % 8 == 3:
            return rg.Scene.builtin(2, 7000 + k, [25000])
        tris = int(np.exp(rng.uniform(np.log(1e3), np.log(3e5))))
        return rg.Scene.builtin(4, 5000 + k, [tris, int(rng.integers(1, 65))])
    tris = int(np.exp(rng.uniform(np.log(2e3), np.log(4e4))))
    return rg.Scene.builtin(4, 5000 + k, [tris, int(rng.integers(1, 9))])


def make_examples(rg, count, size=64, spp_lo=8, spp_hi=512, first=0, generator="narrow", max_depth=6):
    out = []
    for k in range(first, first + count):
        sc = scene_for(rg, k, generator)
        out.append(render_pair(rg, sc, size, size, spp_lo, spp_hi, seed=100 + k, max_depth=max_depth))
        sc.close()
    return out


def relmse(img, ref, eps=0.01):
    a, r = np.asarray(img)[..., :3].astype(np.float64), np.asarray(ref)[..., :3].astype(np.float64)
    return float(np.mean((a - r) ** 2 / (r * r + eps)))


def train(rg, examples, steps=2000, batch=8, lr=1e-3, seed=0, params=None, log=None, denoiser=None):
    """Adam on the examples (a list of render_pair tuples), or on the examples
    already added to `denoiser` when one is given."""
    d = denoiser if denoiser is not None else rg.Denoiser(seed=seed, params=params)
    for ex in examples:
        d.add_example(*ex)
    losses = []
    t0 = time.time()
    done = 0
    while done < steps:
        n = min(250, steps - done)
        # step decay of the learning rate over the run
        cur = lr * (0.3 if done >= 0.75 * steps else 1.0)
        losses.append(d.train(n, batch, cur))
        done += n
        if log:
            log(f"step {done}: loss {losses[-1][-n:].mean():.5f} ({time.time() - t0:.1f} s)")
    return d, np.concatenate(losses) if losses else np.zeros(0)


def evaluate(rg, denoiser, count=16, size=128, spp_lo=8, spp_hi=2048, first=100000, generator="narrow"):
    """relMSE against a high-spp render on held-out jobs: the noisy input, A-Trous
    (the reference's denoiser, default settings) and the learned denoiser."""
    rows = []
    for k in range(first, first + count):
        sc = scene_for(rg, k, generator)
        noisy, normal, albedo, depth, ref, spp = render_pair(rg, sc, size, size, spp_lo, spp_hi, seed=100 + k)
        sc.close()
        atrous = rg.denoise_atrous(noisy[..., :3], normal, depth, albedo, np.ones_like(depth))
        learned = denoiser.apply(noisy, normal, albedo, depth, spp=spp)
        rows.append((relmse(noisy, ref), relmse(atrous, ref), relmse(learned, ref)))
    r = np.array(rows)
    return {"noisy": float(r[:, 0].mean()), "atrous": float(r[:, 1].mean()), "learned": float(r[:, 2].mean()),
            "learned_wins": int((r[:, 2] < r[:, 1]).sum()), "jobs": count, "size": size, "spp": spp_lo,
            "reference_spp": spp_hi}


def main():
    import os
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.dirname(here))
    from __graft_entry__ import load_package
    rg = load_package()
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(here, "kpcn_weights.bin"))
    ap.add_argument("--examples", type=int, default=256)
    ap.add_argument("--size", type=int, default=64)
    ap.add_argument("--spp-lo", type=int, default=8, help="input spp (the lowest, with --spp-lo-max)")
    ap.add_argument("--spp-lo-max", type=int, default=0, help="input spp up to this power-of-two multiple of --spp-lo")
    ap.add_argument("--per-scene", type=int, default=1, help="input spp levels rendered per scene (one reference)")
    ap.add_argument("--spp-hi", type=int, default=512)
    ap.add_argument("--eval-spp", default="8", help="comma-separated input spp of the held-out evaluation")
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--eval", type=int, default=16, help="held-out jobs to evaluate (0: none)")
    ap.add_argument("--generator", default="narrow", choices=["narrow", "config4"],
                    help="training scenes: the narrow batch-job range, or the heterogeneous job mix's")
    ap.add_argument("--init", default=None, help="start from these weights (fine-tuning)")
    a = ap.parse_args()
    t0 = time.time()
    params = np.fromfile(a.init, np.float32) if a.init else None
    d = rg.Denoiser(seed=0, params=params)
    hist = {}
    for k in range(a.examples):  # rendered pairs go to the device one scene at a time
        sc = scene_for(rg, k, a.generator)
        spps = input_spp(k, a.spp_lo, a.spp_lo_max, a.per_scene)
        for ex in render_set(rg, sc, a.size, a.size, spps, a.spp_hi, seed=100 + k):
            d.add_example(*ex)
        for spp in spps:
            hist[spp] = hist.get(spp, 0) + 1
        sc.close()
        if (k + 1) % 128 == 0:
            print(f"{k + 1} scenes ({time.time() - t0:.1f} s)", flush=True)
    print(f"{a.examples} scenes of {a.size}x{a.size}, input spp {dict(sorted(hist.items()))}, reference {a.spp_hi} spp, "
          f"in {time.time() - t0:.1f} s", flush=True)
    d, losses = train(rg, [], a.steps, a.batch, a.lr, log=lambda m: print(m, flush=True), denoiser=d)
    d.save(a.out)
    print(f"saved {a.out}; final loss {losses[-100:].mean():.5f}", flush=True)
    if a.eval > 0:
        for spp in (int(x) for x in a.eval_spp.split(",")):
            for gen in ("narrow", "config4"):
                print(f"held-out relMSE ({gen} scenes, {spp} spp):", evaluate(rg, d, a.eval, spp_lo=spp, generator=gen),
                      flush=True)


if __name__ == "__main__":
    main()
