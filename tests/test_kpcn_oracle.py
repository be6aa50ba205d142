"""The learned denoiser's CPU oracle (oracle/kpcn_oracle.py) pinned by finite
differences: its analytic backward pass agrees with central differences of its
own float64 forward pass (no GPU)."""
import numpy as np

import kpcn_oracle as ko


def tiny_batch(seed, N=2, H=7, W=6):
    rng = np.random.default_rng(seed)
    noisy = rng.gamma(1.5, 0.5, (N, H, W, 3))
    ref = noisy * 0.6 + 0.2
    normal = rng.random((N, H, W, 3))
    albedo = rng.random((N, H, W, 3))
    depth = rng.random((N, H, W))
    return noisy, ref, ko.features(noisy, normal, albedo, depth, exact=True)


def test_param_count_and_layout():
    assert ko.num_params() == 32 * 9 * 16 + 32 + 5 * (32 * 9 * 32 + 32)
    p = ko.init_params(0)
    layers = ko.unpack(p.astype(np.float64))
    assert np.all(layers[0][0][:, :, 11:] == 0) and np.all(layers[5][0][ko.KP:] == 0)


def test_backward_matches_finite_differences():
    noisy, ref, X0 = tiny_batch(1)
    p = ko.init_params(3).astype(np.float64)
    rng = np.random.default_rng(4)
    p += rng.standard_normal(p.shape) * 0.02  # nonzero biases, break symmetries
    layers = ko.unpack(p)
    loss, g = ko.backward(p, X0, noisy, ref, exact=True)
    offs = np.cumsum([0] + [w + b for w, b in ko.layer_sizes()])
    h = 1e-6
    for l in range(6):
        wlen = ko.layer_sizes()[l][0]
        idx = list(rng.integers(offs[l], offs[l] + wlen, 4)) + [offs[l] + wlen + 3]  # weights + one bias
        for i in idx:
            if l == 0 and (i - offs[0]) < wlen and (i - offs[0]) % 16 >= 11:
                continue  # padding input channels carry no signal
            if l == 5 and (i - offs[5]) < wlen and (i - offs[5]) // (9 * 32) >= ko.KP:
                continue  # padding logits
            if l == 5 and i >= offs[5] + wlen and i - offs[5] - wlen >= ko.KP:
                continue
            pp, pm = p.copy(), p.copy()
            pp[i] += h
            pm[i] -= h
            num = (ko.loss_of(ko.forward(pp, X0, noisy, exact=True)["out"], ref) -
                   ko.loss_of(ko.forward(pm, X0, noisy, exact=True)["out"], ref)) / (2 * h)
            assert abs(num - g[i]) <= 1e-6 + 1e-4 * abs(num), (l, i, num, g[i])


def test_head_is_a_normalised_filter():
    noisy, ref, X0 = tiny_batch(2)
    f = ko.forward(ko.init_params(5), X0, noisy)
    assert np.allclose(f["w"].sum(axis=-1), 1.0)
    # a constant image is reproduced exactly by any normalised kernel
    const = np.full_like(noisy, 0.7)
    g = ko.forward(ko.init_params(5), X0, const)
    assert np.allclose(g["out"], 0.7)


def test_training_input_spp_levels():
    """kpcn_train.input_spp: distinct powers of two in [lo, lo_max], the same for a scene
    index every time, and a single level when no range is given."""
    import importlib.util
    import os
    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "raygen-renderer_b200",
                        "kpcn_train.py")
    spec = importlib.util.spec_from_file_location("kpcn_train_cpu", path)
    kt = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(kt)
    seen = set()
    for k in range(200):
        lv = kt.input_spp(k, 4, 256, 2)
        assert lv == kt.input_spp(k, 4, 256, 2)
        assert len(lv) == 2 and len(set(lv)) == 2 and lv == sorted(lv)
        for v in lv:
            assert 4 <= v <= 256 and (v & (v - 1)) == 0
            seen.add(v)
        assert kt.input_spp(k, 8, 0, 1) == [8]
    assert seen == {4, 8, 16, 32, 64, 128, 256}
    # the features' noise-level channel: log2(1 + spp) / 12
    f = ko.features(np.zeros((1, 2, 2, 3)), np.zeros((1, 2, 2, 3)), np.zeros((1, 2, 2, 3)), np.zeros((1, 2, 2)),
                    spp=255.0, exact=True)
    assert np.allclose(f[..., 10], 8.0 / 12.0) and np.all(f[..., 11:] == 0)
