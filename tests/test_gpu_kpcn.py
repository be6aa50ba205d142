"""Learned denoiser on the tensor cores (needs a B200): the tcgen05 BF16 GEMM
building block against a float64 product of the same BF16 operands."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("M,N,K", [(128, 32, 64), (300, 16, 144), (256, 128, 256), (128, 48, 96)])
def test_tc_gemm_matches_fp64(rg, M, N, K):
    rng = np.random.default_rng(M + N + K)
    A = rng.standard_normal((M, K)).astype(np.float32)
    B = rng.standard_normal((N, K)).astype(np.float32)
    got = rg.tc_gemm_bf16(A, B)
    a = rg.from_bf16_bits(rg.to_bf16_bits(A)).astype(np.float64)
    b = rg.from_bf16_bits(rg.to_bf16_bits(B)).astype(np.float64)
    ref = a @ b.T
    np.testing.assert_allclose(got, ref, rtol=1e-5, atol=1e-4 * np.sqrt(K))


# ---------------------------------------------------------------- the network
import kpcn_oracle as ko  # noqa: E402


def synth(n, h, w, seed):
    rng = np.random.default_rng(seed)
    noisy = np.concatenate([rng.gamma(1.5, 0.5, (n, h, w, 3)), np.ones((n, h, w, 1))], -1).astype(np.float32)
    ref = noisy.copy()
    ref[..., :3] = noisy[..., :3] * 0.5 + 0.3
    normal = rng.random((n, h, w, 3)).astype(np.float32)
    albedo = rng.random((n, h, w, 3)).astype(np.float32)
    depth = rng.random((n, h, w)).astype(np.float32)
    return noisy, normal, albedo, depth, ref


def perturbed(d, seed, scale=0.05):
    p = d.params.astype(np.float64)
    rng = np.random.default_rng(seed)
    p += rng.standard_normal(p.shape) * scale
    layers = ko.unpack(p)  # keep the padding entries at zero
    for l, (W, b) in enumerate(layers):
        if l == 0:
            W[:, :, 11:] = 0.0
        if l == 5:
            W[ko.KP:] = 0.0
            b[ko.KP:] = 0.0
    return np.concatenate([np.concatenate([W.ravel(), b]) for W, b in layers]).astype(np.float32)


def test_kpcn_forward_matches_oracle(rg):
    d = rg.Denoiser(seed=3)
    p = perturbed(d, 1)
    d.params = p
    noisy, normal, albedo, depth, ref = synth(1, 37, 45, 1)  # 1665 pixels: a partial last tile
    got = d.apply(noisy[0], normal[0], albedo[0], depth[0], spp=37)
    f = ko.forward(p, ko.features(noisy, normal, albedo, depth, spp=37), noisy)
    np.testing.assert_allclose(got[..., :3], f["out"][0], rtol=2e-3, atol=2e-3)
    assert np.all(got[..., 3] == 1.0)
    d.close()


def test_kpcn_forward_matches_oracle_over_many_tiles(rg):
    """300 rows of 4 column tiles (the last 36 pixels wide): strips of
    several rows, so the ring of input rows wraps inside a strip while the
    next row loads during the current row's MMAs and epilogue."""
    d = rg.Denoiser(seed=4)
    p = perturbed(d, 3)
    d.params = p
    noisy, normal, albedo, depth, ref = synth(1, 300, 420, 6)
    got = d.apply(noisy[0], normal[0], albedo[0], depth[0])
    f = ko.forward(p, ko.features(noisy, normal, albedo, depth), noisy)
    np.testing.assert_allclose(got[..., :3], f["out"][0], rtol=2e-3, atol=2e-3)
    d.close()


def test_kpcn_gradients_match_oracle_over_many_tiles(rg):
    d = rg.Denoiser(seed=6)
    p = perturbed(d, 4)
    d.params = p
    noisy, normal, albedo, depth, ref = synth(2, 160, 300, 7)  # 960 row tiles per convolution
    loss, g = d.gradients(noisy, normal, albedo, depth, ref)
    lo, go = ko.backward(p, ko.features(noisy, normal, albedo, depth), noisy, ref)
    assert loss == pytest.approx(lo, rel=1e-3)
    x, y = g.astype(np.float64), go
    assert x @ y / (np.linalg.norm(x) * np.linalg.norm(y)) > 0.999
    d.close()


def test_kpcn_gradients_match_oracle_with_several_strips_per_cta(rg):
    """450 images of 8 x 8: more column tiles than resident convolution CTAs,
    so each CTA convolves two or three strips in turn and its ring of input
    rows wraps across strip boundaries (forward and backward data)."""
    d = rg.Denoiser(seed=8)
    p = perturbed(d, 5)
    d.params = p
    noisy, normal, albedo, depth, ref = synth(450, 8, 8, 9)
    loss, g = d.gradients(noisy, normal, albedo, depth, ref)
    lo, go = ko.backward(p, ko.features(noisy, normal, albedo, depth), noisy, ref)
    assert loss == pytest.approx(lo, rel=1e-3)
    x, y = g.astype(np.float64), go
    assert x @ y / (np.linalg.norm(x) * np.linalg.norm(y)) > 0.999
    d.close()


def test_kpcn_gradients_match_oracle(rg):
    d = rg.Denoiser(seed=5)
    p = perturbed(d, 2)
    d.params = p
    noisy, normal, albedo, depth, ref = synth(2, 23, 29, 2)
    loss, g = d.gradients(noisy, normal, albedo, depth, ref, spp=512)
    lo, go = ko.backward(p, ko.features(noisy, normal, albedo, depth, spp=512), noisy, ref)
    assert loss == pytest.approx(lo, rel=1e-3)
    offs = np.cumsum([0] + [w + b for w, b in ko.layer_sizes()])
    for l, (wl, bl) in enumerate(ko.layer_sizes()):
        for a, b in ((offs[l], offs[l] + wl), (offs[l] + wl, offs[l + 1])):
            x, y = g[a:b].astype(np.float64), go[a:b]
            cos = x @ y / (np.linalg.norm(x) * np.linalg.norm(y) + 1e-30)
            assert cos > 0.999, (l, a, cos)
            assert abs(np.linalg.norm(x) / np.linalg.norm(y) - 1.0) < 0.01, (l, a)
    d.close()


def test_kpcn_training_steps_are_adam_on_the_gradient(rg):
    """Two replayed training steps on one example (batch 1) equal two Adam updates
    (b1 0.9, b2 0.999, eps 1e-8) with the gradient of that example at the current
    weights: the captured step's gather, backward and device-side step count."""
    d = rg.Denoiser(seed=11)
    d.params = perturbed(d, 6)
    noisy, normal, albedo, depth, ref = synth(1, 24, 40, 12)
    d.add_example(noisy[0], normal[0], albedo[0], depth[0], ref[0])
    lr, b1, b2, eps = 1e-3, 0.9, 0.999, 1e-8
    p = d.params.astype(np.float64)
    m = np.zeros_like(p)
    v = np.zeros_like(p)
    for t in (1, 2):
        loss, g = d.gradients(noisy, normal, albedo, depth, ref)
        g = g.astype(np.float64)
        m = b1 * m + (1 - b1) * g
        v = b2 * v + (1 - b2) * g * g
        want = p - lr * (m / (1 - b1 ** t)) / (np.sqrt(v / (1 - b2 ** t)) + eps)
        losses = d.train(1, 1, lr)
        assert losses[0] == pytest.approx(loss, rel=1e-5)
        p = d.params.astype(np.float64)
        np.testing.assert_allclose(p, want, rtol=0, atol=lr * 1e-3)
    d.close()


def test_kpcn_training_reduces_loss(rg):
    import importlib
    kt = importlib.import_module(rg.__name__ + ".kpcn_train")
    ex = kt.make_examples(rg, 8, size=64, spp_lo=4, spp_hi=128)
    d, losses = kt.train(rg, ex, steps=300, batch=4, lr=2e-3)
    assert np.all(np.isfinite(losses))
    assert losses[-30:].mean() < 0.7 * losses[:10].mean(), (losses[:10].mean(), losses[-30:].mean())
    d.close()


def test_pretrained_beats_atrous_on_held_out_jobs(rg):
    """What the trained network gains: relMSE against a 1024-spp render at 8 spp,
    on jobs whose seeds the training never saw, versus A-Trous and the raw input."""
    import importlib
    kt = importlib.import_module(rg.__name__ + ".kpcn_train")
    d = rg.Denoiser.pretrained()
    res = kt.evaluate(rg, d, count=6, size=96, spp_lo=8, spp_hi=1024, first=300000)
    assert res["learned"] < 0.5 * res["atrous"], res
    assert res["learned"] < 0.2 * res["noisy"], res
    assert res["learned_wins"] == res["jobs"], res
    d.close()


def test_renderer_and_server_use_the_learned_denoiser(rg):
    sc = rg.Scene.builtin(4, 77, [8000, 3])
    d = rg.Denoiser.pretrained()
    st = rg.RendererSettings(resolutionWidth=80, resolutionHeight=64, samples=8, maxDepth=6, seed=9, enableDenoise=True,
                             denoiseIntensity=0.0)
    r = rg.RayRenderer(st)
    r.set_scene(sc)
    r.render()
    noisy = r.get_hdr_result()
    normal, albedo, depth = r.get_aovs()
    expected = d.apply(noisy, normal, albedo, depth, spp=8)  # the renderer passes its per-pixel counts (8)
    r.settings.denoiseIntensity = 1.0
    r.set_denoiser(d)
    r.render()
    np.testing.assert_allclose(r.get_hdr_result(), expected, rtol=1e-5, atol=1e-6)
    r.set_denoiser(None)  # back to A-Trous
    r.render()
    assert np.abs(r.get_hdr_result() - expected).max() > 1e-3
    r.close()
    srv = rg.RenderServer(rg.RendererSettings(denoiseIntensity=1.0), max_resident_jobs=4)
    srv.set_denoiser(d)
    j = srv.submit(sc, 80, 64, 8, max_depth=6, seed=9, denoise=2)
    srv.wait(j)
    np.testing.assert_allclose(srv.result(j), expected, rtol=1e-4, atol=1e-5)
    srv.close()
    d.close()
