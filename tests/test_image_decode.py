"""JPEG and PNG readers (rg_load_image; the loader's 'tex' textures).

PNG must decode exactly: files from the test-side writer cover every colour
type and bit depth, all five row filters, palettes with transparency and
Adam7 interlacing.  JPEG: files from the test-side baseline encoder (own
Huffman tables, 4:4:4 / 4:2:0 / 4:2:2 / grey, restart intervals) must decode
to the encoder's own reconstruction of its quantised coefficients within one
level in 255.  Texture::loadFromFile (texture.cpp:170-195) and
SceneResourcePool::getTexture (scene.cpp:597-681) for the loader side.
"""
import json
import os

import numpy as np
import pytest

import image_codecs as ic

# The reference project's texture folder (resources/textures of its checkout),
# when one is available: RAYGEN_REFERENCE_ROOT names the checkout's root.
REF_TEXTURES = os.path.join(os.environ.get("RAYGEN_REFERENCE_ROOT", ""), "resources", "textures") \
    if os.environ.get("RAYGEN_REFERENCE_ROOT") else ""


def _png_case(rng, ctype, depth, H=13, W=17):
    maxv = (1 << depth) - 1
    if ctype == 3:
        n = min(1 << depth, 40)
        pal = rng.integers(0, 256, (n, 3))
        idx = rng.integers(0, n, (H, W, 1))
        trns = rng.integers(0, 256, n // 2)
        alpha = np.ones((H, W))
        alpha_idx = idx[..., 0] < len(trns)
        alpha[alpha_idx] = trns[idx[..., 0][alpha_idx]] / 255.0
        rgb = pal[idx[..., 0]] / 255.0
        return idx, dict(palette=pal, trns=trns), np.concatenate([rgb, alpha[..., None]], axis=-1)
    chans = {0: 1, 2: 3, 4: 2, 6: 4}[ctype]
    s = rng.integers(0, maxv + 1, (H, W, chans))
    f = s / maxv
    if ctype == 0:
        want = np.concatenate([f, f, f, np.ones((H, W, 1))], axis=-1)
    elif ctype == 4:
        want = np.concatenate([f[..., :1]] * 3 + [f[..., 1:2]], axis=-1)
    elif ctype == 2:
        want = np.concatenate([f, np.ones((H, W, 1))], axis=-1)
    else:
        want = f
    return s, {}, want


PNG_CASES = [(0, d) for d in (1, 2, 4, 8, 16)] + [(3, d) for d in (1, 2, 4, 8)] + \
            [(c, d) for c in (2, 4, 6) for d in (8, 16)]


@pytest.mark.parametrize("interlace", [False, True])
@pytest.mark.parametrize("ctype,depth", PNG_CASES)
def test_png_decodes_exactly(rg, tmp_path, ctype, depth, interlace):
    rng = np.random.default_rng(ctype * 100 + depth + 7 * interlace)
    samples, extra, want = _png_case(rng, ctype, depth)
    p = str(tmp_path / "t.png")
    ic.write_png(p, samples, ctype, depth, interlace=interlace, seed=depth, **extra)
    img, hdr = rg.load_image(p)
    assert not hdr and img.shape == want.shape
    np.testing.assert_allclose(img, want, rtol=0, atol=1e-6)


def test_png_rejects_corruption(rg, tmp_path):
    p = tmp_path / "bad.png"
    ic.write_png(str(p), np.zeros((4, 4, 3), np.int64), 2, 8)
    b = bytearray(p.read_bytes())
    b[40] ^= 0x55  # inside IDAT: the chunk CRC no longer matches
    p.write_bytes(bytes(b))
    with pytest.raises(rg.RayGenError):
        rg.load_image(str(p))


def _photo(rng, H, W, noise=6.0):
    """Smooth image with edges: gradients, a disc, noise."""
    y, x = np.mgrid[0:H, 0:W]
    r = 128 + 100 * np.sin(x / 7.0) * np.cos(y / 9.0)
    g = 255 * x / max(1, W - 1)
    b = np.where((x - W / 2) ** 2 + (y - H / 2) ** 2 < (min(H, W) / 3) ** 2, 230, 30)
    img = np.stack([r, g, b], axis=-1) + rng.normal(0, noise, (H, W, 3))
    return np.clip(np.round(img), 0, 255)


@pytest.mark.parametrize("sampling,restart,size", [
    (((1, 1), (1, 1), (1, 1)), 0, (24, 40)),
    (((2, 2), (1, 1), (1, 1)), 0, (37, 53)),
    (((2, 2), (1, 1), (1, 1)), 3, (64, 48)),
    (((2, 1), (1, 1), (1, 1)), 2, (21, 35)),
    (((1, 2), (1, 1), (1, 1)), 0, (30, 18)),
])
def test_jpeg_baseline_matches_the_encoders_reconstruction(rg, tmp_path, sampling, restart, size):
    H, W = size
    rng = np.random.default_rng(H * W)
    img = _photo(rng, H, W)
    p = str(tmp_path / "t.jpg")
    comps, geom = ic.encode_jpeg(p, img, sampling=sampling, restart=restart)
    want = ic.jpeg_expected(comps, geom)
    got, hdr = rg.load_image(p)
    assert not hdr and got.shape == (H, W, 4)
    diff = np.abs(got[..., :3] - want) * 255
    assert diff.max() <= 1.0 + 1e-3, diff.max()
    assert diff.mean() < 0.05
    assert np.all(got[..., 3] == 1.0)
    # and the image itself survives the round trip (JPEG is lossy)
    assert np.abs(got[..., :3] * 255 - img).mean() < 8


@pytest.mark.parametrize("restart", [0, 5])
def test_jpeg_greyscale(rg, tmp_path, restart):
    rng = np.random.default_rng(3)
    img = _photo(rng, 45, 29)[..., 1]
    p = str(tmp_path / "g.jpg")
    comps, geom = ic.encode_jpeg(p, img, grey=True, restart=restart)
    want = ic.jpeg_expected(comps, geom, grey=True)
    got, _ = rg.load_image(p)
    assert np.abs(got[..., :3] - want).max() * 255 <= 1.0 + 1e-3
    assert np.all(got[..., 0] == got[..., 1])


def test_jpeg_round_trip_through_the_writer(rg, tmp_path):
    rng = np.random.default_rng(5)
    img = np.concatenate([_photo(rng, 40, 56, noise=0.0) / 255.0, np.ones((40, 56, 1))], axis=-1).astype(np.float32)
    p = str(tmp_path / "w.jpg")
    rg.save_image(p, img)  # quality 92, 4:4:4
    got, _ = rg.load_image(p)
    err = np.abs(got[..., :3] - img[..., :3]) * 255
    assert err.mean() < 3.0  # quality 92: ringing only at the disc's hard edge
    flat = np.ones((16, 16, 4), np.float32)
    flat[..., :3] = np.array([100, 150, 200]) / 255.0
    rg.save_image(p, flat)
    got, _ = rg.load_image(p)
    assert np.abs(got[..., :3] * 255 - np.array([100, 150, 200])).max() <= 1.0 + 1e-3


def test_jpeg_refuses_progressive_and_garbage(rg, tmp_path):
    p = tmp_path / "prog.jpg"
    ic.encode_jpeg(str(p), _photo(np.random.default_rng(1), 16, 16))
    b = bytearray(p.read_bytes())
    i = b.index(b"\xff\xc0")
    b[i + 1] = 0xC2  # SOF2: progressive
    p.write_bytes(bytes(b))
    with pytest.raises(rg.RayGenError, match="progressive"):
        rg.load_image(str(p))
    q = tmp_path / "junk.jpg"
    q.write_bytes(b"\xff\xd8\xff\xe0\x00\x02garbage")
    with pytest.raises(rg.RayGenError):
        rg.load_image(str(q))


@pytest.mark.skipif(not REF_TEXTURES or not os.path.isdir(REF_TEXTURES),
                    reason="RAYGEN_REFERENCE_ROOT does not name a reference checkout with its textures")
def test_reference_textures_decode(rg):
    """The reference's own JPEG textures: a grey checkerboard, and 4:2:0 images
    with restart intervals (only where the reference tree is present)."""
    chk, _ = rg.load_image(os.path.join(REF_TEXTURES, "checkerboard.jpg"))
    assert chk.shape == (256, 256, 4) and np.all(chk[..., 0] == chk[..., 2])
    lv = np.sort(np.unique(np.round(chk[..., 0] * 255)))
    assert lv[0] < 60 and lv[-1] > 190  # two tones
    for name, shape in (("wood.jpg", (1024, 1024, 4)), ("sky_test.jpg", (512, 1024, 4))):
        img, hdr = rg.load_image(os.path.join(REF_TEXTURES, name))
        assert img.shape == shape and not hdr
        assert 0.05 < img[..., :3].mean() < 0.95 and img[..., :3].std() > 0.02
        # no blocky garbage: neighbouring pixels mostly agree
        assert np.abs(np.diff(img[..., :3], axis=1)).mean() < 0.05


def test_loader_resolves_tex_through_a_pool(rg, tmp_path):
    rng = np.random.default_rng(8)
    ic.write_png(str(tmp_path / "a.png"), rng.integers(0, 256, (8, 8, 3)), 2, 8)
    ic.encode_jpeg(str(tmp_path / "b.jpg"), _photo(rng, 16, 24))
    doc = {
        "_materials": {"shared": {"tex": "a.png", "texTiling": [2, 3]}},
        "p1": {"mesh": {"type": "plane"}, "mat": "shared"},
        "p2": {"mesh": {"type": "plane"}, "mat": {"tex": "a.png"}},
        "p3": {"mesh": {"type": "plane"}, "mat": {"tex": "b.jpg", "color": [0.5, 0.5, 0.5]}},
        "p4": {"mesh": {"type": "plane"}, "mat": {"tex": "missing.png"}},
        "p5": {"mesh": {"type": "plane"}, "mat": {"tex": "tob://bundle/12"}},
    }
    (tmp_path / "s.json").write_text(json.dumps(doc))
    d = rg.Scene.from_json(str(tmp_path / "s.json")).desc
    texs = [d.materials[d.objects[i].material].texture for i in range(d.num_objects)]
    assert texs[0] == texs[1] >= 0 and texs[2] >= 0 and texs[2] != texs[0]
    assert texs[3] == -1 and texs[4] == -1 and d.num_textures == 2
    assert list(d.materials[d.objects[0].material].tex_tiling) == [2, 3]
    t = d.textures[texs[2]]
    assert (t.width, t.height, t.is_hdr) == (24, 16, 0)
