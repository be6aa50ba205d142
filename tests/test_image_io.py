"""Image files: rg_save_image writers (.hdr RGBE with RLE, .pfm, .jpg, .png,
.ppm) checked with independent decoders (OpenCV, PIL), the readers against an
independent writer, and the oracle's HDR bloom properties (no GPU).

Reference: the CLI's output step (src/main.cpp:479-485), decodeRadianceHDR
(texture.cpp:74-151), RayRenderer::applyPostProcess (rayrenderer.cpp:598-696).
"""
import json

import numpy as np
import pytest

import scenes

cv2 = pytest.importorskip("cv2")
Image = pytest.importorskip("PIL.Image")


def gradient(H=37, W=53, scale=1.0):
    y, x = np.mgrid[0:H, 0:W]
    img = np.stack([x / W, y / H, 0.5 + 0.5 * np.sin(x / 5.0) * np.cos(y / 7.0), np.ones_like(x, float)], -1)
    img[..., :3] *= scale
    return img.astype(np.float32)


@pytest.mark.parametrize("ext,min_psnr", [("png", 55.0), ("ppm", 55.0), ("jpg", 38.0), ("jpeg", 38.0)])
def test_ldr_writers_decode_with_pil(rg, tmp_path, ext, min_psnr):
    img = gradient()
    p = str(tmp_path / f"t.{ext}")
    rg.save_image(p, img)
    a = np.asarray(Image.open(p).convert("RGB")).astype(np.float64) / 255
    assert a.shape == img.shape[:2] + (3,)
    mse = np.mean((a - img[..., :3]) ** 2)
    assert 10 * np.log10(1 / max(mse, 1e-12)) > min_psnr
    if ext in ("png", "ppm"):  # lossless: round(clamp(v) * 255)
        np.testing.assert_array_equal(np.round(a * 255), np.round(np.clip(img[..., :3], 0, 1) * 255))


def test_jpeg_edges_and_clipping(rg, tmp_path):
    img = gradient(9, 13, scale=1.5)  # partial 8x8 blocks, values above 1 clip to white
    img[0, 0, :3] = -1.0
    rg.save_image(str(tmp_path / "e.jpg"), img)
    a = np.asarray(Image.open(tmp_path / "e.jpg").convert("RGB")).astype(np.float64) / 255
    assert np.abs(a - np.clip(img[..., :3], 0, 1)).mean() < 0.02


def test_hdr_writer_decodes_with_opencv(rg, tmp_path):
    img = gradient(21, 67, scale=40.0)
    img[3, :20, :3] = 0.0  # runs
    rg.save_image(str(tmp_path / "t.hdr"), img)
    a = cv2.imread(str(tmp_path / "t.hdr"), cv2.IMREAD_ANYDEPTH | cv2.IMREAD_COLOR)[..., ::-1]
    ref = img[..., :3]
    np.testing.assert_allclose(a, ref, rtol=0, atol=ref.max(-1, keepdims=True).repeat(3, -1).max() / 120)
    rel = np.abs(a - ref) / np.maximum(ref.max(-1, keepdims=True), 1e-6)
    assert rel.max() < 1.0 / 128


def test_pfm_writer_decodes_with_opencv(rg, tmp_path):
    img = gradient(11, 17, scale=7.0)
    rg.save_image(str(tmp_path / "t.pfm"), img)
    a = cv2.imread(str(tmp_path / "t.pfm"), cv2.IMREAD_UNCHANGED)[..., ::-1]
    np.testing.assert_array_equal(a, img[..., :3])


def test_reader_accepts_opencv_rgbe(rg, tmp_path):
    img = gradient(19, 45, scale=12.0)[..., :3]
    cv2.imwrite(str(tmp_path / "cv.hdr"), np.ascontiguousarray(img[..., ::-1]))
    (tmp_path / "s.json").write_text(json.dumps({"envmap": "cv.hdr"}))
    d = rg.Scene.from_json(str(tmp_path / "s.json")).desc
    t = d.textures[0]
    got = np.ctypeslib.as_array(t.rgba, shape=(t.height, t.width, 4))[..., :3]
    ref = cv2.imread(str(tmp_path / "cv.hdr"), cv2.IMREAD_ANYDEPTH | cv2.IMREAD_COLOR)[..., ::-1]
    np.testing.assert_allclose(got, ref, rtol=1e-6)


def test_save_image_errors(rg, tmp_path):
    with pytest.raises(rg.RayGenError) as e:
        rg.save_image(str(tmp_path / "t.tga"), gradient())
    assert e.value.code == rg.RG_ERR_UNSUPPORTED
    with pytest.raises(rg.RayGenError) as e:
        rg.save_image(str(tmp_path / "missing_dir" / "t.png"), gradient())
    assert e.value.code == rg.RG_ERR_IO


def hdr_with_spots(H=90, W=160, seed=0):
    rng = np.random.default_rng(seed)
    img = np.concatenate([rng.random((H, W, 3)) * 0.8, np.ones((H, W, 1))], axis=2).astype(np.float32)
    for _ in range(6):
        y, x = rng.integers(0, H), rng.integers(0, W)
        img[y, x, :3] = rng.uniform(20, 200, 3)
    return img


def test_oracle_bloom_below_threshold_is_identity(orc):
    img = hdr_with_spots()
    img[..., :3] = np.minimum(img[..., :3], 0.9)
    np.testing.assert_array_equal(orc.bloom(img, threshold=1.0), img)


def test_oracle_bloom_energy(orc):
    img = hdr_with_spots(seed=2)
    out = orc.bloom(img, threshold=0.0, strength=1.0, radius=0.02, size_aspect=0.25)
    added = (out - img)[..., :3].sum(axis=(0, 1))
    assert np.allclose(added, img[..., :3].sum(axis=(0, 1)), rtol=0.03)
    assert np.array_equal(out[..., 3], img[..., 3])
    # a halo spreads around each spot
    assert (out[..., :3] - img[..., :3]).min() >= 0.0
