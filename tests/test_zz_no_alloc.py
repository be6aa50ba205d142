"""A-Trous on caller device buffers without allocating
(rg_denoise_atrous_noalloc), checked through the C ABI against the allocating
entry point rg_denoise_atrous on the same inputs.

The file sorts last so that, in a full run, the no-alloc path also runs after
every other GPU test of the process; it passes alone in a fresh process too.
Both entry points run the same kernels on the same inputs, so their outputs
must be equal bit for bit (the allocating entry point is itself checked
against the CPU oracle within 1e-4 relative in test_gpu_post.py).
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_PIXELS = 1 << 20


def make_inputs(seed, h, w):
    rng = np.random.default_rng(seed)
    color = (rng.random((h, w, 3)) * 2).astype(np.float32)
    color[h // 3, w // 4] = 60.0  # firefly
    q = lambda a: a.astype(np.float16).astype(np.float32)
    normal = q(rng.random((h, w, 3)).astype(np.float32) * 0.2 + 0.4)
    depth = q(rng.random((h, w)).astype(np.float32))
    albedo = q(rng.random((h, w, 3)).astype(np.float32))
    alpha = (rng.random((h, w)) > 0.1).astype(np.float32)
    return color, normal, depth, albedo, alpha


def bind(lib):
    f = lib.rg_denoise_atrous_noalloc
    f.restype = C.c_int32
    f.argtypes = [C.c_int32, C.c_int32] + [C.c_void_p] * 5 + [C.c_int32] + [C.c_float] * 4 + [C.c_void_p, C.c_void_p]
    return f


def run_noalloc(f, torch, inputs, stream, levels=5, params=(0.4, 128.0, 0.1, 1.0)):
    color, normal, depth, albedo, alpha = inputs
    h, w = color.shape[:2]
    dev = torch.device("cuda:0")
    rgba = np.concatenate([color, np.ones((h, w, 1), np.float32)], axis=2)
    bufs = [torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in (rgba, normal, depth, albedo, alpha)]
    out = torch.full((h, w, 4), float("nan"), dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    rc = f(w, h, *[b.data_ptr() for b in bufs], levels, *params, out.data_ptr(), stream)
    torch.cuda.synchronize()
    return rc, out.cpu().numpy()


def test_noalloc_matches_allocating_entry_point(rg):
    torch = pytest.importorskip("torch")
    lib = rg.load_library()
    f = bind(lib)
    stream = torch.cuda.Stream()
    # two calls in a row; the second is smaller and reuses what the first left in the working buffers
    for seed, (h, w) in [(11, (72, 96)), (12, (40, 56))]:
        inputs = make_inputs(seed, h, w)
        rc, got = run_noalloc(f, torch, inputs, stream.cuda_stream)
        assert rc == 0, lib.rg_last_error()
        ref = rg.denoise_atrous(*inputs)
        np.testing.assert_array_equal(got[..., :3], ref)
        assert np.all(got[..., 3] == 1.0)


def test_noalloc_default_stream_and_parameters(rg):
    torch = pytest.importorskip("torch")
    lib = rg.load_library()
    f = bind(lib)
    inputs = make_inputs(13, 33, 47)
    rc, got = run_noalloc(f, torch, inputs, None, levels=3, params=(0.8, 64.0, 0.2, 0.6))
    assert rc == 0, lib.rg_last_error()
    ref = rg.denoise_atrous(*inputs, levels=3, sigma_color=0.8, sigma_normal=64.0, sigma_depth=0.2, intensity=0.6)
    np.testing.assert_array_equal(got[..., :3], ref)


def test_noalloc_rejects_oversize_and_host_buffers(rg):
    torch = pytest.importorskip("torch")
    lib = rg.load_library()
    f = bind(lib)
    dev = torch.device("cuda:0")
    small = torch.zeros(64, dtype=torch.float32, device=dev)
    p = small.data_ptr()
    # larger than the working buffers: refused on the host before any device work
    rc = f(1025, 1024, p, p, p, p, p, 5, 0.4, 128.0, 0.1, 1.0, p, None)
    assert rc == rg.RG_ERR_INVALID_ARGUMENT
    assert b"1048576" in lib.rg_last_error()
    assert 1024 * 1024 <= MAX_PIXELS
    # host memory is refused by the pointer check on the host (no kernel is launched)
    host = np.zeros(64, np.float32)
    hp = host.ctypes.data
    rc = f(4, 4, hp, p, p, p, p, 5, 0.4, 128.0, 0.1, 1.0, p, None)
    assert rc == rg.RG_ERR_INVALID_ARGUMENT
    assert b"not device memory" in lib.rg_last_error()


def test_noalloc_rejects_bad_levels_and_aliased_output(rg):
    torch = pytest.importorskip("torch")
    lib = rg.load_library()
    f = bind(lib)
    dev = torch.device("cuda:0")
    h, w = 8, 8
    color = torch.zeros((h, w, 4), dtype=torch.float32, device=dev)
    guides = torch.zeros((h, w, 3), dtype=torch.float32, device=dev)
    depth = torch.zeros((h, w), dtype=torch.float32, device=dev)
    out = torch.zeros((h, w, 4), dtype=torch.float32, device=dev)
    args = [color.data_ptr(), guides.data_ptr(), depth.data_ptr(), guides.data_ptr(), depth.data_ptr()]
    for levels in (0, -1, 17, 1 << 20):
        rc = f(w, h, *args, levels, 0.4, 128.0, 0.1, 1.0, out.data_ptr(), None)
        assert rc == rg.RG_ERR_INVALID_ARGUMENT
        assert b"levels" in lib.rg_last_error()
    # the output may not share memory with an input (here: the colour itself)
    rc = f(w, h, *args, 5, 0.4, 128.0, 0.1, 1.0, color.data_ptr(), None)
    assert rc == rg.RG_ERR_INVALID_ARGUMENT
    assert b"overlaps" in lib.rg_last_error()
    # a valid call still succeeds afterwards
    rc = f(w, h, *args, 5, 0.4, 128.0, 0.1, 1.0, out.data_ptr(), None)
    torch.cuda.synchronize()
    assert rc == 0, lib.rg_last_error()
