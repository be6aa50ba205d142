"""CPU oracle of the learned denoiser (test infrastructure only).

The kernel-predicting CNN (KPCN, after Bako et al. 2017, "Kernel-predicting
convolutional networks for denoising Monte Carlo renderings") in numpy, forward
and backward, with the device's rounding points:
* features X0 [N, H, W, 16]: log1p(max(radiance, 0)) (3), albedo (3), the
  normal guide n * 0.5 + 0.5 (3), the depth guide (1), the noise level
  log2(1 + spp) / 12 (1), zeros (5) -- BF16;
* five 3x3 convolutions with ReLU (16 -> 32, then 32 -> 32), zero padding,
  weights BF16, accumulation wide, outputs rounded to BF16;
* a 3x3 convolution 32 -> 25 logits (padded to 32 channels), FP32;
* softmax over the 25 logits -> a 5 x 5 kernel per pixel, applied to the noisy
  radiance with clamp-to-edge sampling;
* loss: relMSE, mean over pixels and channels of (o - r)^2 / (r^2 + 0.01).
Backward: the head gradient and the data gradients are rounded to BF16 where
the device stores them; weight and bias gradients accumulate wide.

Parameter vector (FP32): for each layer l, W_l [32, 9, Cin_l] (output channel,
tap (dy + 1) * 3 + (dx + 1), input channel) then b_l [32]; Cin = 16, 32, ... .
`exact=True` skips every rounding (float64 throughout) for finite differences.
"""
import numpy as np

CIN = [16, 32, 32, 32, 32, 32]
C = 32
KP = 25
EPS = 0.01


def layer_sizes():
    return [(C * 9 * cin, C) for cin in CIN]


def num_params():
    return sum(w + b for w, b in layer_sizes())


def unpack(params):
    out, o = [], 0
    for cin in CIN:
        n = C * 9 * cin
        W = params[o:o + n].reshape(C, 9, cin)
        o += n
        b = params[o:o + C]
        o += C
        out.append((W, b))
    return out


def bf16(a):
    """Round to BF16 (nearest even) and back, as float64."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint32) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def features(noisy, normal, albedo, depth, spp=8.0, exact=False):
    """noisy [N,H,W,>=3], normal/albedo [N,H,W,3] guides, depth [N,H,W], samples per
    pixel (a number or an [N,H,W] array) -> X0 [N,H,W,16]."""
    N, H, W = depth.shape
    X = np.zeros((N, H, W, 16))
    X[..., 0:3] = np.log1p(np.maximum(noisy[..., :3], 0.0))
    X[..., 3:6] = albedo
    X[..., 6:9] = normal
    X[..., 9] = depth
    X[..., 10] = np.log2(1.0 + np.maximum(np.asarray(spp, np.float64), 0.0)) / 12.0
    return X if exact else bf16(X)


def shift(X, dy, dx):
    """S[n, y, x] = X[n, y + dy, x + dx] (zero outside)."""
    N, H, W, Cc = X.shape
    S = np.zeros_like(X)
    ys, ye = max(0, -dy), min(H, H - dy)
    xs, xe = max(0, -dx), min(W, W - dx)
    S[:, ys:ye, xs:xe] = X[:, ys + dy:ye + dy, xs + dx:xe + dx]
    return S


TAPS = [(t // 3 - 1, t % 3 - 1) for t in range(9)]
KOFF = [(j // 5 - 2, j % 5 - 2) for j in range(KP)]


def conv(X, W, b):
    out = np.zeros(X.shape[:3] + (W.shape[0],))
    for t, (dy, dx) in enumerate(TAPS):
        out += shift(X, dy, dx) @ W[:, t, :].T
    return out + b


def gather_clamped(img, dy, dx):
    N, H, W, _ = img.shape
    ys = np.clip(np.arange(H) + dy, 0, H - 1)
    xs = np.clip(np.arange(W) + dx, 0, W - 1)
    return img[:, ys][:, :, xs]


def forward(params, X0, noisy, exact=False):
    """-> dict with activations, logits, kernel weights and the filtered radiance [N,H,W,3]."""
    r = (lambda a: a) if exact else bf16
    layers = unpack(np.asarray(params, np.float64))
    acts = [X0]
    X = X0
    for l, (W, b) in enumerate(layers):
        Wr = r(W)
        Y = conv(X, Wr, np.asarray(b, np.float64))
        if l < 5:
            Y = r(np.maximum(Y, 0.0))
            acts.append(Y)
            X = Y
        else:
            Z = Y.astype(np.float64) if exact else Y.astype(np.float32).astype(np.float64)
    z = Z[..., :KP]
    z = z - z.max(axis=-1, keepdims=True)
    e = np.exp(z)
    w = e / e.sum(axis=-1, keepdims=True)
    nz = noisy[..., :3].astype(np.float64)
    out = np.zeros(nz.shape)
    for j, (dy, dx) in enumerate(KOFF):
        out += w[..., j:j + 1] * gather_clamped(nz, dy, dx)
    return {"acts": acts, "logits": Z, "w": w, "out": out}


def loss_of(out, ref):
    r = ref[..., :3].astype(np.float64)
    return float(np.mean((out - r) ** 2 / (r * r + EPS)))


def backward(params, X0, noisy, ref, exact=False):
    """-> (loss, gradient vector)."""
    r = (lambda a: a) if exact else bf16
    layers = unpack(np.asarray(params, np.float64))
    f = forward(params, X0, noisy, exact)
    out, w = f["out"], f["w"]
    rr = ref[..., :3].astype(np.float64)
    P = out.shape[0] * out.shape[1] * out.shape[2]
    loss = float(np.mean((out - rr) ** 2 / (rr * rr + EPS)))
    dO = 2.0 * (out - rr) / (rr * rr + EPS) / (3.0 * P)
    nz = noisy[..., :3].astype(np.float64)
    dw = np.zeros(w.shape)
    for j, (dy, dx) in enumerate(KOFF):
        dw[..., j] = (dO * gather_clamped(nz, dy, dx)).sum(axis=-1)
    dz = w * (dw - (w * dw).sum(axis=-1, keepdims=True))
    G = np.zeros(f["logits"].shape)
    G[..., :KP] = dz
    G = r(G)
    grads = [None] * 6
    for l in range(5, -1, -1):
        W, b = layers[l]
        Xin = f["acts"][l]
        dW = np.zeros(W.shape)
        for t, (dy, dx) in enumerate(TAPS):
            S = shift(Xin, dy, dx).reshape(-1, Xin.shape[-1])
            dW[:, t, :] = G.reshape(-1, C).T @ S
        db = G.reshape(-1, C).sum(axis=0)
        grads[l] = (dW, db)
        if l > 0:
            Wr = r(W)
            dX = np.zeros(Xin.shape)
            for t, (dy, dx) in enumerate(TAPS):
                dX += shift(G, -dy, -dx) @ Wr[:, t, :]
            dX = dX * (Xin > 0)
            G = r(dX)
    flat = np.concatenate([np.concatenate([dW.ravel(), db]) for dW, db in grads])
    return loss, flat


def init_params(seed):
    """He-normal weights (fan-in 9 * Cin; the 11 real input channels for layer 1), zero biases;
    the 7 padding logits of the last layer stay zero."""
    rng = np.random.default_rng(seed)
    ps = []
    for l, cin in enumerate(CIN):
        fan = 9 * (11 if l == 0 else cin)
        W = rng.standard_normal((C, 9, cin)) * np.sqrt(2.0 / fan)
        if l == 0:
            W[:, :, 11:] = 0.0
        if l == 5:
            W *= 0.1
            W[KP:] = 0.0
        ps.append(W.ravel())
        ps.append(np.zeros(C))
    return np.concatenate(ps).astype(np.float32)
