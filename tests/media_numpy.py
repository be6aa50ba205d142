"""From-scratch numpy (float32) restatement of the procedural medium fields,
used to pin the oracle: the lattice hash and trilinear value noise, the fBm
sum, densityAt, the cone and path emission profiles and the heat-haze bend
(medium.cpp:127-404).  Every operation is a single float32 operation in the
reference's evaluation order, so the noise values must agree bit for bit.
"""
import numpy as np

F = np.float32


def hash3(x, y, z):
    x = np.asarray(x, np.int64) & 0xFFFFFFFF
    y = np.asarray(y, np.int64) & 0xFFFFFFFF
    z = np.asarray(z, np.int64) & 0xFFFFFFFF
    h = (x * 374761393 + y * 668265263 + z * 2147483647) & 0xFFFFFFFF
    h = ((h ^ (h >> 13)) * 1274126177) & 0xFFFFFFFF
    h ^= h >> 16
    return (h & 0xFFFFFF).astype(F) / F(16777216.0)


def _smooth(x):
    return x * x * (F(3.0) - F(2.0) * x)


def value_noise(x, y, z):
    fx, fy, fz = np.floor(x), np.floor(y), np.floor(z)
    xi, yi, zi = fx.astype(np.int64), fy.astype(np.int64), fz.astype(np.int64)
    xf = _smooth(x - fx.astype(F))
    yf = _smooth(y - fy.astype(F))
    zf = _smooth(z - fz.astype(F))
    one = F(1.0)

    def lerp(a, b, t):
        return a * (one - t) + b * t

    x00 = lerp(hash3(xi, yi, zi), hash3(xi + 1, yi, zi), xf)
    x10 = lerp(hash3(xi, yi + 1, zi), hash3(xi + 1, yi + 1, zi), xf)
    x01 = lerp(hash3(xi, yi, zi + 1), hash3(xi + 1, yi, zi + 1), xf)
    x11 = lerp(hash3(xi, yi + 1, zi + 1), hash3(xi + 1, yi + 1, zi + 1), xf)
    return lerp(lerp(x00, x10, yf), lerp(x01, x11, yf), zf)


def fbm(x, y, z, freq, octaves, gain, lac):
    fx, fy, fz = x * F(freq), y * F(freq), z * F(freq)
    amp, total, amp_sum = F(1.0), np.zeros_like(fx), F(0.0)
    for _ in range(max(1, octaves)):
        total = total + amp * value_noise(fx, fy, fz)
        amp_sum = F(amp_sum + amp)
        amp = F(amp * F(gain))
        fx, fy, fz = fx * F(lac), fy * F(lac), fz * F(lac)
    return total / amp_sum


def density(p, freq, octaves, gain, lac, amplitude, bias, offset=(0, 0, 0)):
    p = np.asarray(p, F)
    n = fbm(p[:, 0] - F(offset[0]), p[:, 1] - F(offset[1]), p[:, 2] - F(offset[2]), freq, octaves, gain, lac)
    return np.maximum(F(0.0), F(amplitude) * n + F(bias))


def cone_emission(p, origin, axis, length, radius, inner, outer, intensity, peak, sharp, dens=1.0):
    """Cone profile (medium.cpp:356-403) at camera-space points; axis unit length."""
    p = np.asarray(p, F)
    o, a = np.asarray(origin, F), np.asarray(axis, F)
    rel = p - o
    ax = rel[:, 0] * a[0] + rel[:, 1] * a[1] + rel[:, 2] * a[2]
    u = ax / F(length)
    perp = rel - a[None, :] * ax[:, None]
    r2 = perp[:, 0] * perp[:, 0] + perp[:, 1] * perp[:, 1] + perp[:, 2] * perp[:, 2]
    v2 = r2 / (F(radius) * F(radius))
    dx = (u - F(peak)) * F(sharp)
    t = np.exp(-(dx * dx)).astype(F) * ((F(1) - v2) * (F(1) - v2))
    col = np.asarray(inner, F)[None, :] * t[:, None] + np.asarray(outer, F)[None, :] * (F(1) - t)[:, None]
    scale = t * F(intensity) * F(max(0.0, dens))
    out = col * scale[:, None]
    out[(u < 0) | (u > 1) | (v2 > 1) | (t <= 0)] = 0
    return out


def path_emission(p, pts, inner, outer, intensity, falloff, dens=1.0):
    """Tube profile (medium.cpp:310-354); pts: list of (xyz, radius, t) in camera space."""
    p = np.asarray(p, np.float64)
    best_d2 = np.full(len(p), np.inf)
    best_t = np.zeros(len(p))
    best_r = np.zeros(len(p))
    for (a, ra, ta), (b, rb, tb) in zip(pts[:-1], pts[1:]):
        a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
        ab = b - a
        ab2 = ab @ ab
        if ab2 < 1e-12:
            continue
        u = np.clip(((p - a) @ ab) / ab2, 0.0, 1.0)
        q = a + u[:, None] * ab
        d2 = ((p - q) ** 2).sum(axis=1)
        m = d2 < best_d2
        best_d2[m] = d2[m]
        best_t[m] = ta + (tb - ta) * u[m]
        best_r[m] = ra + (rb - ra) * u[m]
    out = np.zeros((len(p), 3))
    ok = (best_r > 0) & (best_d2 < best_r * best_r)
    r = np.sqrt(best_d2[ok]) / best_r[ok]
    radial = np.maximum(0.0, 1.0 - r) ** falloff
    tb = np.clip(best_t[ok], 0.0, 1.0)
    col = np.asarray(inner)[None, :] * (1 - tb)[:, None] + np.asarray(outer)[None, :] * tb[:, None]
    out[ok] = col * (radial * intensity * max(0.0, dens))[:, None]
    return out


def ior(p, amplitude, freq, octaves, gain, lac, offset=(0, 0, 0)):
    p = np.asarray(p, F)
    n = fbm(p[:, 0] - F(offset[0]), p[:, 1] - F(offset[1]), p[:, 2] - F(offset[2]), freq, octaves, gain, lac)
    return F(1.0) + F(amplitude) * F(1.0) * (n - F(0.5)) * F(2.0)


def bend(rays, amplitude, freq, octaves, gain, lac, steps):
    """bendRay (medium.cpp:237-274) without falloff: rays n x 7 -> n x 6."""
    rays = np.asarray(rays, F)
    pos, d, length = rays[:, 0:3].copy(), rays[:, 3:6].copy(), rays[:, 6]
    ds = length / F(steps)
    h = F(0.5) / F(freq)
    inv2h = F(0.5) / h
    f = lambda q: ior(q, amplitude, freq, octaves, gain, lac)
    for _ in range(steps):
        mid = pos + d * (ds * F(0.5))[:, None]
        n = f(mid)
        g = np.zeros_like(mid)
        for k in range(3):
            e = np.zeros(3, F)
            e[k] = 1
            hp, hm = mid.copy(), mid.copy()
            hp[:, k] = mid[:, k] + h
            hm[:, k] = mid[:, k] - h
            g[:, k] = (f(hp) - f(hm)) * inv2h
        gd = g[:, 0] * d[:, 0] + g[:, 1] * d[:, 1] + g[:, 2] * d[:, 2]
        perp = g - d * gd[:, None]
        inv_n = np.where(n > F(1e-6), F(1.0) / n, F(1.0)).astype(F)
        nd = d + perp * (ds * inv_n)[:, None]
        l2 = nd[:, 0] * nd[:, 0] + nd[:, 1] * nd[:, 1] + nd[:, 2] * nd[:, 2]
        inv_l = F(1.0) / np.sqrt(l2)
        d = np.where((l2 > F(1e-12))[:, None], nd * inv_l[:, None], d).astype(F)
        pos = pos + d * ds[:, None]
    return np.concatenate([pos, d], axis=1)
