"""Small analytic scenes for known-answer and parity tests (built from arrays)."""
import math

import numpy as np


def material(rg, color=(0.8, 0.8, 0.8), emission=0.0, glossy=0.0, roughness=0.5, metallic=0.0,
             refraction=0.0, ior=1.45, transparency=0.0):
    m = rg.rg_material()
    for i in range(3):
        m.color[i] = color[i]
    m.diffuse = 0.8
    m.glossy = glossy
    m.roughness = roughness
    m.metallic = metallic
    m.refraction = refraction
    m.refraction_ratio = ior
    m.transparency = transparency
    m.emission = emission
    m.texture = -1
    m.tex_tiling[0] = m.tex_tiling[1] = 1.0
    return m


def camera(rg, loc=(0, 0, 0), fov=40.0):
    c = rg.rg_camera()
    for i in range(3):
        c.location[i] = loc[i]
        c.angle[i] = 0.0
    c.field_of_view = fov
    c.view_near = 0.1
    c.view_far = 50.0
    c.depth_of_field = 0.0
    c.aperture = 1.8
    c.aperture_blades = 0
    c.exposure = 1.0
    return c


def quad_z(z, half, facing):
    """Axis-aligned square in the plane z, normal +z (facing=+1) or -z (facing=-1)."""
    a, b, c, d = (-half, -half, z), (half, -half, z), (half, half, z), (-half, half, z)
    if facing < 0:
        b, d = d, b
    n = (0.0, 0.0, float(facing))
    tris = [a + b + c, a + c + d]
    return np.array(tris, np.float32), np.array([n * 3, n * 3], np.float32)


def build(rg, parts, cam, media=(), global_medium=-1):
    """parts: list of (positions n x 9, normals n x 9, rg_material, interior_medium)."""
    pos, nrm, tri_mesh, mesh_obj, objs, mats = [], [], [], [], [], []
    for k, (p, n, m, med) in enumerate(parts):
        pos.append(p)
        nrm.append(n)
        tri_mesh += [k] * len(p)
        mesh_obj.append(k)
        o = rg.rg_object()
        o.material = k
        o.interior_medium = med
        objs.append(o)
        mats.append(m)
    return rg.Scene.from_arrays(np.concatenate(pos), np.concatenate(nrm), tri_mesh, mesh_obj, objs, mats, cam,
                                media=media, global_medium=global_medium)


def form_factor_centered_square(half, h):
    """Point-to-parallel-square form factor, point below the centre (four corner rectangles)."""
    X = Y = half / h
    f = (X / math.sqrt(1 + X * X) * math.atan(Y / math.sqrt(1 + X * X))
         + Y / math.sqrt(1 + Y * Y) * math.atan(X / math.sqrt(1 + Y * Y))) / (2 * math.pi)
    return 4.0 * f


def lit_floor_scene(rg, albedo=0.5, le=2.0, half=3.0, h=3.0):
    """Diffuse floor at z=-2 facing +z under an emitter at z=-2+h facing -z; camera at z=0 looking -z."""
    fp, fn = quad_z(-2.0, 50.0, +1)
    lp, ln = quad_z(-2.0 + h, half, -1)
    parts = [(fp, fn, material(rg, (albedo,) * 3), -1), (lp, ln, material(rg, (1, 1, 1), emission=le), -1)]
    return build(rg, parts, camera(rg, fov=1.0)), albedo * le * form_factor_centered_square(half, h)


def mirror_scene(rg, le=3.0):
    """Smooth metal mirror (F0 = 1) at z=-2 reflecting an emitter at z=+3 facing -z."""
    mp, mn = quad_z(-2.0, 10.0, +1)
    lp, ln = quad_z(3.0, 10.0, -1)
    parts = [(mp, mn, material(rg, (1, 1, 1), glossy=1.0, metallic=1.0, roughness=0.0), -1),
             (lp, ln, material(rg, (1, 1, 1), emission=le), -1)]
    return build(rg, parts, camera(rg, fov=10.0)), le


def absorber_scene(rg, sigma_a=0.1, d=5.0, le=2.0):
    """Emitter at z=-d facing +z seen through a purely absorbing global medium."""
    lp, ln = quad_z(-d, 50.0, +1)
    med = rg.rg_medium()
    for i in range(3):
        med.sigma_a[i] = sigma_a
        med.sigma_s[i] = 0.0
        med.sigma_e[i] = 0.0
    med.g = 0.0
    med.density = 1.0
    parts = [(lp, ln, material(rg, (1, 1, 1), emission=le), -1)]
    return build(rg, parts, camera(rg, fov=1.0), media=[med], global_medium=0), le * math.exp(-sigma_a * d)


def random_rays(scene_bounds, n, seed, camera_fraction=0.5, camera=(0, 0, 0)):
    """Rays in view space: a mix of camera rays and rays from random interior points."""
    rng = np.random.default_rng(seed)
    lo, hi = np.asarray(scene_bounds[0], np.float32), np.asarray(scene_bounds[1], np.float32)
    nc = int(n * camera_fraction)
    o = np.empty((n, 3), np.float32)
    o[:nc] = camera
    o[nc:] = lo + (hi - lo) * rng.random((n - nc, 3), dtype=np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d[:nc, 2] = -np.abs(d[:nc, 2]) - 1.0
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return np.concatenate([o, d], axis=1).astype(np.float32)


# A small room in the reference scene-JSON schema (comments, trailing commas and
# a bare key included): 6 planes, an emissive quad and a rotated box.
JSON_ROOM = """
// a small room in the reference schema (comments, trailing commas and a bare key)
{
  "mainCamera": { "location": [0, 0.5, 6], "angle": [-5, 0, 0], "fieldOfView": 60, exposure: 1.5, },
  "_materials": { "wall": { "color": "#ccbbaa", "diffuse": 0.9 } },
  "room": {
    "lamp": { "location": [0, 2.9, 0], "angle": [180, 0, 0], "scale": [1, 1, 1],
              "mesh": { "type": "plane" }, "mat": { "color": "#fffff0", "emission": 8 } },
    "floor": { "location": [0, -3, 0], "scale": [6, 1, 6], "mesh": { "type": "plane" }, "mat": "wall" },
    "ceiling": { "location": [0, 3, 0], "angle": [180, 0, 0], "scale": [6, 1, 6], "mesh": { "type": "plane" }, "mat": "wall" },
    "left": { "location": [-3, 0, 0], "angle": [0, 0, -90], "scale": [6, 1, 6], "mesh": { "type": "plane" },
              "mat": { "color": "#ff5555" } },
    "right": { "location": [3, 0, 0], "angle": [0, 0, 90], "scale": [6, 1, 6], "mesh": { "type": "plane" },
               "mat": { "color": [0.3, 1.0, 0.3] } },
    "back": { "location": [0, 0, -3], "angle": [90, 0, 0], "scale": [6, 1, 6], "mesh": { "type": "plane" }, "mat": "wall" },
    "box": { "location": [1.2, -2, -0.5], "angle": [0, -30, 0], "scale": [1.6, 2, 1.6], "mesh": { "type": "cube" },
             "mat": { "color": "#ffffff", "glossy": 0.3, "roughness": 0.2 } },
  },
}
"""


# ---------------------------------------------------------------- image files
def rgbe_encode(img):
    """H x W x 3 float -> H x W x 4 uint8 RGBE (mantissa scaled by frexp)."""
    img = np.asarray(img, np.float64)
    m = img.max(axis=2)
    mant, e = np.frexp(m)
    ok = m > 1e-32
    scale = np.where(ok, mant * 256.0 / np.where(ok, m, 1.0), 0.0)
    rgb = np.floor(img * scale[..., None]).clip(0, 255)
    E = np.where(ok, e + 128, 0)
    return np.concatenate([rgb, E[..., None]], axis=2).astype(np.uint8)


def rgbe_decode(q):
    """Radiance decoding: channel * 2^(E - 136), black when E == 0."""
    q = np.asarray(q)
    sc = np.where(q[..., 3] == 0, 0.0, np.ldexp(1.0, q[..., 3].astype(np.int32) - 136))
    return (q[..., :3] * sc[..., None]).astype(np.float32)


def write_hdr(path, img, rle=True):
    """Radiance .hdr writer: adaptive-RLE scanlines (runs of >= 4 equal bytes, else literals) or flat."""
    q = rgbe_encode(img)
    H, W = q.shape[:2]
    out = bytearray(b"#?RADIANCE\n# test image\nFORMAT=32-bit_rle_rgbe\n\n" + f"-Y {H} +X {W}\n".encode())
    for y in range(H):
        if not rle:
            out += q[y].tobytes()
            continue
        out += bytes([2, 2, W >> 8, W & 255])
        for ch in range(4):
            row = [int(v) for v in q[y, :, ch]]
            x = 0
            while x < W:
                run = 1
                while x + run < W and run < 127 and row[x + run] == row[x]:
                    run += 1
                if run >= 4:
                    out += bytes([128 + run, row[x]])
                    x += run
                    continue
                lit = []
                while x < W and len(lit) < 128:
                    r = 1
                    while x + r < W and r < 127 and row[x + r] == row[x]:
                        r += 1
                    if r >= 4:
                        break
                    lit.append(row[x])
                    x += 1
                out += bytes([len(lit)]) + bytes(lit)
    with open(path, "wb") as f:
        f.write(bytes(out))
    return rgbe_decode(q)


def write_pfm(path, img):
    """Little-endian RGB PFM, rows bottom to top."""
    img = np.asarray(img, np.float32)
    H, W = img.shape[:2]
    with open(path, "wb") as f:
        f.write(f"PF\n{W} {H}\n-1.0\n".encode())
        f.write(np.ascontiguousarray(img[::-1]).astype("<f4").tobytes())


def sky_image(W=64, H=32, sun=(0.62, 0.27), sun_radius=0.03, sun_level=80.0, seed=0):
    """Synthetic lat-long sky: blue gradient above, brown ground below, a bright sun disc."""
    rng = np.random.default_rng(seed)
    v = (np.arange(H) + 0.5) / H
    u = (np.arange(W) + 0.5) / W
    U, V = np.meshgrid(u, v)
    img = np.zeros((H, W, 3), np.float32)
    up = V < 0.5
    t = (0.5 - V) * 2
    img[up] = np.stack([0.35 + 0.2 * t, 0.5 + 0.2 * t, 0.9 + 0.1 * t], axis=-1)[up]
    img[~up] = [0.25, 0.2, 0.15]
    d = np.hypot((U - sun[0]) * 2, V - sun[1])
    img[d < sun_radius] = sun_level
    img *= (1.0 + 0.05 * rng.standard_normal((H, W, 1))).astype(np.float32)
    return np.maximum(img, 0).astype(np.float32)


# ---------------------------------------------------------------- GGX furnace
def ggx_directional_albedo(mu_o, ax, ay, n=1536):
    """White-furnace known answer: the directional albedo of the GGX lobe with
    Fresnel 1, E(v) = integral over the hemisphere of D(h) G1(v) G1(l) / (4 v.z)
    dw_l (Smith separable, bsdf.cpp:260-280), by midpoint quadrature in
    (cos theta_l, phi_l).  v lies in the x-z plane at cos theta = mu_o."""
    v = np.array([np.sqrt(max(0.0, 1.0 - mu_o * mu_o)), 0.0, mu_o])
    mu = (np.arange(n) + 0.5) / n
    phi = (np.arange(2 * n) + 0.5) / (2 * n) * 2 * np.pi
    M, P = np.meshgrid(mu, phi, indexing="ij")
    s = np.sqrt(1.0 - M * M)
    lx, ly, lz = s * np.cos(P), s * np.sin(P), M
    hx, hy, hz = lx + v[0], ly + v[1], lz + v[2]
    hn = np.sqrt(hx * hx + hy * hy + hz * hz)
    hx, hy, hz = hx / hn, hy / hn, hz / hn
    den = (hx / ax) ** 2 + (hy / ay) ** 2 + hz * hz
    D = 1.0 / (np.pi * ax * ay * den * den)

    def g1(wx, wy, wz):
        lam = 0.5 * (np.sqrt(1.0 + ((ax * wx) ** 2 + (ay * wy) ** 2) / (wz * wz)) - 1.0)
        return 1.0 / (1.0 + lam)

    f = D * g1(v[0], v[1], v[2]) * g1(lx, ly, lz) / (4.0 * v[2])
    f[hz <= 0] = 0.0
    return float(f.sum() * (1.0 / n) * (2 * np.pi / (2 * n)))


def furnace_scene(rg, roughness, anisotropy=0.0, tilt_deg=0.0):
    """A white GGX metal quad (F0 = 1) filling a narrow camera's view inside a
    constant environment of radiance 1: the image mean is the lobe's
    directional albedo at cos(tilt)."""
    p, nrm = quad_z(-5.0, 1.5, +1)
    if tilt_deg:
        c, s_ = math.cos(math.radians(tilt_deg)), math.sin(math.radians(tilt_deg))
        R = np.array([[1, 0, 0], [0, c, -s_], [0, s_, c]], np.float32)
        centre = np.array([0, 0, -5.0], np.float32)
        p = ((p.reshape(-1, 3) - centre) @ R.T + centre).reshape(-1, 9).astype(np.float32)
        nrm = (nrm.reshape(-1, 3) @ R.T).reshape(-1, 9).astype(np.float32)
    m = material(rg, (1, 1, 1), glossy=1.0, roughness=roughness, metallic=1.0)
    m.anisotropy = anisotropy
    env = np.ones((8, 16, 4), np.float32)
    o = rg.rg_object()
    o.material = 0
    o.interior_medium = -1
    return rg.Scene.from_arrays(p, nrm, [0, 0], [0], [o], [m], camera(rg, fov=6.0), textures=[(env, True)], envmap=0)


FURNACE_CASES = [(0.5, 0.0, 0.0), (0.8, 0.0, 0.0), (0.7, 0.6, 0.0), (0.6, 0.0, 60.0)]


def furnace_expected(roughness, anisotropy, tilt_deg):
    r2 = roughness * roughness
    a = max(-0.99, min(0.99, anisotropy))
    ax, ay = max(1e-3, r2 * (1 - a)), max(1e-3, r2 * (1 + a))
    return ggx_directional_albedo(math.cos(math.radians(tilt_deg)), ax, ay)
