"""Test-side image encoders (numpy) for the decoder tests: a PNG writer (RFC
2083: every colour type and bit depth, the five row filters, Adam7) and a
baseline JPEG encoder (ITU-T T.81: one or three components, any sampling
factors, restart intervals, Huffman tables built from the image's own symbol
counts), plus the reconstruction a conforming decoder must produce from the
JPEG's quantised coefficients."""
import heapq
import math
import struct
import zlib

import numpy as np

# ---------------------------------------------------------------- PNG
ADAM7 = [(0, 0, 8, 8), (4, 0, 8, 8), (0, 4, 4, 8), (2, 0, 4, 4), (0, 2, 2, 4), (1, 0, 2, 2), (0, 1, 1, 2)]


def _chunk(kind, data):
    c = kind + data
    return struct.pack(">I", len(data)) + c + struct.pack(">I", zlib.crc32(c) & 0xFFFFFFFF)


def _paeth(a, b, c):
    p = a + b - c
    pa, pb, pc = abs(p - a), abs(p - b), abs(p - c)
    return a if (pa <= pb and pa <= pc) else (b if pb <= pc else c)


def _pack_row(samples, depth):
    if depth == 8:
        return bytes(int(v) for v in samples)
    if depth == 16:
        return b"".join(struct.pack(">H", int(v)) for v in samples)
    per = 8 // depth
    out = bytearray()
    for i in range(0, len(samples), per):
        byte = 0
        for k in range(per):
            v = int(samples[i + k]) if i + k < len(samples) else 0
            byte |= v << ((per - 1 - k) * depth)
        out.append(byte)
    return bytes(out)


def _filter_rows(rows, bpp, seed):
    rng = np.random.default_rng(seed)
    out, prev = bytearray(), None
    for r in rows:
        ft = int(rng.integers(0, 5))
        f = bytearray()
        for i, x in enumerate(r):
            a = r[i - bpp] if i >= bpp else 0
            b = prev[i] if prev is not None else 0
            c = prev[i - bpp] if (prev is not None and i >= bpp) else 0
            pred = [0, a, b, (a + b) >> 1, _paeth(a, b, c)][ft]
            f.append((x - pred) & 0xFF)
        out.append(ft)
        out += f
        prev = r
    return bytes(out)


def write_png(path, samples, color_type, depth, palette=None, trns=None, interlace=False, seed=0):
    """samples: H x W x C integer array (C = channels of the colour type; palette indices for type 3)."""
    H, W = samples.shape[:2]
    chans = {0: 1, 2: 3, 3: 1, 4: 2, 6: 4}[color_type]
    bpp = max(1, chans * depth // 8)
    raw = b""
    passes = ADAM7 if interlace else [(0, 0, 1, 1)]
    for k, (x0, y0, dx, dy) in enumerate(passes):
        sub = samples[y0::dy, x0::dx]
        if sub.shape[0] == 0 or sub.shape[1] == 0:
            continue
        rows = [_pack_row(sub[y].reshape(-1), depth) for y in range(sub.shape[0])]
        raw += _filter_rows(rows, bpp, seed + k)
    png = b"\x89PNG\r\n\x1a\n" + _chunk(b"IHDR", struct.pack(">IIBBBBB", W, H, depth, color_type, 0, 0, int(interlace)))
    if palette is not None:
        png += _chunk(b"PLTE", bytes(np.asarray(palette, np.uint8).reshape(-1)))
    if trns is not None:
        png += _chunk(b"tRNS", bytes(np.asarray(trns, np.uint8).reshape(-1)))
    png += _chunk(b"IDAT", zlib.compress(raw, 6)) + _chunk(b"IEND", b"")
    with open(path, "wb") as f:
        f.write(png)


# ---------------------------------------------------------------- JPEG
ZIGZAG = np.array([0, 1, 8, 16, 9, 2, 3, 10, 17, 24, 32, 25, 18, 11, 4, 5, 12, 19, 26, 33, 40, 48, 41, 34, 27, 20, 13,
                   6, 7, 14, 21, 28, 35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23, 30, 37, 44, 51, 58, 59, 52, 45,
                   38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63])
_C = np.array([[(math.sqrt(0.5) if u == 0 else 1.0) * 0.5 * math.cos((2 * x + 1) * u * math.pi / 16) for u in range(8)]
               for x in range(8)])  # _C[x, u]


def fdct(block):
    return _C.T @ (block - 128.0) @ _C  # F[v, u]


def idct(F):
    return _C @ F @ _C.T + 128.0


def _bits_needed(v):
    return 0 if v == 0 else int(abs(v)).bit_length()


def _huff_table(freq):
    """Code lengths (<= 16) from symbol counts; a reserved dummy symbol keeps the all-ones code unused."""
    items = [(f, i, [s]) for i, (s, f) in enumerate(sorted(freq.items()))] + [(0, -1, [256])]
    length = {s: 0 for s in list(freq) + [256]}
    if len(items) == 1:
        return {}
    heap = [(f, k, syms) for f, k, syms in items]
    heapq.heapify(heap)
    cnt = len(heap)
    while len(heap) > 1:
        f1, _, a = heapq.heappop(heap)
        f2, _, b = heapq.heappop(heap)
        for s in a + b:
            length[s] += 1
        cnt += 1
        heapq.heappush(heap, (f1 + f2, cnt, a + b))
    if max(length.values()) > 16:  # fall back to equal lengths
        L = max(1, math.ceil(math.log2(len(length) + 1)))
        length = {s: L for s in length}
    order = sorted(length, key=lambda s: (length[s], s == 256, s))  # the dummy is the last (all-ones) code
    code, prev, codes = 0, 0, {}
    for s in order:
        code <<= length[s] - prev
        prev = length[s]
        codes[s] = (code, length[s])
        code += 1
    codes.pop(256)
    return codes


def _dht(tc, th, codes):
    counts = [0] * 16
    syms = sorted(codes, key=lambda s: (codes[s][1], codes[s][0]))
    for s in syms:
        counts[codes[s][1] - 1] += 1
    body = bytes([(tc << 4) | th]) + bytes(counts) + bytes(syms)
    return b"\xff\xc4" + struct.pack(">H", len(body) + 2) + body


class _BitWriter:
    def __init__(self):
        self.out, self.acc, self.n = bytearray(), 0, 0

    def put(self, v, nbits):
        for k in range(nbits - 1, -1, -1):
            self.acc = (self.acc << 1) | ((v >> k) & 1)
            self.n += 1
            if self.n == 8:
                self.out.append(self.acc)
                if self.acc == 0xFF:
                    self.out.append(0)
                self.acc, self.n = 0, 0

    def pad(self):
        while self.n:
            self.put(1, 1)


def encode_jpeg(path, rgb, sampling=((2, 2), (1, 1), (1, 1)), qscale=1.0, restart=0, grey=False):
    """Baseline JPEG of an H x W x 3 uint8 image (grey: H x W).  Returns the image a
    conforming decoder reconstructs (before upsampling and colour conversion:
    the per-component sample planes) and the component geometry."""
    img = np.asarray(rgb, np.float64)
    H, W = img.shape[:2]
    if grey:
        planes = [img]
        sampling = ((1, 1),)
    else:
        R, G, B = img[..., 0], img[..., 1], img[..., 2]
        planes = [0.299 * R + 0.587 * G + 0.114 * B, -0.168736 * R - 0.331264 * G + 0.5 * B + 128,
                  0.5 * R - 0.418688 * G - 0.081312 * B + 128]
    hmax, vmax = max(h for h, v in sampling), max(v for h, v in sampling)
    mcux, mcuy = -(-W // (8 * hmax)), -(-H // (8 * vmax))
    q_base = np.clip(np.round((1 + np.arange(64)[ZIGZAG.argsort()] * 0.7) * qscale), 1, 255)  # natural order
    comps = []
    for ci, (plane, (h, v)) in enumerate(zip(planes, sampling)):
        pw, ph = mcux * 8 * hmax, mcuy * 8 * vmax
        padded = np.pad(plane, ((0, ph - H), (0, pw - W)), mode="edge")
        sx, sy = hmax // h, vmax // v
        sub = padded.reshape(ph // sy, sy, pw // sx, sx).mean(axis=(1, 3))
        sub = np.clip(np.round(sub), 0, 255)
        q = q_base if ci == 0 else np.clip(np.round(q_base * 1.5), 1, 255)
        bw, bh = mcux * h, mcuy * v
        coefs = np.zeros((bh, bw, 8, 8), np.int64)
        recon = np.zeros((bh * 8, bw * 8))
        for by in range(bh):
            for bx in range(bw):
                F = fdct(sub[by * 8:by * 8 + 8, bx * 8:bx * 8 + 8])
                qc = np.round(F / q.reshape(8, 8)).astype(np.int64)
                coefs[by, bx] = qc
                recon[by * 8:by * 8 + 8, bx * 8:bx * 8 + 8] = np.clip(np.floor(idct(qc * q.reshape(8, 8)) + 0.5), 0, 255)
        comps.append(dict(h=h, v=v, q=q, coefs=coefs, recon=recon, w=-(-W * h // hmax), ht=-(-H * v // vmax)))
    # MCU order and symbols
    order = []
    for my in range(mcuy):
        for mx in range(mcux):
            blocks = []
            for ci, c in enumerate(comps):
                for yy in range(c["v"]):
                    for xx in range(c["h"]):
                        blocks.append((ci, my * c["v"] + yy, mx * c["h"] + xx))
            order.append(blocks)
    if len(comps) == 1:  # non-interleaved: the component's own block grid
        c = comps[0]
        order = [[(0, by, bx)] for by in range(-(-c["ht"] // 8)) for bx in range(-(-c["w"] // 8))]

    def symbols():
        pred = [0] * len(comps)
        for m, blocks in enumerate(order):
            if restart and m > 0 and m % restart == 0:
                pred = [0] * len(comps)
                yield ("rst", (m // restart - 1) % 8)
            for ci, by, bx in blocks:
                zz = comps[ci]["coefs"][by, bx].reshape(-1)[ZIGZAG]
                d = int(zz[0]) - pred[ci]
                pred[ci] = int(zz[0])
                yield ("dc", ci, _bits_needed(d), d)
                run = 0
                last = max([k for k in range(1, 64) if zz[k] != 0], default=0)
                for k in range(1, last + 1):
                    if zz[k] == 0:
                        run += 1
                        continue
                    while run > 15:
                        yield ("ac", ci, 0xF0, 0, 0)
                        run -= 16
                    s = _bits_needed(int(zz[k]))
                    yield ("ac", ci, (run << 4) | s, int(zz[k]), s)
                    run = 0
                if last < 63:
                    yield ("ac", ci, 0x00, 0, 0)

    tab = lambda ci: 0 if ci == 0 else 1
    fdc, fac = [{}, {}], [{}, {}]
    for e in symbols():
        if e[0] == "dc":
            fdc[tab(e[1])][e[2]] = fdc[tab(e[1])].get(e[2], 0) + 1
        elif e[0] == "ac":
            fac[tab(e[1])][e[2]] = fac[tab(e[1])].get(e[2], 0) + 1
    ntab = 1 if len(comps) == 1 else 2
    hdc = [_huff_table(fdc[t]) for t in range(ntab)]
    hac = [_huff_table(fac[t]) for t in range(ntab)]
    bw_ = _BitWriter()
    for e in symbols():
        if e[0] == "rst":
            bw_.pad()
            bw_.out += bytes([0xFF, 0xD0 + e[1]])
            continue
        if e[0] == "dc":
            code, n = hdc[tab(e[1])][e[2]]
            bw_.put(code, n)
            if e[2]:
                d = e[3]
                bw_.put(d if d > 0 else d + (1 << e[2]) - 1, e[2])
        else:
            code, n = hac[tab(e[1])][e[2]]
            bw_.put(code, n)
            if e[4]:
                v = e[3]
                bw_.put(v if v > 0 else v + (1 << e[4]) - 1, e[4])
    bw_.pad()
    out = b"\xff\xd8" + b"\xff\xe0" + struct.pack(">H", 16) + b"JFIF\x00\x01\x01\x00\x00\x01\x00\x01\x00\x00"
    for t in range(ntab):
        qn = comps[min(t, len(comps) - 1)]["q"][ZIGZAG].astype(np.uint8)
        out += b"\xff\xdb" + struct.pack(">H", 67) + bytes([t]) + bytes(qn)
    sof = struct.pack(">BHHB", 8, H, W, len(comps))
    for ci, c in enumerate(comps):
        sof += bytes([ci + 1, (c["h"] << 4) | c["v"], tab(ci)])
    out += b"\xff\xc0" + struct.pack(">H", len(sof) + 2) + sof
    for t in range(ntab):
        out += _dht(0, t, hdc[t]) + _dht(1, t, hac[t])
    if restart:
        out += b"\xff\xdd" + struct.pack(">HH", 4, restart)
    sos = bytes([len(comps)]) + b"".join(bytes([ci + 1, (tab(ci) << 4) | tab(ci)]) for ci in range(len(comps)))
    sos += bytes([0, 63, 0])
    out += b"\xff\xda" + struct.pack(">H", len(sos) + 2) + sos + bytes(bw_.out) + b"\xff\xd9"
    with open(path, "wb") as f:
        f.write(out)
    return comps, (W, H, hmax, vmax)


def jpeg_expected(comps, geom, grey=False):
    """Full-resolution RGB in [0, 1] from the component planes: linear
    interpolation between chroma sample centres, JFIF YCbCr -> RGB."""
    W, H, hmax, vmax = geom
    ys, xs = np.mgrid[0:H, 0:W]

    def up(c):
        if c["h"] == hmax and c["v"] == vmax:
            return c["recon"][:H, :W]
        sx = (xs + 0.5) * c["h"] / hmax - 0.5
        sy = (ys + 0.5) * c["v"] / vmax - 0.5
        x0, y0 = np.floor(sx).astype(int), np.floor(sy).astype(int)
        fx, fy = sx - x0, sy - y0
        at = lambda xx, yy: c["recon"][np.clip(yy, 0, c["ht"] - 1), np.clip(xx, 0, c["w"] - 1)]
        return (at(x0, y0) * (1 - fx) + at(x0 + 1, y0) * fx) * (1 - fy) + (at(x0, y0 + 1) * (1 - fx) + at(x0 + 1, y0 + 1) * fx) * fy

    to8 = lambda v: np.clip(np.floor(v + 0.5), 0, 255) / 255.0
    if grey:
        g = to8(up(comps[0]))
        return np.stack([g, g, g], axis=-1)
    Y, cb, cr = up(comps[0]), up(comps[1]) - 128, up(comps[2]) - 128
    return np.stack([to8(Y + 1.402 * cr), to8(Y - 0.344136 * cb - 0.714136 * cr), to8(Y + 1.772 * cb)], axis=-1)
