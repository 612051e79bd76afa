"""Seeded synthetic frame pairs for the benchmark workloads and tests.

No public clip is used: reference frames are sums of 32 random 2-D sinusoids (periods 4 to
512 px, random orientation, phase and amplitude) plus N(0, 3) noise, clamped to 0-255;
distorted frames are the reference after 8x8 block-DCT quantisation (and, for the
Butteraugli workload, a Gaussian blur).  Frames are emitted as 8-bit full-range RGB planes or
as 10-bit limited-range BT.709 Y'CbCr 4:2:0 planes (16-bit little-endian words).

The sinusoids are placed on the FFT grid so one inverse real FFT per channel builds a frame.
"""
import numpy as np

_DCT8 = None


def _dct_matrix():
    global _DCT8
    if _DCT8 is None:
        k = np.arange(8)[:, None]
        n = np.arange(8)[None, :]
        m = np.sqrt(2.0 / 8) * np.cos(np.pi * (2 * n + 1) * k / 16)
        m[0, :] = np.sqrt(1.0 / 8)
        _DCT8 = m.astype(np.float64)
    return _DCT8


def sinusoid_field(rng, w, h, count=32, pmin=4.0, pmax=512.0):
    """One channel: sum of `count` sinusoids (float64, zero mean) built with irfft2."""
    spec = np.zeros((h, w // 2 + 1), dtype=np.complex128)
    for _ in range(count):
        period = np.exp(rng.uniform(np.log(pmin), np.log(pmax)))
        theta = rng.uniform(0, np.pi)
        u = int(round(w * np.cos(theta) / period))
        v = int(round(h * np.sin(theta) / period))
        if u < 0:
            u, v = -u, -v
        u = min(u, w // 2)
        v %= h
        if u == 0 and v == 0:
            continue
        amp = rng.uniform(2.0, 14.0)
        phase = rng.uniform(0, 2 * np.pi)
        spec[v, u] += amp * np.exp(1j * phase) * (w * h) / (2.0 if 0 < u < w / 2 else 1.0)
    return np.fft.irfft2(spec, s=(h, w))


def reference_rgb(rng, w, h):
    """(3, h, w) float64 in [0, 255]."""
    img = np.empty((3, h, w))
    base = sinusoid_field(rng, w, h)
    for c in range(3):
        img[c] = 128.0 + 0.7 * base + 0.5 * sinusoid_field(rng, w, h, count=16)
    img += rng.normal(0.0, 3.0, size=img.shape)
    return np.clip(img, 0.0, 255.0)


def dct_quantize(img, step):
    """8x8 block DCT quantisation of each channel (edges padded by replication)."""
    c, h, w = img.shape
    H8, W8 = (h + 7) // 8 * 8, (w + 7) // 8 * 8
    pad = np.pad(img, ((0, 0), (0, H8 - h), (0, W8 - w)), mode="edge")
    blocks = pad.reshape(c, H8 // 8, 8, W8 // 8, 8)
    D = _dct_matrix()
    coef = np.einsum("ij,cajbk,lk->caibl", D, blocks, D, optimize=True)
    coef = np.round(coef / step) * step
    rec = np.einsum("ij,caibl,lk->cajbk", D, coef, D, optimize=True)
    return np.clip(rec.reshape(c, H8, W8)[:, :h, :w], 0.0, 255.0)


def gaussian_blur(img, sigma):
    if sigma <= 0.05:
        return img
    r = int(np.ceil(3 * sigma))
    x = np.arange(-r, r + 1)
    g = np.exp(-x * x / (2 * sigma * sigma))
    g /= g.sum()
    out = np.empty_like(img)
    for c in range(img.shape[0]):
        t = np.apply_along_axis(lambda v: np.convolve(np.pad(v, r, mode="edge"), g, mode="valid"), 1, img[c])
        out[c] = np.apply_along_axis(lambda v: np.convolve(np.pad(v, r, mode="edge"), g, mode="valid"), 0, t)
    return out


def to_rgb8(img):
    """-> three uint8 planes (h, w) and their line sizes."""
    q = np.clip(np.round(img), 0, 255).astype(np.uint8)
    planes = [np.ascontiguousarray(q[c]) for c in range(3)]
    return planes, [planes[0].shape[1]] * 3


def to_yuv420_10bit(img):
    """R'G'B' in [0,255] -> BT.709 Y'CbCr, 10-bit limited range, 4:2:0 (2x2 box on chroma)."""
    r, g, b = img[0] / 255.0, img[1] / 255.0, img[2] / 255.0
    y = 0.2126 * r + 0.7152 * g + 0.0722 * b
    cb = (b - y) / 1.8556
    cr = (r - y) / 1.5748
    h, w = y.shape
    hc, wc = (h + 1) // 2, (w + 1) // 2

    def down(p):
        pp = np.pad(p, ((0, 2 * hc - h), (0, 2 * wc - w)), mode="edge")
        return 0.25 * (pp[0::2, 0::2] + pp[1::2, 0::2] + pp[0::2, 1::2] + pp[1::2, 1::2])

    Y = np.clip(np.round((219.0 * y + 16.0) * 4.0), 0, 1023).astype(np.uint16)
    U = np.clip(np.round((224.0 * down(cb) + 128.0) * 4.0), 0, 1023).astype(np.uint16)
    V = np.clip(np.round((224.0 * down(cr) + 128.0) * 4.0), 0, 1023).astype(np.uint16)
    planes = [np.ascontiguousarray(Y), np.ascontiguousarray(U), np.ascontiguousarray(V)]
    return planes, [w * 2, wc * 2, wc * 2]


def make_pairs(n, w, h, fmt="rgb8", seed=0, unique=None, steps=(4.0, 48.0), blur=None):
    """n frame pairs [(planes_ref, planes_dist, line_sizes)].  `unique` reference contents are
    cycled (each pair still gets its own quantisation step); blur=(lo, hi) adds a Gaussian
    blur with sigma drawn from [lo, hi] to the distorted frame."""
    rng = np.random.default_rng(seed)
    unique = n if unique is None else max(1, min(unique, n))
    refs = [reference_rgb(rng, w, h) for _ in range(unique)]
    out = []
    for i in range(n):
        ref = refs[i % unique]
        step = rng.uniform(*steps) if isinstance(steps, tuple) else float(steps)
        dist = dct_quantize(ref, step)
        if blur is not None:
            dist = gaussian_blur(dist, rng.uniform(*blur))
        if fmt == "rgb8":
            p1, ls = to_rgb8(ref)
            p2, _ = to_rgb8(dist)
        elif fmt == "yuv420p10":
            p1, ls = to_yuv420_10bit(ref)
            p2, _ = to_yuv420_10bit(dist)
        else:
            raise ValueError(fmt)
        out.append((p1, p2, ls))
    return out


def with_padding(planes, line_sizes, extra, rng=None, garbage=True):
    """Copies planes into rows of line_sizes[i] + extra[i] bytes, filling the padding with
    random bytes (the stride-padding case of the reference's identity test)."""
    rng = rng or np.random.default_rng(1)
    out, ls = [], []
    for p, l, e in zip(planes, line_sizes, extra):
        raw = p.view(np.uint8).reshape(p.shape[0], -1)
        stride = l + e
        buf = rng.integers(0, 256, size=(p.shape[0], stride), dtype=np.uint8) if garbage else np.zeros((p.shape[0], stride), np.uint8)
        buf[:, :l] = raw
        out.append(np.ascontiguousarray(buf))
        ls.append(stride)
    return out, ls
