"""FP64 restatement of the learned SSIMULACRA2 surrogate network, for checking the CUDA
training kernels.  Test infrastructure only: never imported by the library.

The network (vship_b200/csrc/surrogate.cu) has no counterpart in the reference; this module
restates its definition independently of the CUDA code:

  input   per level (1/8 and 1/16 of the frame): 6 channels [a_X, a_Y, a_B, d_X, d_Y, d_B],
          a = reference XYB, d = distorted - reference, normalised as (x - shift[c]) * scale[c]
  conv1   3x3, 6 -> 16, zero padding, bias, ReLU
  conv2   3x3, 16 -> 16, zero padding, bias, ReLU
  conv3   1x1, 16 -> 8, bias, ReLU
  pool    per channel: mean(x) and (mean(x^4) + 1e-8)^(1/4); level 1/8 first -> 32 features
  head    y = bh + Wh . f;  predicted score = 70 + 20 y
  loss    mean over samples of (y - (target - 70) / 20)^2

Conv weights enter the forward and backward passes rounded to FP16 (as the CUDA kernels read
them); gradients are with respect to the parameters themselves.  The parameter vector is laid
out as W1[16][6][3][3], b1[16], W2[16][16][3][3], b2[16], W3[8][16], b3[8], Wh[32], bh.
"""
import numpy as np

CIN, C1, C2, C3 = 6, 16, 16, 8
FEAT = 2 * 2 * C3
SHIFT, SCALE = 70.0, 20.0
EPS = 1e-8

SHAPES = [("W1", (C1, CIN, 3, 3)), ("b1", (C1,)), ("W2", (C2, C1, 3, 3)), ("b2", (C2,)),
          ("W3", (C3, C2, 1, 1)), ("b3", (C3,)), ("Wh", (FEAT,)), ("bh", (1,))]
NPARAMS = sum(int(np.prod(s)) for _, s in SHAPES)


def unpack(vec):
    out, o = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = np.asarray(vec[o:o + n], dtype=np.float64).reshape(shape)
        o += n
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name], np.float64).reshape(-1) for name, _ in SHAPES])


def _fp16(w):
    return w.astype(np.float16).astype(np.float64)


def _conv(x, w, b):
    """x [N, Cin, H, W], w [Cout, Cin, k, k] -> pre-activation [N, Cout, H, W] (zero padding)."""
    k = w.shape[2]
    r = k // 2
    n, cin, h, wd = x.shape
    xp = np.zeros((n, cin, h + 2 * r, wd + 2 * r))
    xp[:, :, r:r + h, r:r + wd] = x
    out = np.zeros((n, w.shape[0], h, wd))
    for ky in range(k):
        for kx in range(k):
            out += np.einsum("nchw,oc->nohw", xp[:, :, ky:ky + h, kx:kx + wd], w[:, :, ky, kx])
    return out + b[None, :, None, None]


def _conv_backward(x, w, g):
    """Gradients of _conv for upstream g [N, Cout, H, W]: (dx, dw, db)."""
    k = w.shape[2]
    r = k // 2
    n, cin, h, wd = x.shape
    xp = np.zeros((n, cin, h + 2 * r, wd + 2 * r))
    xp[:, :, r:r + h, r:r + wd] = x
    dxp = np.zeros_like(xp)
    dw = np.zeros_like(w)
    for ky in range(k):
        for kx in range(k):
            dw[:, :, ky, kx] = np.einsum("nohw,nchw->oc", g, xp[:, :, ky:ky + h, kx:kx + wd])
            dxp[:, :, ky:ky + h, kx:kx + wd] += np.einsum("nohw,oc->nchw", g, w[:, :, ky, kx])
    return dxp[:, :, r:r + h, r:r + wd], dw, g.sum(axis=(0, 2, 3))


def _level_forward(x, p):
    z1 = _conv(x, _fp16(p["W1"]), p["b1"]); a1 = np.maximum(z1, 0)
    z2 = _conv(a1, _fp16(p["W2"]), p["b2"]); a2 = np.maximum(z2, 0)
    z3 = _conv(a2, _fp16(p["W3"]), p["b3"]); a3 = np.maximum(z3, 0)
    hw = x.shape[2] * x.shape[3]
    m1 = a3.sum(axis=(2, 3)) / hw
    m4 = (a3 ** 4).sum(axis=(2, 3)) / hw
    q = (m4 + EPS) ** 0.25
    return np.concatenate([m1, q], axis=1), (x, z1, a1, z2, a2, z3, a3, m4, hw)


def _level_backward(df, cache, p, grads):
    x, z1, a1, z2, a2, z3, a3, m4, hw = cache
    dm1, dq = df[:, :C3], df[:, C3:]
    k = (m4 + EPS) ** -0.75
    da3 = (dm1[:, :, None, None] + (dq * k)[:, :, None, None] * a3 ** 3) / hw
    g3 = da3 * (z3 > 0)
    da2, dw3, db3 = _conv_backward(a2, _fp16(p["W3"]), g3)
    g2 = da2 * (z2 > 0)
    da1, dw2, db2 = _conv_backward(a1, _fp16(p["W2"]), g2)
    g1 = da1 * (z1 > 0)
    _, dw1, db1 = _conv_backward(x, _fp16(p["W1"]), g1)
    for name, v in (("W1", dw1), ("b1", db1), ("W2", dw2), ("b2", db2), ("W3", dw3), ("b3", db3)):
        grads[name] += v


def normalise(level, norm):
    """level [N, 6, H, W] (values as stored, FP16), norm = shift[6] + scale[6]."""
    shift, scale = np.asarray(norm[:CIN], np.float64), np.asarray(norm[CIN:], np.float64)
    return (np.asarray(level, np.float64) - shift[None, :, None, None]) * scale[None, :, None, None]


def forward(params, norm, level3, level4):
    """Predicted scores of N samples (levels as [N, 6, H, W] arrays)."""
    p = unpack(params)
    f3, _ = _level_forward(normalise(level3, norm), p)
    f4, _ = _level_forward(normalise(level4, norm), p)
    f = np.concatenate([f3, f4], axis=1)
    return SHIFT + SCALE * (p["bh"][0] + f @ p["Wh"])


def loss_and_grad(params, norm, level3, level4, targets):
    """(loss, gradient vector) of the mean squared error on normalised scores."""
    p = unpack(params)
    f3, c3 = _level_forward(normalise(level3, norm), p)
    f4, c4 = _level_forward(normalise(level4, norm), p)
    f = np.concatenate([f3, f4], axis=1)
    y = p["bh"][0] + f @ p["Wh"]
    t = (np.asarray(targets, np.float64) - SHIFT) / SCALE
    n = len(t)
    e = y - t
    loss = float(np.mean(e * e))
    dy = 2 * e / n
    grads = {name: np.zeros(shape) for name, shape in SHAPES}
    grads["Wh"] = dy @ f
    grads["bh"] = np.array([dy.sum()])
    df = dy[:, None] * p["Wh"][None, :]
    _level_backward(df[:, :2 * C3], c3, p, grads)
    _level_backward(df[:, 2 * C3:], c4, p, grads)
    return loss, pack(grads)


def split_inputs(block, h3, w3, h4, w4):
    """[N, elems] FP16 input blocks -> (level3 [N, 6, h3, w3], level4 [N, 6, h4, w4])."""
    b = np.asarray(block)
    n3 = CIN * h3 * w3
    return (b[:, :n3].reshape(-1, CIN, h3, w3).astype(np.float64),
            b[:, n3:n3 + CIN * h4 * w4].reshape(-1, CIN, h4, w4).astype(np.float64))
