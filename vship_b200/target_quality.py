"""Target-quality search with the learned SSIMULACRA2 surrogate.

A target-quality encoder looks, per frame, for the coarsest quantisation whose SSIMULACRA2
stays at or above a target (80 here).  Bisection over the quantisation step needs one score
per probe; most probes land far from the target, where only the side of the threshold
matters.  `search` consults the surrogate for every probe (the reference's coarse levels
prepared once per frame, VshipExt_SurrogateReferences, then VshipExt_SurrogatePredictAgainst
per probe) and calls the exact metric only when the prediction is within `margin` of the
target; the exact metric also judges the surrogate's error on those probes.
`search(..., surrogate=None)` is the method without it (every probe exact).

Frames come from `GpuFrames`, the generator of vship_b200.synth moved to the GPU with torch
(seeded sums of random sinusoids plus noise; the distortion is 8x8 block-DCT quantisation
with a given step; 10-bit limited-range BT.709 Y'CbCr 4:2:0 output), so that training sets of
hundreds of thousands of pairs and searches over 1080p frames are not bound by the host.
"""
import math

import numpy as np

from . import abi


class GpuFrames:
    """Seeded synthetic frames on the GPU (float32 R'G'B' in [0, 255], shape [n, 3, h, w])."""

    def __init__(self, device="cuda"):
        import torch
        self.torch = torch
        self.device = device
        k = np.arange(8)[:, None]
        n = np.arange(8)[None, :]
        m = np.sqrt(2.0 / 8) * np.cos(np.pi * (2 * n + 1) * k / 16)
        m[0, :] = np.sqrt(1.0 / 8)
        self.D = torch.tensor(m, dtype=torch.float32, device=device)

    def _spectra(self, rng, n, w, h, count):
        """n random spectra of `count` sinusoids (periods 4-512 px) on the rfft2 grid."""
        torch = self.torch
        period = np.exp(rng.uniform(np.log(4.0), np.log(512.0), size=(n, count)))
        theta = rng.uniform(0, np.pi, size=(n, count))
        u = np.round(w * np.cos(theta) / period).astype(np.int64)
        v = np.round(h * np.sin(theta) / period).astype(np.int64)
        neg = u < 0
        u[neg], v[neg] = -u[neg], -v[neg]
        u = np.minimum(u, w // 2)
        v %= h
        amp = rng.uniform(2.0, 14.0, size=(n, count))
        phase = rng.uniform(0, 2 * np.pi, size=(n, count))
        keep = ~((u == 0) & (v == 0))
        scale = (w * h) / np.where((u > 0) & (u < w / 2), 2.0, 1.0)
        val = amp * np.exp(1j * phase) * scale * keep
        spec = torch.zeros((n, h, w // 2 + 1), dtype=torch.complex64, device=self.device)
        idx = torch.tensor((np.arange(n)[:, None] * h * (w // 2 + 1) + v * (w // 2 + 1) + u).reshape(-1),
                           device=self.device)
        spec.view(-1).index_add_(0, idx, torch.tensor(val.reshape(-1), dtype=torch.complex64, device=self.device))
        return spec

    def references(self, n, w, h, seed):
        torch = self.torch
        rng = np.random.default_rng(seed)
        base = torch.fft.irfft2(self._spectra(rng, n, w, h, 32), s=(h, w))
        img = torch.empty((n, 3, h, w), dtype=torch.float32, device=self.device)
        for c in range(3):
            img[:, c] = 128.0 + 0.7 * base + 0.5 * torch.fft.irfft2(self._spectra(rng, n, w, h, 16), s=(h, w))
        g = torch.Generator(device=self.device)
        g.manual_seed(int(seed) & 0x7FFFFFFF)
        img += 3.0 * torch.randn(img.shape, generator=g, device=self.device)
        return img.clamp_(0.0, 255.0)

    def dct_quantize(self, img, steps):
        """8x8 block-DCT quantisation of every channel with a per-frame step (edges replicated)."""
        torch = self.torch
        n, c, h, w = img.shape
        H8, W8 = (h + 7) // 8 * 8, (w + 7) // 8 * 8
        x = torch.nn.functional.pad(img, (0, W8 - w, 0, H8 - h), mode="replicate")
        b = x.reshape(n, c, H8 // 8, 8, W8 // 8, 8).permute(0, 1, 2, 4, 3, 5)
        coef = self.D @ b @ self.D.T
        s = torch.as_tensor(np.asarray(steps, dtype=np.float32), device=self.device).reshape(n, 1, 1, 1, 1, 1)
        coef = torch.round(coef / s) * s
        rec = (self.D.T @ coef @ self.D).permute(0, 1, 2, 4, 3, 5).reshape(n, c, H8, W8)
        return rec[:, :, :h, :w].clamp(0.0, 255.0)

    def yuv420p10(self, img):
        """-> (Y [n, h, w], U [n, hc, wc], V) int16 tensors (10-bit limited BT.709, 2x2 chroma box)."""
        torch = self.torch
        r, g, b = img[:, 0] / 255.0, img[:, 1] / 255.0, img[:, 2] / 255.0
        y = 0.2126 * r + 0.7152 * g + 0.0722 * b
        cb = (b - y) / 1.8556
        cr = (r - y) / 1.5748
        n, h, w = y.shape
        hc, wc = (h + 1) // 2, (w + 1) // 2

        def down(p):
            pp = torch.nn.functional.pad(p[:, None], (0, 2 * wc - w, 0, 2 * hc - h), mode="replicate")[:, 0]
            return 0.25 * (pp[:, 0::2, 0::2] + pp[:, 1::2, 0::2] + pp[:, 0::2, 1::2] + pp[:, 1::2, 1::2])

        Y = torch.round((219.0 * y + 16.0) * 4.0).clamp(0, 1023).to(torch.int16)
        U = torch.round((224.0 * down(cb) + 128.0) * 4.0).clamp(0, 1023).to(torch.int16)
        V = torch.round((224.0 * down(cr) + 128.0) * 4.0).clamp(0, 1023).to(torch.int16)
        return Y.contiguous(), U.contiguous(), V.contiguous()


def planes_of(yuv):
    """Per-frame device plane addresses (3 per frame) and the line sizes of a yuv420p10 batch."""
    Y, U, V = yuv
    n, h, w = Y.shape
    wc = U.shape[2]
    ptrs = []
    for i in range(n):
        ptrs += [Y[i].data_ptr(), U[i].data_ptr(), V[i].data_ptr()]
    return ptrs, [2 * w, 2 * wc, 2 * wc]


def build_training_set(surrogate, exact, n, w, h, seed=1, chunk=512, steps=(2.0, 64.0), refs_per_chunk=64):
    """n pairs of w x h frames (steps uniform in `steps`): network inputs (device FP16
    [n, elems]) and exact scores (device float32 [n])."""
    import torch
    gen = GpuFrames()
    inputs = torch.empty((n, surrogate.input_elems()), dtype=torch.float16, device="cuda")
    targets = torch.empty(n, dtype=torch.float32, device="cuda")
    scores = torch.empty(chunk, dtype=torch.float64, device="cuda")
    rng = np.random.default_rng(seed)
    for start in range(0, n, chunk):
        k = min(chunk, n - start)
        refs = gen.references(refs_per_chunk, w, h, seed=int(rng.integers(1 << 31)))
        ref = refs[torch.arange(k, device="cuda") % refs_per_chunk]
        st = rng.uniform(steps[0], steps[1], size=k)
        dist = gen.dct_quantize(ref, st)
        a, b = gen.yuv420p10(ref), gen.yuv420p10(dist)
        p1, ls = planes_of(a)
        p2, _ = planes_of(b)
        surrogate.inputs(k, p1, p2, ls, ls, inputs[start].data_ptr())
        exact.compute_device(k, p1, p2, ls, ls, scores.data_ptr(), 0, 0)
        targets[start:start + k] = scores[:k].float()
        torch.cuda.synchronize()
    return inputs, targets


def search(frames_yuv_fn, distort_fn, nframes, exact, surrogate=None, target=80.0, margin=2.0, lo=2.0, hi=64.0,
           iters=7, batch=32):
    """Bisection per frame for the largest step in [lo, hi] whose score is at least `target`.

    frames_yuv_fn(i0, i1) -> the reference yuv420p10 batch of frames i0..i1-1;
    distort_fn(i0, i1, steps) -> the distorted yuv420p10 batch at those steps.
    Returns dict(step=np.array, exact_calls=int, probes=int, surrogate_errors=list of
    |prediction - exact| on the probes scored both ways)."""
    import torch
    lo_s = np.full(nframes, lo)
    hi_s = np.full(nframes, hi)
    exact_calls, probes, errors = 0, 0, []
    pred = torch.empty(batch, dtype=torch.float32, device="cuda")
    ex = torch.empty(batch, dtype=torch.float64, device="cuda")
    refs = None
    if surrogate is not None:
        # Every probe of a frame shares its reference: its coarse levels are computed once.
        refs = torch.empty((nframes, surrogate.reference_floats()), dtype=torch.float32, device="cuda")
        for i0 in range(0, nframes, batch):
            i1 = min(nframes, i0 + batch)
            p1, ls = planes_of(frames_yuv_fn(i0, i1))
            surrogate.references(i1 - i0, p1, ls, refs[i0].data_ptr())
    for _ in range(iters):
        mid = 0.5 * (lo_s + hi_s)
        for i0 in range(0, nframes, batch):
            i1 = min(nframes, i0 + batch)
            k = i1 - i0
            a = frames_yuv_fn(i0, i1)
            b = distort_fn(i0, i1, mid[i0:i1])
            p1, ls = planes_of(a)
            p2, _ = planes_of(b)
            probes += k
            if surrogate is not None:
                surrogate.predict_against(k, refs[i0].data_ptr(), p2, ls, pred.data_ptr())
                score = pred[:k].double().cpu().numpy()
                near = np.abs(score - target) <= margin
            else:
                score = np.zeros(k)
                near = np.ones(k, dtype=bool)
            idx = np.nonzero(near)[0]
            if len(idx):
                q1 = [p1[3 * j + c] for j in idx for c in range(3)]
                q2 = [p2[3 * j + c] for j in idx for c in range(3)]
                exact.compute_device(len(idx), q1, q2, ls, ls, ex.data_ptr(), 0, 0)
                e = ex[:len(idx)].cpu().numpy()
                if surrogate is not None:
                    errors += list(np.abs(score[idx] - e))
                score[idx] = e
                exact_calls += len(idx)
            ok = score >= target
            lo_s[i0:i1] = np.where(ok, mid[i0:i1], lo_s[i0:i1])
            hi_s[i0:i1] = np.where(ok, hi_s[i0:i1], mid[i0:i1])
    return {"step": lo_s, "exact_calls": exact_calls, "probes": probes, "surrogate_errors": errors}


def final_scores(frames_yuv_fn, distort_fn, nframes, exact, steps, batch=32):
    """Exact scores of every frame at the given steps."""
    import torch
    out = np.zeros(nframes)
    ex = torch.empty(batch, dtype=torch.float64, device="cuda")
    for i0 in range(0, nframes, batch):
        i1 = min(nframes, i0 + batch)
        a = frames_yuv_fn(i0, i1)
        b = distort_fn(i0, i1, steps[i0:i1])
        p1, ls = planes_of(a)
        p2, _ = planes_of(b)
        exact.compute_device(i1 - i0, p1, p2, ls, ls, ex.data_ptr(), 0, 0)
        out[i0:i1] = ex[:i1 - i0].cpu().numpy()
    return out


def colorspace(w, h):
    return abi.yuv420_10bit_bt709(w, h)


def rmse(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(math.sqrt(np.mean((a - b) ** 2))) if len(a) else float("nan")
