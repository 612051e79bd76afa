"""GPU checks of the learned surrogate (VshipExt_Surrogate*) and of what it buys.

* Gradients and loss of the CUDA training kernels against the FP64 oracle
  (oracle/surrogate.py) on random inputs and weights: FP16 conv weights on both sides and
  FP32 accumulation on the GPU, so the tolerance is FP32 rounding (2e-3 relative per
  parameter, 1e-5 on the loss).
* Predictions of the CUDA forward pass against the oracle's forward (1e-3 score units).
* The coarse inputs (XYB levels 1/8 and 1/16 from raw frames) against the FP64 oracle's
  pyramid levels, to FP16 storage rounding.
* End to end: a network trained on 16k seeded 512x512 pairs predicts held-out scores to a
  quarter of their spread, and a bisection to SSIMULACRA2 = 80 that consults it calls the
  exact metric at most 60 % as often as the same bisection without it, ending within 0.5 of
  the exact-only search's mean distance to the target.
"""
import numpy as np
import pytest

from oracle import surrogate as S
from vship_b200 import abi, api, synth, target_quality as tq

pytestmark = pytest.mark.gpu

W, H = 192, 160  # levels 1/8 and 1/16: 24 x 20 and 12 x 10


def _level_dims(w, h):
    dims = [(w, h)]
    for _ in range(4):
        pw, ph = dims[-1]
        dims.append(((pw - 1) // 2 + 1, (ph - 1) // 2 + 1))
    (w3, h3), (w4, h4) = dims[3], dims[4]
    return h3, w3, h4, w4


def _random_model(seed):
    rng = np.random.default_rng(seed)
    p = S.unpack(np.zeros(S.NPARAMS))
    p["W1"] = rng.normal(0, np.sqrt(2 / 54), p["W1"].shape)
    p["W2"] = rng.normal(0, np.sqrt(2 / 144), p["W2"].shape)
    p["W3"] = rng.normal(0, np.sqrt(2 / 16), p["W3"].shape)
    p["b1"] = rng.uniform(0.0, 0.2, 16)
    p["b2"] = rng.uniform(0.0, 0.2, 16)
    p["b3"] = rng.uniform(0.0, 0.2, 8)
    p["Wh"] = rng.normal(0, 0.3, 32)
    p["bh"] = np.array([0.1])
    params = S.pack(p).astype(np.float32).astype(np.float64)
    norm = np.concatenate([[0.42, 0.45, 0.55], [0.0, 0.0, 0.0], [20.0, 5.0, 8.0], [60.0, 80.0, 70.0]])
    return params, norm


def _random_inputs(n, seed):
    rng = np.random.default_rng(seed)
    h3, w3, h4, w4 = _level_dims(W, H)
    blocks = []
    for _ in range(n):
        parts = []
        for h, w in ((h3, w3), (h4, w4)):
            a = np.stack([rng.normal(0.42, 0.03, (h, w)), rng.uniform(0.05, 0.8, (h, w)), rng.normal(0.55, 0.08, (h, w))])
            d = rng.normal(0, 0.01, (3, h, w))
            parts.append(np.concatenate([a, d]).reshape(-1))
        blocks.append(np.concatenate(parts))
    return np.stack(blocks).astype(np.float16)


def test_gradients_match_oracle(gpu):
    import torch
    with api.Surrogate(abi.yuv420_10bit_bt709(W, H)) as sur:
        h3, w3, h4, w4 = _level_dims(W, H)
        assert sur.input_elems() == 6 * (h3 * w3 + h4 * w4)
        params, norm = _random_model(3)
        sur.set_model(np.concatenate([params, norm]))
        x = _random_inputs(7, 4)
        t = np.random.default_rng(5).uniform(20, 95, 7)
        xd = torch.from_numpy(x).cuda()
        td = torch.from_numpy(t.astype(np.float32)).cuda()
        loss, g = sur.gradients(7, xd.data_ptr(), td.data_ptr())
        l3, l4 = S.split_inputs(x, h3, w3, h4, w4)
        loss_ref, g_ref = S.loss_and_grad(params, norm, l3, l4, t.astype(np.float32).astype(np.float64))
        assert abs(loss - loss_ref) <= 1e-5 * max(1.0, loss_ref), (loss, loss_ref)
        scale = np.abs(g_ref).max()
        np.testing.assert_allclose(g, g_ref, rtol=2e-3, atol=1e-5 * scale)


def test_predictions_match_oracle(gpu):
    import torch
    with api.Surrogate(abi.yuv420_10bit_bt709(W, H)) as sur:
        h3, w3, h4, w4 = _level_dims(W, H)
        params, norm = _random_model(8)
        sur.set_model(np.concatenate([params, norm]))
        x = _random_inputs(9, 9)
        xd = torch.from_numpy(x).cuda()
        pred = torch.zeros(9, dtype=torch.float32, device="cuda")
        sur.predict_inputs(9, xd.data_ptr(), pred.data_ptr())
        torch.cuda.synchronize()
        l3, l4 = S.split_inputs(x, h3, w3, h4, w4)
        np.testing.assert_allclose(pred.cpu().numpy(), S.forward(params, norm, l3, l4), rtol=0, atol=1e-3)
        # the model round-trips through SetModel / Model
        np.testing.assert_array_equal(sur.model(), np.concatenate([params, norm]).astype(np.float32))


def test_coarse_inputs_match_oracle_levels(gpu, oracle_lib):
    import torch
    cs = abi.yuv420_10bit_bt709(W, H)
    pairs = synth.make_pairs(3, W, H, fmt="yuv420p10", seed=12)
    h3, w3, h4, w4 = _level_dims(W, H)
    with api.Surrogate(cs) as sur:
        dev = [([torch.from_numpy(p.view(np.uint8).copy()).cuda() for p in a],
                [torch.from_numpy(p.view(np.uint8).copy()).cuda() for p in b]) for a, b, _ in pairs]
        ls = pairs[0][2]
        out = torch.zeros((3, sur.input_elems()), dtype=torch.float16, device="cuda")
        sur.inputs(3, [t.data_ptr() for d in dev for t in d[0]], [t.data_ptr() for d in dev for t in d[1]], ls, ls,
                   out.data_ptr())
        torch.cuda.synchronize()
        got = out.cpu().numpy().astype(np.float64)
    for i, (a, b, ls_) in enumerate(pairs):
        ra, rb = oracle_lib.convert(a, ls_, cs), oracle_lib.convert(b, ls_, cs)
        l3, l4 = S.split_inputs(got[i:i + 1], h3, w3, h4, w4)
        for lv, level in ((l3[0], 3), (l4[0], 4)):
            xa, xb = oracle_lib.pyramid_level(ra, level), oracle_lib.pyramid_level(rb, level)
            np.testing.assert_allclose(lv[:3], xa, rtol=0, atol=6e-4)          # FP16 of values up to ~1
            np.testing.assert_allclose(lv[3:], xb - xa, rtol=2e-3, atol=2e-5)  # FP16 of small differences


def test_predictions_against_prepared_references_equal_pair_predictions(gpu):
    import torch
    cs = abi.yuv420_10bit_bt709(W, H)
    pairs = synth.make_pairs(5, W, H, fmt="yuv420p10", seed=21)
    with api.Surrogate(cs) as sur:
        params, norm = _random_model(13)
        sur.set_model(np.concatenate([params, norm]))
        dev = [([torch.from_numpy(p.view(np.uint8).copy()).cuda() for p in a],
                [torch.from_numpy(p.view(np.uint8).copy()).cuda() for p in b]) for a, b, _ in pairs]
        ls = pairs[0][2]
        p1 = [t.data_ptr() for d in dev for t in d[0]]
        p2 = [t.data_ptr() for d in dev for t in d[1]]
        direct = torch.zeros(5, dtype=torch.float32, device="cuda")
        sur.predict(5, p1, p2, ls, ls, direct.data_ptr())
        refs = torch.zeros((5, sur.reference_floats()), dtype=torch.float32, device="cuda")
        sur.references(5, p1, ls, refs.data_ptr())
        against = torch.zeros(5, dtype=torch.float32, device="cuda")
        sur.predict_against(5, refs.data_ptr(), p2, ls, against.data_ptr())
        torch.cuda.synchronize()
        np.testing.assert_array_equal(against.cpu().numpy(), direct.cpu().numpy())


def test_trained_surrogate_saves_exact_calls(gpu):
    import torch
    w = h = 512
    cs = abi.yuv420_10bit_bt709(w, h)
    with api.Surrogate(cs) as sur, api.SSIMU2(cs) as ex:
        n, held = 16384, 1024
        X, T = tq.build_training_set(sur, ex, n + held, w, h, seed=7)
        hist = sur.train(n, X.data_ptr(), T.data_ptr(), epochs=8, batch=256, lr=3e-3, seed=3)
        assert hist[-1] < 0.25 * hist[0]
        pred = torch.zeros(held, dtype=torch.float32, device="cuda")
        sur.predict_inputs(held, X[n].data_ptr(), pred.data_ptr())
        torch.cuda.synchronize()
        t = T[n:].cpu().numpy()
        assert tq.rmse(pred.cpu().numpy(), t) < 0.25 * t.std()
        del X, T
        gen = tq.GpuFrames()
        frames = 48
        refs = gen.references(frames, w, h, seed=99)
        ref_yuv = gen.yuv420p10(refs)

        def fy(i0, i1):
            return tuple(x[i0:i1] for x in ref_yuv)

        def dy(i0, i1, st):
            return gen.yuv420p10(gen.dct_quantize(refs[i0:i1], st))

        exact_only = tq.search(fy, dy, frames, ex, None)
        guided = tq.search(fy, dy, frames, ex, sur)
        assert guided["probes"] == exact_only["probes"] == exact_only["exact_calls"]
        assert guided["exact_calls"] <= 0.6 * exact_only["exact_calls"], (guided["exact_calls"], exact_only["exact_calls"])
        fa = tq.final_scores(fy, dy, frames, ex, exact_only["step"])
        fb = tq.final_scores(fy, dy, frames, ex, guided["step"])
        assert np.mean(np.abs(fb - 80.0)) <= np.mean(np.abs(fa - 80.0)) + 0.5
