"""The FP64 surrogate oracle's analytic gradients against central finite differences (CPU).

The oracle is what the CUDA training kernels are checked against (tests/test_surrogate_gpu.py),
so its own backward pass is pinned here first.
"""
import numpy as np

from oracle import surrogate as S


def _problem(seed=0, n=3, h3=6, w3=5, h4=3, w4=3):
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
    # FP16-exact conv weights so that finite differences see the same function the gradient
    # describes (the forward pass rounds them to FP16).
    for k in ("W1", "W2", "W3"):
        p[k] = p[k].astype(np.float16).astype(np.float64)
    params = S.pack(p)
    norm = np.concatenate([rng.uniform(-0.1, 0.1, 6), rng.uniform(0.5, 2.0, 6)])
    l3 = rng.normal(0, 1, (n, 6, h3, w3))
    l4 = rng.normal(0, 1, (n, 6, h4, w4))
    t = rng.uniform(20, 95, n)
    return params, norm, l3, l4, t


def test_oracle_gradient_matches_finite_differences():
    params, norm, l3, l4, t = _problem()
    loss, g = S.loss_and_grad(params, norm, l3, l4, t)
    assert np.isfinite(loss) and g.shape == (S.NPARAMS,)
    rng = np.random.default_rng(5)
    biases_and_head = list(range(864, 880)) + list(range(3184, 3200)) + list(range(3328, 3369))
    conv = list(rng.choice(864, 12, replace=False)) + list(880 + rng.choice(2304, 12, replace=False))
    conv += list(3200 + rng.choice(128, 8, replace=False))
    for i in biases_and_head + conv:
        # Conv weights move by one FP16 spacing, so that the rounded weights move by exactly
        # that amount (small enough that no ReLU changes side); the rest by 1e-6.
        h = float(np.spacing(np.float16(params[i]))) if i in conv else 1e-6
        pp, pm = params.copy(), params.copy()
        pp[i] += h
        pm[i] -= h
        lp, _ = S.loss_and_grad(pp, norm, l3, l4, t)
        lm, _ = S.loss_and_grad(pm, norm, l3, l4, t)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 2e-3 * max(1.0, abs(g[i])), (i, fd, g[i])


def test_oracle_forward_matches_loss_definition():
    params, norm, l3, l4, t = _problem(seed=2)
    pred = S.forward(params, norm, l3, l4)
    loss, _ = S.loss_and_grad(params, norm, l3, l4, t)
    assert np.isclose(loss, np.mean(((pred - t) / 20.0) ** 2), rtol=1e-12)
