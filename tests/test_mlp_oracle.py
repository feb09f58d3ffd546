"""CPU oracle of the warm-start network: its analytic gradients (FP64, no
BF16 rounding) against central finite differences, and the BF16 rounding
helper against known values."""
import numpy as np


def mlp_oracle():
    import sys, os
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))
    import mlp_oracle as m
    return m


def random_params(m, rng, scale=0.3):
    layers = []
    for i, o in zip(m.DIMS_IN, m.DIMS_OUT):
        w = rng.uniform(-scale, scale, (o, i)) * np.sqrt(6.0 / (i + o)) / scale
        if i == 16:
            w[:, 4:] = 0.0
        layers.append((w, rng.uniform(-0.1, 0.1, o)))
    return m.flatten(layers)


def test_bf16_rounding_known_values():
    m = mlp_oracle()
    v = m.bf16(np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.0 ** -130, 65504.0]))
    assert v[0] == 1.0 and v[1] == 1.0              # tie to even
    assert v[2] == 1.0 + 2 ** -6                    # tie rounds up to the even neighbour
    assert v[3] == -2.0 ** -130                     # subnormal-range value representable
    assert v[4] == 65536.0


def test_gradients_match_finite_differences():
    m = mlp_oracle()
    rng = np.random.default_rng(0)
    flat = random_params(m, rng)
    x = rng.uniform(-1, 1, (6, 4))
    t = rng.normal(size=(6, 512))
    _, g = m.loss_and_gradients(flat, x, t, rounding=False)
    offs = np.cumsum([0] + [o * i + o for i, o in zip(m.DIMS_IN, m.DIMS_OUT)])
    picks = []
    for l in range(4):
        lo, hi = offs[l], offs[l + 1]
        cand = np.arange(lo, hi)
        if l == 0:  # padded inputs have zero gradient; test real weights and biases
            w = np.arange(lo, lo + 256 * 16).reshape(256, 16)[:, :4].ravel()
            cand = np.concatenate([w, np.arange(lo + 256 * 16, hi)])
        picks.extend(rng.choice(cand, 12, replace=False))
    h = 1e-6
    for i in picks:
        fp, fm = flat.copy(), flat.copy()
        fp[i] += h
        fm[i] -= h
        lp, _ = m.loss_and_gradients(fp, x, t, rounding=False)
        lm, _ = m.loss_and_gradients(fm, x, t, rounding=False)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-7 + 1e-5 * abs(g[i]), (i, fd, g[i])
    # padded layer-0 inputs get exactly zero gradient
    w0 = g[:256 * 16].reshape(256, 16)
    assert np.all(w0[:, 4:] == 0.0)
