"""The CPU restatement of the surrogate network: its analytic gradient against central finite
differences (without the BF16 roundings, which make the rounded network piecewise constant), and the
BF16 rounding against its definition."""
import numpy as np

from oracle import surrogate_oracle as O


def _case(seed, n=64):
    theta, freq = O.random_params(seed, freq_sigma=1.5)
    theta = theta.astype(np.float64)
    rng = np.random.default_rng(seed + 1)
    pts = rng.uniform(-1, 1, (n, 3)).astype(np.float32)
    tgt = rng.uniform(-0.3, 0.3, n).astype(np.float32)
    io = np.array([0, 0, 0, 1, 1, 1, 0.25], np.float32)
    return theta, freq, pts, tgt, io


def _loss(theta, freq, pts, tgt, io):
    f = O.forward(pts, theta, freq, io, rounding=False)
    t = np.clip(tgt.astype(np.float64), -io[6], io[6])
    return float(np.mean((f - t) ** 2))


def test_gradient_matches_finite_differences():
    theta, freq, pts, tgt, io = _case(3)
    g, loss = O.gradient(pts, tgt, theta, freq, io, rounding=False)
    assert abs(loss - _loss(theta, freq, pts, tgt, io)) < 1e-12
    rng = np.random.default_rng(0)
    # every block of the parameter vector: hidden weights of each layer, biases, output weights and bias
    idx = np.concatenate([rng.choice(O.W * O.W, 6, replace=False) + l * O.W * O.W for l in range(O.NL)] +
                         [O.NW + rng.choice(O.NL * O.W, 8, replace=False),
                          O.NW + O.NL * O.W + rng.choice(O.W, 4, replace=False), [O.NPARAM - 1]])
    h = 1e-6
    for i in idx:
        tp, tm = theta.copy(), theta.copy()
        tp[i] += h
        tm[i] -= h
        fd = (_loss(tp, freq, pts, tgt, io) - _loss(tm, freq, pts, tgt, io)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)) + 1e-9, (i, fd, g[i])


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -2.5, 3.0e-3, 65504.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8],
                 np.float32)
    r = O.bf16(x)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: nearest even is 1; 1 + 3 * 2^-8 rounds up to 1 + 2^-6
    assert r[0] == 1.0 and r[6] == 1.0 and r[7] == np.float32(1.0 + 2 ** -6)
    assert (r.view(np.uint32) & 0xFFFF == 0).all()
    assert np.all(np.abs(r - x) <= np.abs(x) * 2 ** -8)
