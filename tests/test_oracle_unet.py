"""The CPU oracle of the warm-start network: its analytic gradient against central finite
differences (float64, no BF16 rounding), and its BF16 rounding helper."""
import numpy as np

from unet_oracle import LAYERS, UNetOracle, bf16_round, init_params, num_params


def test_bf16_round_to_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 3.140625, 1e-3], dtype=np.float64)
    r = bf16_round(x)
    assert r[0] == 1.0
    assert r[1] == 1.0                      # tie -> even (mantissa 0)
    assert r[2] == 1.0 + 2 ** -7            # above the tie -> up
    assert r[3] == -2.5 and r[4] == 3.140625
    assert abs(r[5] - 1e-3) <= 2 ** -9 * 1e-3


def test_gradient_matches_finite_differences():
    nodes = (5, 3, 3)
    orc = UNetOracle(nodes, bf16=False)
    rng = np.random.default_rng(2)
    p = init_params(7).astype(np.float64) + 0.05 * rng.standard_normal(num_params())
    inp = rng.uniform(-1, 1, (1,) + nodes + (8,))
    tgt = rng.standard_normal((1,) + nodes + (9,))
    loss, g = orc.loss_and_gradients(p, inp, tgt)
    # two weights and one bias of every layer (first layer: weights on the 8 live input channels)
    idx, off = [], 0
    for ci, co, t, _ in LAYERS:
        nw = t * co * ci
        cand = [off + int(k) for k in rng.choice(nw, 40, replace=False) if off != 0 or (k % ci) < 8]
        idx += cand[:2] + [off + nw + int(rng.integers(co))]
        off += nw + co
    eps = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += eps
        pm[i] -= eps
        fd = (orc.loss_and_gradients(pp, inp, tgt)[0] - orc.loss_and_gradients(pm, inp, tgt)[0]) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-5 * max(abs(fd), abs(g[i])) + 1e-9, (i, fd, g[i])
