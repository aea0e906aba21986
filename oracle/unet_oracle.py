"""CPU oracle of the learned warm-start network (test infrastructure only).

A float64 numpy restatement of the 3-level 3D U-Net that platoanalyze_b200/csrc/unet.cu
evaluates and trains on the GPU (no Plato Analyze counterpart: the reference has no learned
component).  With `bf16=True` it rounds to bfloat16 (round to nearest even) at exactly the
points where the GPU stores BF16 - the packed input, the weights, every hidden activation,
the pooled tensors, and the masked output gradients fed to the tensor cores - so the GPU
and the oracle differ only by FP32 accumulation order.  With `bf16=False` it is a plain
float64 network whose analytic gradient is checked against finite differences.

Layout: node grid n = (n0, n1, n2) padded with zeros to multiples of 4 (level 0), halved
twice by 2x2x2 average pooling; tensors are (batch, d, h, w, channels).  Parameters: per
layer, weights [taps][cout][cin] then bias [cout], layers in the order below.
"""
from __future__ import annotations

import numpy as np

# (cin, cout, taps, relu): e0a e0b e1a e1b e2a e2b d1a d1b d0a d0b head
LAYERS = [(16, 16, 27, 1), (16, 16, 27, 1), (16, 32, 27, 1), (32, 32, 27, 1), (32, 64, 27, 1), (64, 64, 27, 1),
          (96, 32, 27, 1), (32, 32, 27, 1), (48, 16, 27, 1), (16, 16, 27, 1), (16, 9, 1, 0)]


def num_params() -> int:
    return sum(t * co * ci + co for ci, co, t, _ in LAYERS)


def bf16_round(x: np.ndarray) -> np.ndarray:
    """Round to the nearest bfloat16 (ties to even), returned as float64."""
    f = np.ascontiguousarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def split_params(p: np.ndarray):
    out, off = [], 0
    for ci, co, t, _ in LAYERS:
        w = p[off:off + t * co * ci].reshape(t, co, ci)
        off += t * co * ci
        b = p[off:off + co]
        off += co
        out.append((w, b))
    return out


def _taps(t):
    return [(0, 0, 0)] if t == 1 else [(dz, dy, dx) for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1)]


def conv(x, w, b, relu):
    """y[v, o] = act(b[o] + sum_t sum_c w[t, o, c] x[v + o_t, c]) with zero padding."""
    B, D, H, W, _ = x.shape
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (1, 1), (0, 0)))
    y = np.zeros((B, D, H, W, w.shape[1]))
    for k, (dz, dy, dx) in enumerate(_taps(w.shape[0])):
        xs = xp[:, 1 + dz:1 + dz + D, 1 + dy:1 + dy + H, 1 + dx:1 + dx + W, :]
        y += np.einsum("bzyxc,oc->bzyxo", xs, w[k])
    if b is not None:
        y += b
    return np.maximum(y, 0.0) if relu else y


def conv_data_grad(m, w):
    """dx[u, c] = sum_t sum_o w[t, o, c] m[u - o_t, o]."""
    B, D, H, W, _ = m.shape
    mp = np.pad(m, ((0, 0), (1, 1), (1, 1), (1, 1), (0, 0)))
    dx = np.zeros((B, D, H, W, w.shape[2]))
    for k, (dz, dy, dx_) in enumerate(_taps(w.shape[0])):
        ms = mp[:, 1 - dz:1 - dz + D, 1 - dy:1 - dy + H, 1 - dx_:1 - dx_ + W, :]
        dx += np.einsum("bzyxo,oc->bzyxc", ms, w[k])
    return dx


def conv_weight_grad(x, m, taps):
    B, D, H, W, _ = x.shape
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (1, 1), (0, 0)))
    out = []
    for dz, dy, dx in _taps(taps):
        xs = xp[:, 1 + dz:1 + dz + D, 1 + dy:1 + dy + H, 1 + dx:1 + dx + W, :]
        out.append(np.einsum("bzyxo,bzyxc->oc", m, xs))
    return np.stack(out)


def pool(x):
    B, D, H, W, C = x.shape
    return x.reshape(B, D // 2, 2, H // 2, 2, W // 2, 2, C).mean(axis=(2, 4, 6))


def pool_grad(g):
    return np.repeat(np.repeat(np.repeat(g, 2, axis=1), 2, axis=2), 2, axis=3) * 0.125


def upsample(x):
    return np.repeat(np.repeat(np.repeat(x, 2, axis=1), 2, axis=2), 2, axis=3)


def upsample_grad(g):
    B, D, H, W, C = g.shape
    return g.reshape(B, D // 2, 2, H // 2, 2, W // 2, 2, C).sum(axis=(2, 4, 6))


class UNetOracle:
    def __init__(self, nodes, bf16: bool = True):
        self.n = tuple(int(v) for v in nodes)
        self.g0 = tuple((v + 3) // 4 * 4 for v in self.n)
        self.bf16 = bf16

    def _r(self, x):
        return bf16_round(x) if self.bf16 else x

    def forward(self, params, inp):
        """inp [B][n0][n1][n2][8] -> output [B][n0][n1][n2][9]; keeps the activations."""
        P = [(self._r(w), b) for w, b in split_params(np.asarray(params, np.float64))]
        B = inp.shape[0]
        x = np.zeros((B,) + self.g0 + (16,))
        n0, n1, n2 = self.n
        x[:, :n0, :n1, :n2, :8] = self._r(inp)
        a = {"in": x}
        a["x0a"] = self._r(conv(x, *P[0], True))
        a["s0"] = self._r(conv(a["x0a"], *P[1], True))
        a["p1"] = self._r(pool(a["s0"]))
        a["x1a"] = self._r(conv(a["p1"], *P[2], True))
        a["s1"] = self._r(conv(a["x1a"], *P[3], True))
        a["p2"] = self._r(pool(a["s1"]))
        a["x2a"] = self._r(conv(a["p2"], *P[4], True))
        a["x2b"] = self._r(conv(a["x2a"], *P[5], True))
        a["cat1"] = np.concatenate([upsample(a["x2b"]), a["s1"]], axis=-1)
        a["x1c"] = self._r(conv(a["cat1"], *P[6], True))
        a["x1d"] = self._r(conv(a["x1c"], *P[7], True))
        a["cat0"] = np.concatenate([upsample(a["x1d"]), a["s0"]], axis=-1)
        a["x0c"] = self._r(conv(a["cat0"], *P[8], True))
        a["x0d"] = self._r(conv(a["x0c"], *P[9], True))
        a["out"] = conv(a["x0d"], *P[10], False)
        self._a, self._P = a, P
        return a["out"][:, :n0, :n1, :n2, :9]

    def loss_and_gradients(self, params, inp, tgt):
        out = self.forward(params, inp)
        a, P = self._a, self._P
        n0, n1, n2 = self.n
        cnt = out.size
        loss = float(np.sum((out - tgt) ** 2) / cnt)
        g = np.zeros_like(a["out"])
        g[:, :n0, :n1, :n2, :9] = 2.0 / cnt * (out - tgt)
        grads = [None] * len(LAYERS)

        def layer(k, dy, y, x, relu=True):
            m = self._r(dy * (y > 0) if relu else dy)
            grads[k] = (conv_weight_grad(x, m, LAYERS[k][2]), m.sum(axis=(0, 1, 2, 3)))
            return conv_data_grad(m, P[k][0])

        d = layer(10, g, None, a["x0d"], relu=False)
        d = layer(9, d, a["x0d"], a["x0c"])
        dcat0 = layer(8, d, a["x0c"], a["cat0"])
        d = upsample_grad(dcat0[..., :32])
        d = layer(7, d, a["x1d"], a["x1c"])
        dcat1 = layer(6, d, a["x1c"], a["cat1"])
        d = upsample_grad(dcat1[..., :64])
        d = layer(5, d, a["x2b"], a["x2a"])
        d = layer(4, d, a["x2a"], a["p2"])
        ds1 = dcat1[..., 64:] + pool_grad(d)
        d = layer(3, ds1, a["s1"], a["x1a"])
        d = layer(2, d, a["x1a"], a["p1"])
        ds0 = dcat0[..., 32:] + pool_grad(d)
        d = layer(1, ds0, a["s0"], a["x0a"])
        layer(0, d, a["x0a"], a["in"])
        flat = np.concatenate([np.concatenate([w.reshape(-1), b]) for w, b in grads])
        return loss, flat


def init_params(seed: int = 0) -> np.ndarray:
    """He-normal weights (fan-in = taps * cin), zero biases, FP32."""
    rng = np.random.default_rng(seed)
    parts = []
    for ci, co, t, relu in LAYERS:
        std = np.sqrt((2.0 if relu else 1.0) / (t * ci))
        parts += [rng.standard_normal(t * co * ci) * std, np.zeros(co)]
    return np.concatenate(parts).astype(np.float32)
