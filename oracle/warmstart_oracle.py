"""CPU oracle of the Darcy warm-start network -- TEST INFRASTRUCTURE ONLY.

A plain numpy restatement of the network the engine trains on the tensor
cores (4 -> 16 -> 16 -> 1 channels, 3x3x3 kernels with zero padding, ReLU
after layers 1 and 2), its mean-squared-error loss over free cells and the
gradients of every weight and bias.  Arithmetic is float64; with
``bf16=True`` the values are rounded to BF16 (round to nearest even) at the
same points as the device kernels: the packed inputs, the weights, the
activations after ReLU, and the gradients stored between layers.  Without
rounding the gradients are exact and are checked against finite
differences in tests/test_warmstart_oracle.py.

Layouts match the C ABI: inputs [ncells][4] and outputs [ncells] with x
fastest; weights [27 taps][16 out][16 in] with tap = (dz+1)*9 + (dy+1)*3 +
(dx+1); biases [16].
"""
import numpy as np

TAPS = [(dz, dy, dx) for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1)]
INPUTS = 4   # previous pressure, porosity, porosity change, previous pressure change


def bf16_round(a):
    """float -> nearest BF16 (ties to even), returned as float64."""
    f = np.asarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    u = ((u + 0x7FFF + lsb) & 0xFFFF0000).astype(np.uint32)
    return u.view(np.float32).astype(np.float64)


def _shift(x, dz, dy, dx):
    """y[z, y, x] = x[z + dz, y + dy, x + dx], zero outside the grid."""
    nz, ny, nx = x.shape[:3]
    out = np.zeros_like(x)
    zs, ys, xs = slice(max(0, -dz), nz - max(0, dz)), slice(max(0, -dy), ny - max(0, dy)), \
        slice(max(0, -dx), nx - max(0, dx))
    zt, yt, xt = slice(max(0, dz), nz + min(0, dz)), slice(max(0, dy), ny + min(0, dy)), \
        slice(max(0, dx), nx + min(0, dx))
    out[zs, ys, xs] = x[zt, yt, xt]
    return out


def conv(x, w):
    """out[c, o] = sum_tap sum_i w[tap, o, i] x[c + off(tap), i]."""
    out = np.zeros(x.shape[:3] + (w.shape[1],))
    for t, (dz, dy, dx) in enumerate(TAPS):
        out += _shift(x, dz, dy, dx) @ w[t].T
    return out


def conv_input_grad(g, w):
    """d/dx of sum(g * conv(x, w)): dx[c, i] = sum w[tap, o, i] g[c - off(tap), o]."""
    out = np.zeros(g.shape[:3] + (w.shape[2],))
    for t, (dz, dy, dx) in enumerate(TAPS):
        out += _shift(g, -dz, -dy, -dx) @ w[t]
    return out


def conv_weight_grad(x, g):
    """dw[tap, o, i] = sum_c x[c + off(tap), i] g[c, o]."""
    dw = np.zeros((27, g.shape[-1], x.shape[-1]))
    gf = g.reshape(-1, g.shape[-1])
    for t, (dz, dy, dx) in enumerate(TAPS):
        dw[t] = gf.T @ _shift(x, dz, dy, dx).reshape(-1, x.shape[-1])
    return dw


class Net:
    def __init__(self, shape, params, bf16=True):
        """shape = (nx, ny, nz); params = [(w, b)] * 3."""
        self.nx, self.ny, self.nz = shape
        self.r = bf16_round if bf16 else (lambda a: np.asarray(a, dtype=np.float64))
        self.w = [self.r(np.asarray(w, dtype=np.float64)) for w, _ in params]
        self.b = [np.asarray(b, dtype=np.float64) for _, b in params]

    def _grid(self, a):
        return a.reshape(self.nz, self.ny, self.nx, -1)

    def forward(self, x4):
        x0 = np.zeros((self.nz, self.ny, self.nx, 16))
        x0[..., :INPUTS] = self._grid(self.r(np.asarray(x4, dtype=np.float64)))
        a1 = self.r(np.maximum(conv(x0, self.w[0]) + self.b[0], 0.0))
        a2 = self.r(np.maximum(conv(a1, self.w[1]) + self.b[1], 0.0))
        out = conv(a2, self.w[2])[..., 0] + self.b[2][0]
        self.cache = (x0, a1, a2)
        self.out = out.reshape(-1)
        return self.out

    def loss(self, target, free):
        f = np.asarray(free) != 0
        e = self.out - np.asarray(target, dtype=np.float64)
        return float(np.sum(e[f] ** 2) / max(int(f.sum()), 1))

    def gradients(self, target, free):
        x0, a1, a2 = self.cache
        f = np.asarray(free) != 0
        nf = max(int(f.sum()), 1)
        g3 = np.zeros((self.out.size, 16))
        g3[:, 0] = np.where(f, 2.0 * (self.out - np.asarray(target, dtype=np.float64)) / nf, 0.0)
        g3 = self._grid(self.r(g3))
        dw3, db3 = conv_weight_grad(a2, g3), g3.reshape(-1, 16).sum(axis=0)
        g2 = self.r(conv_input_grad(g3, self.w[2]) * (a2 > 0))
        dw2, db2 = conv_weight_grad(a1, g2), g2.reshape(-1, 16).sum(axis=0)
        g1 = self.r(conv_input_grad(g2, self.w[1]) * (a1 > 0))
        dw1, db1 = conv_weight_grad(x0, g1), g1.reshape(-1, 16).sum(axis=0)
        return [dw1, dw2, dw3], [db1, db2, db3]


def random_params(seed, scale=1.0):
    """Parameters with the engine's structure: layer 1 reads INPUTS
    channels, layer 3 writes channel 0 only."""
    rng = np.random.default_rng(seed)
    out = []
    for layer in range(3):
        cin = INPUTS if layer == 0 else 16
        cout = 1 if layer == 2 else 16
        w = np.zeros((27, 16, 16), dtype=np.float32)
        w[:, :cout, :cin] = rng.normal(0.0, scale * np.sqrt(2.0 / (27 * cin)), (27, cout, cin))
        b = np.zeros(16, dtype=np.float32)
        b[:cout] = rng.normal(0.0, 0.05 * scale, cout)
        out.append((w, b))
    return out
