"""The warm-start network's CPU oracle pinned by finite differences: with
BF16 rounding switched off its gradients must match central differences of
its own loss, so the oracle can stand as the reference for the device's
tensor-core backward pass."""
import numpy as np

import warmstart_oracle as W


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 3.0e-20, 0.0], dtype=np.float32)
    r = W.bf16_round(x)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: ties go to even (1.0)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2 ** -7
    assert r[3] == -2.5 and r[5] == 0.0
    assert abs(r[4] - 3.0e-20) / 3.0e-20 < 2 ** -8


def test_gradients_match_finite_differences():
    shape = (4, 3, 5)
    n = 4 * 3 * 5
    rng = np.random.default_rng(3)
    params = [(w.astype(np.float64), b.astype(np.float64)) for w, b in W.random_params(11, 2.0)]
    x3 = rng.normal(size=(n, W.INPUTS))
    target = rng.normal(size=n)
    free = (rng.uniform(size=n) > 0.2).astype(np.uint8)

    def loss_of(ps):
        net = W.Net(shape, ps, bf16=False)
        net.forward(x3)
        return net.loss(target, free)

    net = W.Net(shape, params, bf16=False)
    net.forward(x3)
    dw, db = net.gradients(target, free)
    eps = 1e-6
    checked = 0
    for layer in range(3):
        cin = W.INPUTS if layer == 0 else 16
        cout = 1 if layer == 2 else 16
        for _ in range(12):
            t, o, i = rng.integers(27), rng.integers(cout), rng.integers(cin)
            up = [(w.copy(), b.copy()) for w, b in params]
            dn = [(w.copy(), b.copy()) for w, b in params]
            up[layer][0][t, o, i] += eps
            dn[layer][0][t, o, i] -= eps
            fd = (loss_of(up) - loss_of(dn)) / (2 * eps)
            assert abs(fd - dw[layer][t, o, i]) <= 1e-5 * max(1.0, abs(fd)), (layer, t, o, i)
            checked += 1
        o = rng.integers(cout)
        up = [(w.copy(), b.copy()) for w, b in params]
        dn = [(w.copy(), b.copy()) for w, b in params]
        up[layer][1][o] += eps
        dn[layer][1][o] -= eps
        fd = (loss_of(up) - loss_of(dn)) / (2 * eps)
        assert abs(fd - db[layer][o]) <= 1e-5 * max(1.0, abs(fd))
    assert checked == 36
    # unused channels get exactly zero gradient
    assert np.all(dw[0][:, :, W.INPUTS:] == 0.0) and np.all(dw[2][:, 1:, :] == 0.0)
    assert np.all(db[2][1:] == 0.0)
