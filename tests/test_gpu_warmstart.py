"""The Darcy warm-start network's tensor-core kernels against the CPU
oracle (oracle/warmstart_oracle.py, itself pinned by finite differences),
and the learned warm start inside the Darcy solve.

The device rounds to BF16 at the same points as the oracle; what remains is
FP32 (device) against FP64 (oracle) accumulation, which can flip an
occasional BF16 rounding of an activation.  Tolerances: outputs within
1e-2 of their largest magnitude, weight gradients within a relative L2
error of 2e-2 per layer (the bias gradients likewise)."""
import numpy
import pytest

import warmstart_oracle as WO

pytestmark = pytest.mark.gpu


def _case(shape, seed):
    nx, ny, nz = shape
    n = nx * ny * nz
    rng = numpy.random.default_rng(seed)
    x3 = rng.normal(size=(n, WO.INPUTS)).astype(numpy.float32)
    target = rng.normal(size=n).astype(numpy.float32)
    free = (rng.uniform(size=n) > 0.15).astype(numpy.uint8)
    return x3, target, free


@pytest.mark.parametrize("shape", [(12, 10, 9), (16, 16, 8), (5, 7, 3)])
def test_network_matches_oracle(shape):
    from sphere_b200.engine import WSNet
    params = WO.random_params(7, 1.5)
    net = WSNet(*shape)
    for layer, (w, b) in enumerate(params):
        net.set_params(layer, w, b)
    x3, target, free = _case(shape, 5)
    out = net.forward(x3)
    ref = WO.Net(shape, params, bf16=True)
    out_ref = ref.forward(x3)
    assert numpy.abs(out - out_ref).max() <= 1e-2 * numpy.abs(out_ref).max()
    dw, db = net.gradients(x3, target, free)
    dw_ref, db_ref = ref.gradients(target, free)
    for layer in range(3):
        e = numpy.linalg.norm(dw[layer] - dw_ref[layer]) / numpy.linalg.norm(dw_ref[layer])
        assert e <= 2e-2, (layer, e)
        eb = numpy.linalg.norm(db[layer] - db_ref[layer]) / max(numpy.linalg.norm(db_ref[layer]), 1e-30)
        assert eb <= 2e-2, (layer, eb)
    # structure: unused input channels and output channels get no gradient
    assert numpy.all(dw[0][:, :, WO.INPUTS:] == 0.0) and numpy.all(dw[2][:, 1:, :] == 0.0)
    net.close()


def test_parameters_round_trip():
    from sphere_b200.engine import WSNet
    net = WSNet(8, 8, 8, seed=3)
    w, b = net.get_params(1)
    assert numpy.abs(w).max() > 0.0 and w.shape == (27, 16, 16)
    w2 = w * 0.5
    net.set_params(1, w2, b)
    w3, _ = net.get_params(1)
    assert numpy.array_equal(w3, w2)
    net.close()


def _consolidation(seed=61, n=400, steps_dt=1.0):
    from sphere_b200 import configs
    d = configs.settling_lattice(n=n, seed=seed, nx=8, ny=8, nz=8, spacing=0.0195, steps=40)
    configs.add_top_wall(d, 40e3)
    d.w_x[0] -= 0.002
    configs.init_fluid_darcy(d, mu=1.797e-6, k_c=3.5e-13, tolerance=1e-8, maxiter=200000,
                             bottom_no_flow=True)
    return d


def test_warm_start_in_the_solve():
    """The learned start trains on the engine's own solves; afterwards its
    first-iteration residual wins the comparison with the previous-step
    guess on most solves, and the solves it starts need fewer iterations to
    reach the same tolerance than the plain engine's (exact counts)."""
    from sphere_b200.engine import Engine
    d = _consolidation()
    plain = Engine(d, fluid=True)
    warm = Engine(d, fluid=True, warm_start=True)
    it_plain, it_warm = [], []
    for step in range(160):
        assert plain.step(1) == 0
        assert warm.step(1) == 0
        it_plain.append(int(plain.get("darcy_iters_exact")[0]))
        it_warm.append(int(warm.get("darcy_iters_exact")[0]))
    stats = warm.get("darcy_warm")
    predictions, trained, picked = int(stats[0]), int(stats[1]), int(stats[2])
    loss = float(stats[3:4].view(numpy.float64)[0])
    print("iterations plain", numpy.mean(it_plain[-60:]), "warm", numpy.mean(it_warm[-60:]),
          "predictions", predictions, "trained", trained, "picked", picked, "loss", loss)
    # training starts with the second solve (the first sets the scale)
    assert predictions == 160 and trained == 159
    assert numpy.isfinite(loss)
    assert picked > 0
    assert numpy.mean(it_warm[-60:]) < numpy.mean(it_plain[-60:])
    plain.close()
    warm.close()


def test_extrapolation_start():
    """warm_start = 2: the start is the linear extrapolation of the last two
    solutions (no network); the solve still runs to the same tolerance and
    the fallback keeps the previous solution when it is better."""
    from sphere_b200.engine import Engine
    d = _consolidation(seed=62)
    plain = Engine(d, fluid=True)
    extra = Engine(d, fluid=True, warm_start=2)
    it_plain, it_extra = [], []
    for step in range(80):
        assert plain.step(1) == 0
        assert extra.step(1) == 0
        it_plain.append(int(plain.get("darcy_iters_exact")[0]))
        it_extra.append(int(extra.get("darcy_iters_exact")[0]))
    stats = extra.get("darcy_warm")
    print("iterations plain", numpy.mean(it_plain[-40:]), "extrapolation", numpy.mean(it_extra[-40:]),
          "picked", int(stats[2]))
    assert int(stats[1]) == 0           # no network, no training
    assert numpy.mean(it_extra[-40:]) <= numpy.mean(it_plain[-40:])
    plain.close()
    extra.close()


def test_learned_start_against_extrapolation_alone():
    """What the trained network adds to its extrapolation in time
    (warm_start 1 against 2, same tolerance and stop rule, exact iteration
    counts over the second half of the run).  On the consolidation runs
    measured so far it adds nothing: the extrapolation alone already halves
    the iterations of the plain start, and the network's corrected guess,
    when it wins the first-residual comparison, converges no faster.  The
    comparison with the fallback bounds what the network can cost: at most
    5 % more iterations than the extrapolation alone."""
    from sphere_b200.engine import Engine
    d = _consolidation(seed=61)
    runs = {}
    for mode in (0, 1, 2):
        e = Engine(d, fluid=True, warm_start=mode)
        it = []
        for step in range(120):
            assert e.step(1) == 0
            it.append(int(e.get("darcy_iters_exact")[0]))
        runs[mode] = float(numpy.mean(it[60:]))
        e.close()
    print("iterations per solve: plain", runs[0], "learned", runs[1], "extrapolation", runs[2],
          "network gain", runs[2] / max(runs[1], 1e-9))
    assert runs[2] < runs[0] and runs[1] < runs[0]
    assert runs[1] <= 1.05 * runs[2]
