"""The warm-start MLP's own BF16 tensor-core kernels (three engines: warp-level mma.sync, tcgen05 a
layer per launch, and the fused tcgen05 kernel that is the default at width 128) against the numpy
restatement (tests/oracle.py mlp_forward_backward): loss and parameter gradient of one forward and
backward pass, predictions, a training run that fits a smooth field, and the exact wall
distance."""

import numpy as np
import pytest

import oracle as O
from autan_b200.warmstart import MLP, wall_distance

pytestmark = pytest.mark.gpu


def data(n, seed=0):
    rng = np.random.default_rng(seed)
    x = rng.normal(size=(n, 7)).astype(np.float32)
    y = np.stack([np.sin(x[:, 0]) * x[:, 1], np.cos(x[:, 2]), x[:, 3] * x[:, 4], np.tanh(x[:, 5]),
                  0.1 * x[:, 6] ** 2], axis=1).astype(np.float32)  # fmt: skip
    return x, y


def scaling(x, y):
    return (x.mean(0), x.std(0), y.mean(0), y.std(0))


@pytest.mark.parametrize("engine", [0, 1, 2], ids=["mma_sync", "tcgen05", "tcgen05_fused"])
def test_gradient_against_the_restatement(engine):
    """BF16 operands, FP32 sums in another order: a BF16 rounding of an activation or a dZ may
    flip; the bounds (1e-4 on the loss, 2e-2 on the gradient's norm) leave room for that."""
    x, y = data(1000)
    net = MLP(seed=3)
    net.set_engine(engine)
    sc = scaling(x, y)
    net.set_scaling(*sc)
    p = net.parameters()
    loss, g = net.gradient(x, y)
    loss0, g0 = O.mlp_forward_backward(p, x, y, tuple(np.float32(v) for v in sc))
    assert abs(loss - loss0) <= 1e-4 * loss0
    assert np.linalg.norm(g - g0) <= 2e-2 * np.linalg.norm(g0)
    # the output layer's bias gradient is an FP32 column sum of the same dZ: close
    assert np.allclose(g[-5:], g0[-5:], rtol=1e-3, atol=1e-6)


@pytest.mark.parametrize("engine", [0, 1, 2], ids=["mma_sync", "tcgen05", "tcgen05_fused"])
def test_training_fits_a_smooth_field(engine):
    x, y = data(65536, seed=1)
    net = MLP(seed=4)
    net.set_engine(engine)
    net.set_scaling(*scaling(x, y))
    net.set_data(x, y)
    loss = net.train(epochs=20, batch=4096, lr=2e-3, seed=5)
    assert loss[-1] < 0.05 * loss[0], loss
    xt, yt = data(4096, seed=2)
    pred = net.predict(xt)
    assert np.sqrt(np.mean((pred - yt) ** 2)) < 0.3 * np.sqrt(np.mean((yt - yt.mean(0)) ** 2))


@pytest.mark.parametrize("engine", [0, 1, 2], ids=["mma_sync", "tcgen05", "tcgen05_fused"])
def test_prediction_matches_the_restatement(engine):
    x, y = data(3000, seed=6)
    net = MLP(seed=7)
    net.set_engine(engine)
    sc = scaling(x, y)
    net.set_scaling(*sc)
    p = net.parameters()
    pred = net.predict(x)
    # the restatement's standardised prediction (its loss path), de-standardised
    spec, _ = O.mlp_layers(7, 128, 4, 5)
    W = [O.bf16(p[o : o + a * b].reshape(b, a)) for a, b, o in spec]
    bias = [p[o + a * b : o + a * b + b] for a, b, o in spec]
    act = O.bf16((x - sc[0]) / sc[1])
    for l in range(5):
        z = act @ W[l].T + bias[l]
        act = O.bf16(0.5 * z * (1.0 + O._erf(z / np.sqrt(2.0)))) if l < 4 else z
    want = act * sc[3] + sc[2]
    assert np.abs(pred - want).max() <= 2e-2 * np.abs(want).max()


def test_wall_distance_bit_for_bit():
    rng = np.random.default_rng(8)
    tris = [rng.normal(size=(17, 9)), rng.normal(size=(5, 9))]
    pts = [rng.normal(size=(3, 300)) * 2, rng.normal(size=(3, 100))]
    got = wall_distance(tris, pts)
    for k in range(2):
        want = [min(O.point_triangle(pts[k][:, i], t[0:3], t[3:6], t[6:9]) for t in tris[k])
                for i in range(pts[k].shape[1])]  # fmt: skip
        assert np.array_equal(got[k], np.array(want))


@pytest.mark.parametrize("rows", [5000, 40000])
def test_engines_agree(rows):
    """tcgen05 per layer, fused tcgen05 (tensor memory accumulators) and mma.sync: the same BF16
    operands and FP32 sums in different orders; predictions and gradients within the BF16 flips
    that allows. 40 000 rows: more 128-row tiles than SMs, so fused CTAs take several tiles each."""
    x, y = data(rows, seed=9)
    out = []
    for engine in (0, 1, 2):
        net = MLP(seed=10)
        net.set_engine(engine)
        net.set_scaling(*scaling(x, y))
        out.append((net.predict(x), net.gradient(x, y)))
    p0, (l0, g0) = out[0]
    for p1, (l1, g1) in out[1:]:
        assert np.abs(p0 - p1).max() <= 1e-2 * np.abs(p0).max()
        assert abs(l0 - l1) <= 1e-4 * l0
        assert np.linalg.norm(g0 - g1) <= 2e-2 * np.linalg.norm(g0)


def test_fused_engine_is_the_default_and_deterministic():
    """Width 128: the fused engine unless another is chosen; two passes give the same bits (the
    CTAs' partials are summed in a fixed order); other widths refuse it."""
    x, y = data(3000, seed=11)
    runs = []
    for _ in range(2):
        net = MLP(seed=12)
        net.set_scaling(*scaling(x, y))
        runs.append(net.gradient(x, y))
    fused = MLP(seed=12)
    fused.set_engine(2)
    fused.set_scaling(*scaling(x, y))
    assert runs[0][0] == runs[1][0] and np.array_equal(runs[0][1], runs[1][1])
    assert np.array_equal(fused.gradient(x, y)[1], runs[0][1])
    narrow = MLP(width=64, seed=12)
    with pytest.raises(Exception, match="E1101"):
        narrow.set_engine(2)


def test_experiment_small_round_trip(tmp_path):
    """The warm-start experiment end to end on a few small channels: the result's fields, one row
    per test case, the subset re-march reproducing each case's iterations, and a saved network
    that, loaded, starts the test cases the same way (same iterations, same forces)."""
    from autan_b200 import warmstart

    path = tmp_path / "net.npz"
    res = warmstart.experiment(train_cases=3, test_cases=3, cells=(300, 500), epochs=2,
                               batch_rows=256, max_steps=4000, save=path, log=lambda m: None)  # fmt: skip
    assert len(res["cases"]) == 3
    assert res["both_converged"] == sum(r["cold_converged"] and r["warm_converged"] for r in res["cases"])
    if res["both_converged"]:
        assert res["subset_iterations_match"]
        assert res["gpu_time_ratio"] > 0
    again = warmstart.experiment(train_cases=3, test_cases=3, cells=(300, 500), max_steps=4000,
                                 load=path, log=lambda m: None)  # fmt: skip
    assert [r["warm_iterations"] for r in again["cases"]] == [r["warm_iterations"] for r in res["cases"]]
    assert [r["force_rel_diff"] for r in again["cases"]] == [r["force_rel_diff"] for r in res["cases"]]
