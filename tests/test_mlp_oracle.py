"""The numpy restatement of the warm-start MLP (tests/oracle.py), pinned on CPU: its backward pass
against central finite differences of its own loss in FP64 without rounding, and its BF16
rounding against the standard round-to-nearest-even; the point-triangle distance against brute
force sampling of the triangle."""

import numpy as np

import oracle as O


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(0)
    inputs, width, layers, outputs = 7, 16, 2, 5
    _, count = O.mlp_layers(inputs, width, layers, outputs)
    p = rng.normal(0.0, 0.3, count)
    x = rng.normal(size=(23, inputs))
    y = rng.normal(size=(23, outputs))
    sc = (np.zeros(inputs), np.ones(inputs), np.zeros(outputs), np.ones(outputs))
    kw = dict(inputs=inputs, width=width, layers=layers, outputs=outputs, exact=True)
    _, g = O.mlp_forward_backward(p, x, y, sc, **kw)
    for i in rng.choice(count, 40, replace=False):
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (O.mlp_forward_backward(pp, x, y, sc, **kw)[0] - O.mlp_forward_backward(pm, x, y, sc, **kw)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])), (i, fd, g[i])


def test_bf16_rounding():
    v = np.array([1.0, 1.0 + 2**-8, 1.0 + 3 * 2**-9, -2.5, 3.0e38, 1e-40], dtype=np.float32)
    r = O.bf16(v)
    assert r[0] == 1.0
    assert r[1] == 1.0  # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: even is 1
    assert r[2] == np.float32(1.0 + 2**-7)
    assert r[3] == -2.5
    assert np.all((r.view(np.uint32) & 0xFFFF) == 0)


def test_point_triangle_distance_against_sampling():
    rng = np.random.default_rng(1)
    for _ in range(200):
        a, b, c = rng.normal(size=(3, 3))
        p = rng.normal(size=3) * 2
        d = O.point_triangle(p, a, b, c)
        u, v = rng.random((2, 20000))
        flip = u + v > 1
        u[flip], v[flip] = 1 - u[flip], 1 - v[flip]
        pts = a + u[:, None] * (b - a) + v[:, None] * (c - a)
        sampled = np.sqrt(((pts - p) ** 2).sum(axis=1)).min()
        assert d <= sampled + 1e-12
        assert d >= sampled - 0.05 * np.linalg.norm(np.cross(b - a, c - a)) ** 0.5
