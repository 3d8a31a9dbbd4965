"""The steady convergence rule (runtime/src/run.cpp:2351-2389 with round_off.hpp), host side: the
library's autan_convergence_iteration against the Python restatement in tests/oracle.py, on
synthetic residual histories that exercise the drop, the momentum reference, the exemption of an
identically zero equation (and its waking) and the round-off plateau of fp32+acc64 runs."""

import numpy as np
import pytest

import oracle as O
from autan_b200 import cases
from autan_b200.euler import ROUND_OFF_FLOOR, convergence_iteration, residual_scales


def history(n, rates, start, noise=0.05, seed=0, floor=None):
    rng = np.random.default_rng(seed)
    it = np.arange(n)[:, None]
    r = np.asarray(start)[None, :] * np.exp(-np.asarray(rates)[None, :] * it)
    r = r * (1.0 + noise * rng.standard_normal(r.shape))
    if floor is not None:
        r = np.maximum(r, np.asarray(floor)[None, :] * (1.0 + 0.02 * rng.standard_normal(r.shape)))
    return np.abs(r)


@pytest.mark.parametrize("orders", [3.0, 5.0, 8.0])
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_drop_matches_the_restatement(orders, seed):
    r = history(3000, [0.010, 0.012, 0.009, 0.011, 0.010], [1.0, 0.4, 0.3, 0.2, 2.0], seed=seed)
    want = O.convergence_iteration(r, orders)
    got = convergence_iteration(r, orders)
    assert got == want
    assert got[0] > 0


def test_momentum_drops_from_the_largest_momentum_reference():
    # momentum z starts tiny (but above the zero floor) and never drops: it converges against the
    # largest first momentum residual, so the run still converges
    r = history(2000, [0.02, 0.02, 0.02, 0.0, 0.02], [1.0, 0.5, 0.5, 1e-9, 1.0], noise=0.0)
    it, _ = convergence_iteration(r, 6.0)
    assert it > 0 and (it, 0) == O.convergence_iteration(r, 6.0)


def test_zero_equation_is_exempt_until_it_wakes():
    r = history(1500, [0.02, 0.02, 0.02, 0.0, 0.02], [1.0, 0.5, 0.5, 0.0, 1.0], noise=0.0)
    r[:, 3] = 0.0
    assert convergence_iteration(r, 4.0) == O.convergence_iteration(r, 4.0)
    assert convergence_iteration(r, 4.0)[0] > 0
    woke = r.copy()
    woke[200:, 3] = 1e-3  # leaves its floor and stays there: never converges
    assert convergence_iteration(woke, 4.0) == O.convergence_iteration(woke, 4.0) == (0, 0)


def test_round_off_plateau_of_fp32_runs():
    floors = np.full(5, 1e-6)
    r = history(4000, [0.01] * 5, [1.0, 0.5, 0.5, 0.5, 1.0], floor=[2e-6] * 5, seed=4)
    it, mask = convergence_iteration(r, 8.0, floors)
    assert (it, mask) == O.convergence_iteration(r, 8.0, floors)
    assert it > 0 and mask == 0b11111  # every equation on its plateau
    assert convergence_iteration(r, 8.0) == (0, 0)  # without floors: never


def test_residual_scales_of_the_channel():
    case = cases.bump_channel(24, 12, 4)
    g = 1.4
    phi = residual_scales(case.mesh, 1.0, 1.0 / g, 0.5, g)
    c = 1.0
    assert phi[1] == phi[2] == phi[3] == pytest.approx(phi[0] * (0.5 + c))
    assert phi[4] == pytest.approx(phi[0] * (c * c / (g - 1) + 0.125))
    assert np.all(ROUND_OFF_FLOOR * phi > 0)


@pytest.mark.parametrize("seed", [5, 6, 7, 8])
def test_plateau_with_repeated_values(seed):
    """Residuals quantised to a few levels (many equal values in the median window) and a slow
    staircase down onto the plateau: the window's median, kept incrementally, against the
    restatement's nth_element on each window."""
    rng = np.random.default_rng(seed)
    n = 3000
    floors = np.full(5, 1e-6)
    base = np.maximum(np.exp(-0.006 * np.arange(n))[:, None] * np.ones(5), 1.5e-6)
    levels = rng.choice([0.9, 1.0, 1.1, 1.2], size=(n, 5))
    r = np.round(base * levels, 8)
    got = convergence_iteration(r, 8.0, floors)
    assert got == O.convergence_iteration(r, 8.0, floors)
    assert got[0] > 0
