"""The CPU oracle against golden vectors evaluated from the reference's own kernels/euler.py bodies
(tests/golden/make_golden.py): bit for bit, every body, residual, spectral radius and step."""

from pathlib import Path

import numpy as np
import pytest

import oracle as O

GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = sorted(p.stem for p in GOLDEN.glob("*.npz") if p.stem != "bodies")

BASE = dict(gamma=1.4, gas_constant=287.0, venkat_k=5.0, length=1.0, mach_ref=0.4,
            scale=[1.0] * 5, reference=[1.0, 0.0, 0.0, 0.0, 2.5])  # fmt: skip


def _bits_equal(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return np.array_equal(a.view(np.int64), b.view(np.int64)) or np.array_equal(a, b)


@pytest.mark.parametrize("tag", ["f64", "f32"])
@pytest.mark.parametrize("flux", [0, 1, 2])
def test_flux_bodies(tag, flux):
    z = np.load(GOLDEN / "bodies.npz")
    name = ["roe", "hllc", "ausm"][flux]
    # make_golden calls the bodies with g = 1.4, M_co = 0.4 and the p_ref of the reference state
    # (1, 0, 0, 0, 2.5).
    s = dict(BASE, flux=flux, precision=int(tag == "f32"))
    wl, wr, n = z[f"flux_{tag}_wl"], z[f"flux_{tag}_wr"], z[f"flux_{tag}_n"]
    want = z[f"flux_{tag}_{name}"]
    got = np.stack([O.flux(s, wl[:, i], wr[:, i], n[:, i]) for i in range(wl.shape[1])], axis=1)
    assert _bits_equal(got, want), np.abs(got - want).max()


@pytest.mark.parametrize("tag", ["f64", "f32"])
def test_boundary_states(tag):
    z = np.load(GOLDEN / "bodies.npz")
    s = dict(BASE, precision=int(tag == "f32"))
    w, kind, data, n, want = (z[f"bv_{tag}_{k}"] for k in ("w", "kind", "data", "n", "out"))
    got = np.stack([O.boundary_value(s, w[:, i], kind[i], data[:, i], n[:, i])
                    for i in range(w.shape[1])], axis=1)  # fmt: skip
    assert _bits_equal(got, want), np.abs(got - want).max()


@pytest.mark.parametrize("tag", ["f64", "f32"])
def test_primitives(tag):
    z = np.load(GOLDEN / "bodies.npz")
    s = dict(BASE, precision=int(tag == "f32"),
             reference=[1.2, 0.36, -0.24, 0.12, 1.0 / 0.4 + 0.5 * 1.2 * 0.14])  # fmt: skip
    dq, want = z[f"prim_{tag}_dq"], z[f"prim_{tag}_out"]
    got = np.stack([O.to_primitive(s, dq[:, i]) for i in range(dq.shape[1])], axis=1)
    assert _bits_equal(got, want), np.abs(got - want).max()


@pytest.mark.parametrize("case", CASES)
def test_residual(case):
    mesh, scheme, z = O.load_case(GOLDEN / f"{case}.npz")
    o = O.Oracle(mesh, scheme, z["bc_kind"], z["bc"], z["source"])
    res = o.residual(z["u"])
    no = mesh["n_owned_cells"]
    arrays = o.arrays()
    for k in ("prim", "grad", "phi", "wmin", "wmax"):
        assert _bits_equal(arrays[k][:, :no], z[k][:, :no]), k
    assert _bits_equal(arrays["prim_b"][:, mesh["n_interior_faces"]:],
                       z["prim_b"][:, mesh["n_interior_faces"]:])  # fmt: skip
    assert _bits_equal(res[:, :no], z["res"][:, :no]), np.abs(res - z["res"])[:, :no].max()
    lam = o.spectral_radius()
    assert _bits_equal(lam[:no], z["lam"][:no])


STEP_CASES = [c for c in CASES if "step3_u" in np.load(GOLDEN / f"{c}.npz").files]


@pytest.mark.parametrize("case", STEP_CASES)
@pytest.mark.parametrize("rk", [3, 4])
def test_step(case, rk):
    mesh, scheme, z = O.load_case(GOLDEN / f"{case}.npz")
    o = O.Oracle(mesh, scheme, z["bc_kind"], z["bc"], z["source"])
    u = np.ascontiguousarray(z["u"].copy())
    norms, dt, bad = o.step(u, rk=rk, cfl=0.5)
    no = mesh["n_owned_cells"]
    assert bad == -1
    assert dt == float(z[f"step{rk}_dt"])
    assert _bits_equal(norms, z[f"step{rk}_norms"])
    assert _bits_equal(u[:, :no], z[f"step{rk}_u"][:, :no])


def test_exact_sum_is_correctly_rounded():
    import math

    rng = np.random.default_rng(5)
    for scale in (1e-300, 1e-8, 1.0, 1e200):
        t = rng.standard_normal(2000) * scale * np.exp(rng.uniform(-30, 30, 2000))
        assert O.exact_sum(t) == math.fsum(t)
        assert O.exact_sum(t[::-1]) == math.fsum(t)
    assert O.exact_sum(np.array([1.0, 1e100, 1.0, -1e100])) == 2.0
    assert math.isnan(O.exact_sum(np.array([1.0, np.inf, -np.inf])))
    assert O.exact_sum(np.array([np.inf, 1.0])) == np.inf
    assert O.exact_sum(np.array([5e-324, 5e-324])) == 1e-323
