"""Discrete conservation and the boundary pressure force on the oracle (CPU), on the golden meshes:
each cell's face part R^F is its faces' written fluxes summed in its face order, bit for bit (the
assumption of the reference's conservation gate, docs/validation/acceptance.md, D2 gate 7); the
gate's ratio q_k = |sum R^F - sum F_b| / D_k stays within tau = max(64 2^-52, 2 gamma_(d+2));
Euler<P>::boundary_pressure of a uniform state is that state's pressure, its force p S."""

import math
from pathlib import Path

import numpy as np
import pytest

import oracle as O

GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = sorted(p.stem for p in GOLDEN.glob("*.npz") if p.stem != "bodies")


def tau(max_faces: int) -> float:
    """The bound of D2 gate 7 (tools/gate7.py): max(64 2^-52, 2 gamma_(d+2)), gamma_m = m u /
    (1 - m u), u = 2^-53."""
    u = 2.0**-53
    m = max_faces + 2
    return max(64 * 2.0**-52, 2 * m * u / (1 - m * u))


def oracle_of(case):
    mesh, scheme, z = O.load_case(GOLDEN / f"{case}.npz")
    o = O.Oracle(mesh, scheme, z["bc_kind"], z["bc"], z["source"])
    return o, mesh, scheme, z


def max_faces(mesh) -> int:
    off = mesh["cell_face_offsets"]
    n = mesh["n_owned_cells"]
    return int(np.diff(off[: n + 1]).max())


@pytest.mark.parametrize("case", CASES)
def test_face_parts_sum_each_cells_written_fluxes(case):
    o, mesh, _, z = oracle_of(case)
    rf, ff = o.face_parts(z["u"])
    n, ni = mesh["n_owned_cells"], mesh["n_interior_faces"]
    owner = mesh["owner"]
    off, cf = mesh["cell_face_offsets"], mesh["cell_faces"]
    want = np.zeros((5, n))
    for c in range(n):
        acc = [0.0] * 5
        for f in cf[off[c] : off[c + 1]]:
            sign = 1.0 if (f >= ni or owner[f] == c) else -1.0
            for k in range(5):
                acc[k] = acc[k] + sign * ff[k, f] if sign > 0 else acc[k] - ff[k, f]
        want[:, c] = acc
    assert np.array_equal(rf[:, :n].view(np.int64), want.view(np.int64))


@pytest.mark.parametrize("case", CASES)
def test_conservation_within_gate_bound(case):
    o, mesh, scheme, z = oracle_of(case)
    rf, ff = o.face_parts(z["u"])
    sums = O.conservation_sums(mesh, rf, ff)
    E, D = sums[0], sums[1]
    t = tau(max_faces(mesh))
    assert np.all(np.isfinite(sums)) and np.all(D >= 0)
    if mesh["n_cells"] > mesh["n_owned_cells"] and scheme["second_order"]:
        # A periodic mesh holds each face across the period twice, once from each side, from
        # translated geometry: the two fluxes need not cancel bit for bit, which the reference's
        # gate counts as a flux mismatch and voids (euler_physics.cpp:1780-1800).
        pytest.skip("periodic images: interface fluxes evaluated twice (the gate voids the case)")
    for k in range(5):
        if D[k] == 0:
            assert E[k] == 0
        else:
            assert abs(E[k]) / D[k] <= t, (k, E[k], D[k], t)
    # faces - boundary = E exactly up to the one rounding of each sum
    assert np.all(np.abs(sums[3] - sums[2] - E) <= 4 * np.spacing(np.abs(sums[3]) + np.abs(sums[2])))


@pytest.mark.parametrize("case", CASES)
def test_boundary_pressure_of_a_uniform_state(case):
    o, mesh, scheme, z = oracle_of(case)
    nc = mesh["n_cells"]
    rho, vel, p = 1.1, (0.3, -0.2, 0.1), 0.9
    g = scheme["gamma"]
    e = p / (g - 1) + 0.5 * rho * sum(v * v for v in vel)
    u = np.tile(np.array([rho, rho * vel[0], rho * vel[1], rho * vel[2], e])[:, None], (1, nc))
    o.residual(u)
    pf, force = o.boundary_pressure()
    arr = o.arrays()
    # the stored pressure (p_ref + gauge), in FP64, identical on every face: no gradient
    ref = np.asarray(scheme["reference"])
    p_ref = (g - 1.0) * (ref[4] - 0.5 * (ref[1] ** 2 + ref[2] ** 2 + ref[3] ** 2) / ref[0])
    stored = p_ref + arr["prim"][4, 0]
    ni, nf = mesh["n_interior_faces"], mesh["n_faces"]
    # Faces whose owner sees no density or pressure gradient (boundary states of other kinds
    # enter the stencils of the cells next to them): p_f is the stored pressure, the force p S.
    owner = mesh["owner"][ni:]
    flat = np.all(arr["grad"][[0, 1, 2, 12, 13, 14]][:, owner] == 0.0, axis=0)
    if not flat.any():
        pytest.skip("every boundary face's owner sees a boundary state in its stencil")
    assert np.all(pf[flat] == stored)
    nrm = mesh["face_normal"].reshape(3, nf)[:, ni:]
    area = mesh["face_area_magnitude"][ni:]
    if scheme["precision"] == 1:
        nrm, area = nrm.astype(np.float32).astype(np.float64), area.astype(np.float32).astype(np.float64)
    assert np.array_equal(force[:, flat], (stored * (nrm * area))[:, flat])
