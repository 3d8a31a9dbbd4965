"""Known answers of the reference's own tests for the residual, restated on the CPU oracle (which
the CUDA path equals bit for bit on the golden cases, tests/test_gpu_parity.py): the planar loops
equal the full loops on a planar mesh (tests/physics/test_euler.cpp:277), a uniform flow is a
steady state to round-off (tests/physics/test_euler.cpp:158-240, the freestream-preservation gate
of docs/validation/acceptance.md:27), and the convected vortex converges at second order (the
vortex-order gate, 2 +- 0.1, docs/validation/acceptance.md:30)."""

import dataclasses

import numpy as np
import pytest

import oracle as O
from autan_b200 import cases


def bits_equal(a, b):
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    return np.array_equal(a.view(np.int64), b.view(np.int64))


@pytest.mark.parametrize("precision", ["fp64", "fp32+acc64"])
def test_planar_loops_equal_the_full_loops(precision):
    """On tetrahedra (every face planar, every face moment zero) the planar loops, which skip the
    warped-face terms, give the residual of the full loops: the terms they skip are exact zeros."""
    case = cases.vortex_tets(16, 16, 6, precision=precision)
    assert case.mesh.all_planar
    md = cases.oracle_mesh_dict(case)
    out = {}
    for planar in (True, False):
        sch = dataclasses.replace(case.scheme, planar=planar).as_dict()
        out[planar] = O.Oracle(md, sch, case.bc_kind, case.bc_data).residual(case.u0)
    no = case.mesh.n_owned_cells
    assert np.array_equal(out[True][:, :no], out[False][:, :no])


@pytest.mark.parametrize("precision", ["fp64", "fp32+acc64"])
def test_uniform_flow_is_steady(precision):
    """A uniform freestream on the jittered periodic tetrahedra (slip walls across it) is a steady
    state to round-off: every |R| <= 64 eps (|F| A) per cell, eps of the compute type (the bound
    of the GPU test at full size in fp64); in fp32+acc64 the fluxes, normals and areas are floats,
    whose faces do not close exactly, so the residual is of FP32 size."""
    case = cases.vortex_tets(24, 24, 6, precision=precision)
    u = np.repeat(np.array(cases.freestream_reference())[:, None], case.mesh.n_cells, axis=1)
    o = O.Oracle(cases.oracle_mesh_dict(case), case.scheme.as_dict(), case.bc_kind, case.bc_data)
    res = o.residual(u)
    no = case.mesh.n_owned_cells
    scale = 3.5 * 2.0 * case.mesh.face_area_magnitude.max() * 6
    eps = np.finfo(np.float64 if precision == "fp64" else np.float32).eps
    assert np.abs(res[:, :no]).max() <= 64 * eps * scale


def vortex_density_error(n, t_end=1.0):
    """L1 error (volume-weighted) of the density of the jittered-tet vortex (h = 10 / n, two cell
    layers across, the benchmark's scheme in fp64) after SSP-RK3 steps at CFL 0.8 to t_end, the
    last step shortened to land on it, against the exact vortex translated by the freestream."""
    h = 10.0 / n
    case = cases.vortex_tets(n, n, 2, precision="fp64", extent=(10.0, 10.0, 2 * h))
    o = O.Oracle(cases.oracle_mesh_dict(case), case.scheme.as_dict(), case.bc_kind, case.bc_data)
    u = case.u0.copy()
    t = 0.0
    while t_end - t > 1e-12:
        _, dt, bad = o.step(u, rk=3, cfl=0.8)
        assert bad < 0
        t += dt
        if 1e-12 < t_end - t < dt:
            o.step(u, rk=3, cfl=0.8, dt=t_end - t)
            t = t_end
    m = case.mesh
    no = m.n_owned_cells
    centre = ((5.0 + cases.FREESTREAM[1] * t_end) % 10.0, (5.0 + cases.FREESTREAM[2] * t_end) % 10.0)
    exact = cases.isentropic_vortex(m, centre=centre)
    vol = m.cell_volume[:no]
    return np.sum(np.abs(u[0, :no] - exact[0, :no]) * vol) / vol.sum()


def test_vortex_converges_at_second_order():
    """Lattices of 24 and 48 boxes a side (6 912 and 27 648 tetrahedra): the observed order of the
    density error is 2 +- 0.1 (2.06 here; 1.92 from 48 to 96 boxes, too slow for this suite)."""
    order = np.log2(vortex_density_error(24) / vortex_density_error(48))
    assert abs(order - 2.0) <= 0.1, order
