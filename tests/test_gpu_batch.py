"""Batched cases on the GPU (autan_euler_device_set_cases and the batched march) against the
oracle: per-case RMS bit for bit, stopped cases unchanged while the others match their own runs,
and each case of a batched march converging at the iteration of its own march."""

import numpy as np
import pytest

import oracle as O
from autan_b200 import cases
from autan_b200 import mesh as M
from autan_b200.euler import EulerDevice

pytestmark = pytest.mark.gpu


def bits_equal(a, b):
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    return np.array_equal(a.view(np.int64), b.view(np.int64))


def small_batch(cells=(800, 3000), n=3, seed=2):
    return cases.bump_batch(n, seed=seed, cells=cells, precision="fp64", inlet="state")


def device_of(b):
    dev = EulerDevice(b.mesh, b.scheme, bc_kind=b.bc_kind, bc_data=b.bc_data, weights=b.weights)
    dev.set_cases(b.cell_offsets)
    dev.upload(b.u0)
    return dev


def case_oracle(b, k, scheme=None):
    """Case k alone: its own mesh, boundary data and oracle (with `scheme`, default the batch's)."""
    p = b.params[k]
    m = M.bump_channel(*p["boxes"], bump=p["bump"])
    first = sum(cases_b(b, j) for j in range(k))
    nb = m.n_boundary_faces
    kind = np.ascontiguousarray(b.bc_kind[first : first + nb])
    data = np.ascontiguousarray(b.bc_data[:, first : first + nb])
    c0, c1 = b.cell_offsets[k], b.cell_offsets[k + 1]
    u0 = np.ascontiguousarray(b.u0[:, c0:c1])
    sch = b.scheme if scheme is None else scheme
    md = cases.oracle_mesh_dict(cases.Case("k", m, sch, kind, data, u0, 3, 1.5, 1, True))
    return O.Oracle(md, sch.as_dict(), kind, data), u0


def cases_b(b, j):
    p = b.params[j]
    nx, ny, nz = p["boxes"]
    return M.bump_channel(nx, ny, nz, bump=p["bump"]).n_boundary_faces


def test_per_case_rms_bit_for_bit():
    b = small_batch()
    with device_of(b) as dev:
        dev.step(cfl=b.cfl, rk=3, n_steps=3, local=True)
        hist = dev.case_history(3)
    o = O.Oracle(b.mesh, b.scheme.as_dict(), b.bc_kind, b.bc_data)
    u = b.u0.copy()
    for s in range(3):
        res = o.residual(u)
        for k in range(3):
            c0, c1 = b.cell_offsets[k], b.cell_offsets[k + 1]
            rms = [np.sqrt(O.exact_sum(res[q, c0:c1] ** 2) / (c1 - c0)) for q in range(5)]
            assert bits_equal(hist[s, k], rms), (s, k)
        o.step(u, rk=3, cfl=b.cfl, local=True)


def test_stopped_case_is_unchanged_and_the_others_match_their_own_runs():
    b = small_batch()
    with device_of(b) as dev:
        dev.set_active([1, 0, 1])
        dev.step(cfl=b.cfl, rk=3, n_steps=5, local=True)
        u = dev.download()
    c0, c1 = b.cell_offsets[1], b.cell_offsets[2]
    assert bits_equal(u[:, c0:c1], b.u0[:, c0:c1])
    for k in (0, 2):
        o, uk = case_oracle(b, k)
        for _ in range(5):
            o.step(uk, rk=3, cfl=b.cfl, local=True)
        c0, c1 = b.cell_offsets[k], b.cell_offsets[k + 1]
        assert bits_equal(u[:, c0:c1], uk)


def test_batched_march_converges_each_case_at_its_own_iteration():
    b = small_batch(cells=(300, 1500), n=4, seed=5)
    with device_of(b) as dev:
        res = dev.march_cases(cfl=b.cfl, local=True, rk=3, max_steps=3000, batch=16, orders=2.0)
    assert res["converged"].all()
    for k in range(4):
        o, uk = case_oracle(b, k)
        norms = [o.step(uk, rk=3, cfl=b.cfl, local=True)[0] for _ in range(int(res["iterations"][k]))]
        it, _ = O.convergence_iteration(np.array(norms), 2.0)
        assert it == res["iterations"][k], (k, it, res["iterations"][k])


def test_per_case_cut_off_mach_numbers():
    """AUSM+-up with each case's own cut-off Mach number (Batch.open): every case steps bit for bit
    as its own run whose scheme has mach_ref = the case's Mach number."""
    import dataclasses

    b = cases.bump_batch(3, seed=2, cells=(800, 3000), precision="fp64", inlet="state", flux="ausm")
    assert len(set(b.mach_ref)) == 3
    with b.open() as dev:
        dev.upload(b.u0)
        dev.step(cfl=b.cfl, rk=3, n_steps=4, local=True)
        u = dev.download()
    for k in range(3):
        o, uk = case_oracle(b, k, dataclasses.replace(b.scheme, mach_ref=float(b.mach_ref[k])))
        for _ in range(4):
            o.step(uk, rk=3, cfl=b.cfl, local=True)
        c0, c1 = b.cell_offsets[k], b.cell_offsets[k + 1]
        assert bits_equal(u[:, c0:c1], uk), k


def test_per_case_cut_off_mach_numbers_are_checked():
    """One positive cut-off per case, and only after set_cases: anything else is refused with the
    library's error code, and the handle keeps working."""
    from autan_b200._native import NativeError

    b = small_batch()
    with EulerDevice(b.mesh, b.scheme, bc_kind=b.bc_kind, bc_data=b.bc_data, weights=b.weights) as dev:
        dev.n_cases = 3
        with pytest.raises(NativeError, match="E1101"):
            dev.set_case_mach_ref([0.5, 0.5, 0.5])  # no cases set yet
        dev.set_cases(b.cell_offsets)
        with pytest.raises(NativeError, match="E1101"):
            dev.set_case_mach_ref([0.5, 0.0, 0.5])
        with pytest.raises(ValueError):
            dev.set_case_mach_ref([0.5, 0.5])
        dev.set_case_mach_ref([0.4, 0.5, 0.6])
        dev.upload(b.u0)
        dev.step(cfl=b.cfl, rk=3, n_steps=2, local=True)
