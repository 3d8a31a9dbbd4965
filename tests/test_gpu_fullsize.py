"""The CUDA path against the CPU oracle at the benchmark configurations' full sizes (the sizes the
index arithmetic and the layouts meet in production):
- the 2 073 600-cell jittered tetrahedral vortex (HLLC, SSP-RK3, CFL 0.8): 3 steps, fp64 and
  fp32+acc64, state, residual norms and time steps bit for bit; fp32+acc64 against the FP64 oracle
  within 2e-6 of the state's largest magnitude;
- the 8 002 500-cell hybrid bump channel (AUSM+-up, total-pressure inlet, local steps, CFL 1.5,
  fp32+acc64): one step; the inlet's boundary states take exp and log, where CUDA's and the C
  library's FP32 results may differ in the last place, so the bound is 1e-5 of each component's
  largest magnitude (the momenta: the largest momentum), and at least 95 % of the cells bit for
  bit;
- 16 cases of the batched channels at their real sizes (cells log-uniform in [20 000, 500 000],
  seed 0, Roe, farfield inflow and outflow, fp32+acc64): 2 batched steps against the oracle on
  the union mesh, 1e-5 of each case's component magnitudes (the farfield states take exp and log).
Oracle runs here take tens of seconds each (one host thread)."""

import numpy as np
import pytest

import oracle as O
from autan_b200 import cases
from autan_b200.euler import EulerDevice

pytestmark = pytest.mark.gpu


def same_bits(a, b):
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    return np.array_equal(a.view(np.uint64), b.view(np.uint64))


def component_rel(a, b):
    """Largest difference of each conserved component relative to its scale in b: density and
    energy their own largest magnitude, the three momenta the largest momentum magnitude (a
    momentum component that is about zero, as z in an extruded channel, has no scale of its own)."""
    mom = max(np.abs(b[1:4]).max(), 1e-300)
    scale = [max(np.abs(b[0]).max(), 1e-300), mom, mom, mom, max(np.abs(b[4]).max(), 1e-300)]
    return np.array([np.abs(a[k] - b[k]).max() / scale[k] for k in range(5)])


def march_device(mesh, scheme, kind, data, u0, steps, cfl, local, cell_offsets=None, weights=None):
    with EulerDevice(mesh, scheme, kind, data, weights=weights) as dev:
        if cell_offsets is not None:
            dev.set_cases(cell_offsets)
        dev.upload(u0)
        r = dev.step(cfl=cfl, rk=3, n_steps=steps, local=local)
        rms, dts = dev.history(steps)
        return dev.download(), r, rms, dts


def march_oracle(md, scheme, kind, data, u0, steps, cfl, local, precision=None):
    s = scheme.as_dict()
    if precision is not None:
        s["precision"] = precision
    o = O.Oracle(md, s, kind, data)
    u = u0.copy()
    norms, dts, bad = [], [], -1
    for _ in range(steps):
        n, dt, bad = o.step(u, rk=3, cfl=cfl, local=local)
        norms.append(n)
        dts.append(dt)
    return u, np.array(norms), np.array(dts), bad


@pytest.mark.parametrize("precision", ["fp64", "fp32+acc64"])
def test_tetrahedral_vortex_full_lattice(precision):
    case = cases.vortex_tets(240, 240, 6, precision=precision)
    assert case.mesh.n_owned_cells == 2_073_600
    steps = 3
    u_d, r, rms_d, dt_d = march_device(case.mesh, case.scheme, case.bc_kind, case.bc_data, case.u0,
                                       steps, case.cfl, False)  # fmt: skip
    md = cases.oracle_mesh_dict(case)
    u_o, rms_o, dt_o, bad = march_oracle(md, case.scheme, case.bc_kind, case.bc_data, case.u0,
                                         steps, case.cfl, False)  # fmt: skip
    no = case.mesh.n_owned_cells
    assert r.invalid_cell is None and bad == -1
    assert same_bits(u_d[:, :no], u_o[:, :no])
    assert same_bits(rms_d, rms_o)
    assert same_bits(dt_d, dt_o)
    if precision != "fp64":
        u_64, *_ = march_oracle(md, case.scheme, case.bc_kind, case.bc_data, case.u0, steps,
                                case.cfl, False, precision=0)  # fmt: skip
        err = np.abs(u_d[:, :no] - u_64[:, :no]).max() / np.abs(u_64[:, :no]).max()
        print(f"fp32+acc64 vs the FP64 oracle after {steps} steps: {err:.3e}")
        assert err <= 2e-6


def test_bump_channel_full_size_one_step():
    case = cases.bump_channel(480, 150, 100)
    assert case.mesh.n_owned_cells == 8_002_500
    u_d, r, rms_d, dt_d = march_device(case.mesh, case.scheme, case.bc_kind, case.bc_data, case.u0,
                                       1, case.cfl, True)  # fmt: skip
    md = cases.oracle_mesh_dict(case)
    u_o, rms_o, dt_o, bad = march_oracle(md, case.scheme, case.bc_kind, case.bc_data, case.u0, 1,
                                         case.cfl, True)  # fmt: skip
    no = case.mesh.n_owned_cells
    assert r.invalid_cell is None and bad == -1
    rel = component_rel(u_d[:, :no], u_o[:, :no])
    print("channel, one step, per-component difference:", rel)
    assert rel.max() <= 1e-5
    same = np.all(u_d[:, :no].view(np.uint64) == u_o[:, :no].view(np.uint64), axis=0)
    print(f"cells bit for bit: {same.mean():.6f}")
    assert same.mean() >= 0.95
    assert np.allclose(rms_d, rms_o, rtol=1e-5, atol=0)


def test_batched_channels_at_real_sizes():
    b = cases.bump_batch(256, seed=0, cells=(20_000, 500_000), select=list(range(16)))
    cells = np.diff(b.cell_offsets)
    assert cells.min() >= 15_000 and cells.max() <= 600_000 and len(cells) == 16
    steps = 2
    u_d, r, *_ = march_device(b.mesh, b.scheme, b.bc_kind, b.bc_data, b.u0, steps, b.cfl, True,
                              cell_offsets=b.cell_offsets, weights=b.weights)  # fmt: skip
    u_o, _, _, bad = march_oracle(b.mesh, b.scheme, b.bc_kind, b.bc_data, b.u0, steps, b.cfl, True)
    assert r.invalid_cell is None and bad == -1
    for k in range(16):
        c0, c1 = b.cell_offsets[k], b.cell_offsets[k + 1]
        rel = component_rel(u_d[:, c0:c1], u_o[:, c0:c1])
        assert rel.max() <= 1e-5, (k, rel)
    # every inflow and outflow face takes exp and log here, and small cases are few cells long, so
    # the cells that the last-place differences reach after 2 steps are a larger share
    same = np.all(u_d.view(np.uint64) == u_o.view(np.uint64), axis=0)
    print(f"batched cells bit for bit: {same.mean():.6f}")
    assert same.mean() >= 0.5
