"""Failure detection on the GPU, without faulting it.

- Divergence (CudaStepper::invalid, physics/src/device_stepper.cuh:107-164, and the host's
  first_invalid_cell, physics/src/euler_physics.cpp:1399-1435): a state with a NaN, a non-positive
  density and a non-positive pressure planted at chosen cells, in the host input. evaluate() and
  step() report the least invalid cell, as the oracle does (the reference's test
  tests/physics/test_euler_device.cpp:295 checks the least cell whatever the numbering); the
  handle then steps a valid state bit for bit as the oracle.
- A bounded device wait that runs out: the test hook makes every warp of the TMA-ring gradient
  kernel wait a few polls on a barrier that nothing arrives on. The step call returns E1201, and
  the same handle then steps bit for bit as the oracle.
- The same for the warm-start MLP's fused tcgen05 kernel: gradient, predict and train return
  E1201 and leave the parameters as they were; with the hook off the same handle gives the bits
  of a fresh network."""

import numpy as np
import pytest

import oracle as O
from autan_b200 import cases
from autan_b200._native import NativeError
from autan_b200.euler import EulerDevice
from autan_b200.warmstart import MLP

pytestmark = pytest.mark.gpu


def same_bits(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint64), np.ascontiguousarray(b).view(np.uint64))


def oracle_of(case):
    return O.Oracle(cases.oracle_mesh_dict(case), case.scheme.as_dict(), case.bc_kind, case.bc_data)


def planted(case, plants):
    """u0 with each (cell, kind) planted: "nan" density, "rho" density -1e-3, "p" energy that
    leaves the pressure negative (internal energy removed), at the cell and its periodic images."""
    u = case.u0.copy()
    m = case.mesh
    ghosts = m.ghost_owner if m.n_cells > m.n_owned_cells else np.zeros(0, dtype=np.int32)
    for c, kind in plants:
        cells = [c] + [m.n_owned_cells + g for g in np.nonzero(ghosts == c)[0]]
        for x in cells:
            if kind == "nan":
                u[0, x] = np.nan
            elif kind == "rho":
                u[0, x] = -1e-3
            else:
                kinetic = 0.5 * (u[1, x] ** 2 + u[2, x] ** 2 + u[3, x] ** 2) / u[0, x]
                u[4, x] = kinetic - 0.1
    return u


@pytest.mark.parametrize("precision", ["fp64", "fp32+acc64"])
@pytest.mark.parametrize("plants", [[(911, "nan"), (407, "p")], [(1500, "rho")],
                                    [(2000, "p"), (63, "nan"), (1200, "rho")]])
def test_least_invalid_cell_is_reported(precision, plants):
    case = cases.vortex_tets(16, 16, 6, precision=precision)
    no = case.mesh.n_owned_cells
    u = planted(case, plants)
    o = oracle_of(case)
    want_eval = o.first_invalid(u, o.residual(u))
    assert want_eval == min(c for c, _ in plants)
    u_o = u.copy()
    _, _, want_step = o.step(u_o, rk=3, cfl=case.cfl)
    with EulerDevice(case.mesh, case.scheme, case.bc_kind, case.bc_data) as dev:
        dev.upload(u)
        assert dev.evaluate().invalid_cell == want_eval
        r = dev.step(cfl=case.cfl, rk=3, n_steps=1)
        assert r.invalid_cell == want_step
        # the same handle, a valid state: bit for bit as the oracle
        dev.upload(case.u0)
        r = dev.step(cfl=case.cfl, rk=3, n_steps=2)
        u_d = dev.download()
    u_v = case.u0.copy()
    for _ in range(2):
        _, _, bad = o.step(u_v, rk=3, cfl=case.cfl)
    assert r.invalid_cell is None and bad == -1
    assert same_bits(u_d[:, :no], u_v[:, :no])


def test_bounded_wait_runs_out_and_the_handle_recovers():
    case = cases.vortex_tets(24, 24, 6, precision="fp32+acc64")
    no = case.mesh.n_owned_cells
    with EulerDevice(case.mesh, case.scheme, case.bc_kind, case.bc_data) as dev:
        dev.set_tuning(grad_mode=5, grad_chunk=2, grad_block=128, grad_depth=4, grad_narrow=0)
        dev.upload(case.u0)
        dev.set_stall_test(16)
        for graph in (False, True):
            with pytest.raises(NativeError, match="E1201"):
                dev.step(cfl=case.cfl, rk=3, n_steps=1, graph=graph)
        dev.set_stall_test(0)
        dev.upload(case.u0)
        r = dev.step(cfl=case.cfl, rk=3, n_steps=3)
        u_d = dev.download()
    o = oracle_of(case)
    u_o = case.u0.copy()
    for _ in range(3):
        _, _, bad = o.step(u_o, rk=3, cfl=case.cfl)
    assert r.invalid_cell is None and bad == -1
    assert same_bits(u_d[:, :no], u_o[:, :no])


def test_mlp_bounded_wait_runs_out_and_the_handle_recovers():
    rng = np.random.default_rng(13)
    x = rng.normal(size=(2000, 7)).astype(np.float32)
    y = rng.normal(size=(2000, 5)).astype(np.float32)
    sc = (x.mean(0), x.std(0), y.mean(0), y.std(0))
    ref = MLP(seed=14)
    ref.set_scaling(*sc)
    loss0, g0 = ref.gradient(x, y)
    net = MLP(seed=14)
    net.set_scaling(*sc)
    net.set_data(x, y)
    net.set_stall_test(16)
    with pytest.raises(NativeError, match="E1201"):
        net.gradient(x, y)
    with pytest.raises(NativeError, match="E1201"):
        net.predict(x)
    with pytest.raises(NativeError, match="E1201"):
        net.train(epochs=1, batch=1024, lr=1e-3, seed=1)
    assert np.array_equal(net.parameters(), ref.parameters())  # no update was applied
    net.set_stall_test(0)
    loss1, g1 = net.gradient(x, y)
    assert loss1 == loss0 and np.array_equal(g1, g0)
    net.close()
    ref.close()
