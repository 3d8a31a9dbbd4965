"""Partitioned stepping of one mesh on the GPU: the ranks of a partition, each a stepper over its
local mesh in a thread of its own (ThreadRanks: host barriers between the ranks' streams, no
kernel waits on another), take the whole mesh's steps bit for bit: every owned cell's state, the
residual norms and the step of every step, and the least invalid cell. The exchange and
reductions are those a multi-GPU run makes through NCCL (TorchRanks), here between streams of one
GPU."""

import threading

import numpy as np
import pytest

from autan_b200 import cases as K
from autan_b200 import partition as PT
from autan_b200.euler import EulerDevice

pytestmark = pytest.mark.gpu


def perturbed(case, amplitude, seed):
    """The case's start with a seeded relative perturbation of every conserved value, so that
    every face and every stencil entry sees differences."""
    rng = np.random.default_rng(seed)
    u = case.u0 * (1.0 + amplitude * rng.uniform(-1.0, 1.0, case.u0.shape))
    m = case.mesh
    if m.n_cells > m.n_owned_cells:
        u[:, m.n_owned_cells :] = u[:, m.ghost_owner]
    return np.ascontiguousarray(u)


def whole(case, weights, u0, steps, dt=0.0, tuning=None):
    """The whole mesh on one stepper: the owned state after `steps` steps, the last step's result,
    the steps' norms and steps, and an evaluation of the final state."""
    with EulerDevice(case.mesh, case.scheme, case.bc_kind, case.bc_data, weights=weights) as d:
        if tuning:
            d.set_tuning(**tuning)
        d.upload(u0)
        r = d.step(case.cfl, dt, case.local, case.rk, steps)
        rms, hdt = d.history(steps)
        ev = d.evaluate()
        return d.download()[:, : case.mesh.n_owned_cells], r, rms, hdt, ev


def partitioned(case, weights, u0, parts, steps, dt=0.0, tuning=None):
    """The same on the ranks of `parts`, one thread each: the gathered owned state and, per
    rank, the result, norms, steps and evaluation."""
    ps = PT.extract_partitions(case.mesh, weights, parts)
    ranks = PT.ThreadRanks(len(ps), timeout=300)
    members = [PT.PartitionedEuler(p, case.scheme, ranks, case.bc_kind, case.bc_data) for p in ps]
    if tuning:
        for mb in members:
            mb.dev.set_tuning(**tuning)
    out, errors = [None] * len(ps), []

    def run(i):
        try:
            mb = members[i]
            mb.upload(u0)
            r = mb.step(case.cfl, dt, case.local, case.rk, steps)
            rms, hdt = mb.history(steps)
            ev = mb.evaluate()
            out[i] = (mb.download(), r, rms, hdt, ev)
        except BaseException as e:  # noqa: BLE001 (reported below)
            errors.append(e)
            ranks.barrier.abort()

    threads = [threading.Thread(target=run, args=(i,)) for i in range(len(ps))]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=600)
    for mb in members:
        mb.close()
    assert not errors, errors
    state = PT.gather_state(ps, [o[0] for o in out], case.mesh.n_owned_cells)
    return state, [o[1:] for o in out], ps


def same_bits(a, b) -> bool:
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return a.shape == b.shape and np.array_equal(a.view(np.int64), b.view(np.int64))


def check_same(case, weights, u0, parts, steps, dt=0.0, tuning=None):
    ref_state, ref_r, ref_rms, ref_dt, ref_ev = whole(case, weights, u0, steps, dt, tuning)
    state, per_rank, ps = partitioned(case, weights, u0, parts, steps, dt, tuning)
    assert any(p.n_external > 0 for p in ps)
    assert same_bits(state, ref_state)
    for r, h, d, ev in per_rank:
        assert same_bits(h, ref_rms)
        assert same_bits(d, ref_dt)
        assert same_bits(r.residuals, ref_r.residuals)
        assert same_bits(r.time_step, ref_r.time_step)
        assert r.invalid_cell == ref_r.invalid_cell
        assert same_bits(ev.residuals, ref_ev.residuals)
    return ref_r, per_rank


CASES = {
    # config-3 channel: AUSM+-up, second order, local steps, inlet / outlet / slip
    "channel": lambda precision: K.bump_channel(24, 12, 4, precision=precision, steps=4),
    # config-2 vortex: HLLC, Venkatakrishnan, global CFL step, periodic images
    "tets": lambda precision: K.vortex_tets(12, 12, 3, steps=4, precision=precision,
                                            extent=(10.0, 10.0, 2.5)),  # fmt: skip
    # config-1 vortex: first-order Roe, classical RK4, periodic images
    "hex": lambda precision: K.vortex_hex(16, 16, 2, steps=4, precision=precision),
}


@pytest.mark.parametrize("precision", ["fp32+acc64", "fp64"])
@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("split", ["blocks3", "random2", "random4"])
def test_partitioned_steps_are_the_whole_mesh_bits(name, precision, split):
    case = CASES[name](precision)
    m = case.mesh
    weights = m.gradient_weights(case.bc_kind)
    u0 = perturbed(case, 1e-3, 5)
    steps = case.steps
    if split == "blocks3":
        parts = PT.partition_cells(m, 3)
    else:
        n = int(split[-1])
        rng = np.random.default_rng(11)
        parts = rng.integers(0, n, m.n_owned_cells).astype(np.int32)
        parts[:n] = np.arange(n)
    ref_r, _ = check_same(case, weights, u0, parts, steps)
    assert ref_r.invalid_cell is None


@pytest.mark.parametrize("tuning", [
    dict(face_mode=0),
    dict(face_mode=2),
    dict(grad_mode=4, grad_block=128, grad_chunk=2, grad_minb=7, grad_widen=2, grad_narrow=1),
    dict(grad_mode=5, grad_block=128, grad_chunk=2, grad_depth=4),
    dict(grad_mode=1, grad_block=128, grad_chunk=4),
    dict(grad_mode=3, grad_block=128, grad_chunk=4),
])
def test_partitioned_steps_under_each_launch_choice(tuning):
    case = CASES["channel"]("fp32+acc64")
    m = case.mesh
    weights = m.gradient_weights(case.bc_kind)
    check_same(case, weights, perturbed(case, 1e-3, 6), PT.partition_cells(m, 3), 3,
               tuning=tuning)  # fmt: skip


def test_partitioned_reports_the_least_global_invalid_cell():
    """A non-positive density planted in two cells of different ranks: every rank reports the
    least of them, as the whole mesh does (first_invalid_cell, euler_physics.cpp:1399-1435)."""
    case = CASES["tets"]("fp32+acc64")
    m = case.mesh
    weights = m.gradient_weights(case.bc_kind)
    parts = PT.partition_cells(m, 3)
    u0 = perturbed(case, 1e-3, 5)
    bad = [int(np.nonzero(parts == 2)[0][5]), int(np.nonzero(parts == 1)[0][9])]
    for c in bad:
        u0[0, c] = -1.0
    ref_r, per_rank = check_same(case, weights, u0, parts, 1, dt=1e-3)
    assert ref_r.invalid_cell is not None and ref_r.invalid_cell <= min(bad)
    for r, *_ in per_rank:
        assert r.invalid_cell == ref_r.invalid_cell


class _Failing:
    """A backend whose exchange fails (a peer that has gone): the step call fails with that error
    as its cause."""

    def join(self, member):
        return self

    def exchange(self, member, what, record_bytes, stream):
        raise ConnectionError("peer gone")

    def reduce(self, member, op, count, stream):
        pass

    def min_host(self, member, value):
        return value


def test_a_failed_exchange_fails_the_step_with_its_cause():
    case = CASES["channel"]("fp32+acc64")
    m = case.mesh
    weights = m.gradient_weights(case.bc_kind)
    (p,) = PT.extract_partitions(m, weights, PT.partition_cells(m, 2), ranks=[0])
    mb = PT.PartitionedEuler(p, case.scheme, _Failing(), case.bc_kind, case.bc_data)
    try:
        mb.upload(case.u0)
        with pytest.raises(RuntimeError) as info:
            mb.step(case.cfl, 0.0, case.local, case.rk, 1)
        assert isinstance(info.value.__cause__, ConnectionError)
        # entry points that would read stale ghosts are refused
        from autan_b200._native import NativeError

        with pytest.raises(NativeError, match="E1101"):
            mb.dev.residual(np.zeros((5, p.mesh["n_cells"])))
        with pytest.raises(NativeError, match="E1101"):
            mb.dev.face_parts()
        with pytest.raises(NativeError, match="E1101"):
            mb.dev.time_steps(case.cfl)
    finally:
        mb.close()


def test_a_mesh_with_external_ghosts_needs_its_ranks():
    case = CASES["channel"]("fp32+acc64")
    m = case.mesh
    weights = m.gradient_weights(case.bc_kind)
    (p,) = PT.extract_partitions(m, weights, PT.partition_cells(m, 2), ranks=[1])
    kind = case.bc_kind[p.bc_index]
    data = case.bc_data[:, p.bc_index]
    from autan_b200._native import NativeError

    with EulerDevice(p.mesh, case.scheme, kind, data, weights=p.weights) as d:
        d.upload(case.u0[:, p.cell_global])
        with pytest.raises(NativeError, match="E1101"):
            d.step(case.cfl, 0.0, case.local, case.rk, 1)


def test_partitioned_full_size_lattice():
    """The 2 073 600-cell tetrahedral vortex on four ranks: two steps, the whole mesh's bits (the
    ghost records' indices and the exchange buffers at a production size)."""
    case = K.vortex_tets(240, 240, 6, precision="fp32+acc64")
    m = case.mesh
    assert m.n_owned_cells == 2_073_600
    weights = m.gradient_weights(case.bc_kind)
    check_same(case, weights, case.u0, PT.partition_cells(m, 4), 2)


def _nccl_one_rank(port, out):
    import datetime
    import os

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    try:
        import torch
        import torch.distributed as dist

        torch.cuda.set_device(0)
        dist.init_process_group("nccl", rank=0, world_size=1,
                                timeout=datetime.timedelta(seconds=60))  # fmt: skip
        case = CASES["channel"]("fp32+acc64")
        m = case.mesh
        weights = m.gradient_weights(case.bc_kind)
        u0 = perturbed(case, 1e-3, 3)
        ref_state, ref_r, ref_rms, *_ = whole(case, weights, u0, 3)
        (p,) = PT.extract_partitions(m, weights, np.zeros(m.n_owned_cells, np.int32))
        mb = PT.PartitionedEuler(p, case.scheme, PT.TorchRanks(), case.bc_kind, case.bc_data)
        mb.upload(u0)
        r = mb.step(case.cfl, 0.0, case.local, case.rk, 3)
        rms, _ = mb.history(3)
        ok = same_bits(mb.download(), ref_state) and same_bits(rms, ref_rms)
        ok = ok and same_bits(r.residuals, ref_r.residuals)
        mb.close()
        dist.destroy_process_group()
        out.put("ok" if ok else "different bits")
    except BaseException as e:  # noqa: BLE001
        out.put(repr(e))


def test_torch_ranks_on_nccl_streams():
    """The NCCL backend's reductions on the stepper's stream (a group of one rank: the norms and
    the step pass through NCCL all-reduces between the step's launches)."""
    import multiprocessing as mp
    import socket

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    proc = ctx.Process(target=_nccl_one_rank, args=(port, out))
    proc.start()
    got = out.get(timeout=300)
    proc.join(timeout=60)
    assert got == "ok"
    assert proc.exitcode == 0


@pytest.mark.parametrize("bad", [False, True])
def test_partitioned_march_takes_the_whole_mesh_steps(bad):
    """A steady march to the convergence rule on three ranks: the same iterations, decision and
    final state as on the whole mesh (the rule reads the whole mesh's norms on every rank). With a
    non-positive density planted in one rank's cell, every rank stops after the first batch and
    reports the whole mesh's least invalid cell."""
    case = K.bump_channel(24, 12, 4, steps=1)
    m = case.mesh
    weights = m.gradient_weights(case.bc_kind)
    parts = PT.partition_cells(m, 3)
    u0 = case.u0.copy()
    if bad:
        u0[0, int(np.nonzero(parts == 2)[0][7])] = -1.0
    with EulerDevice(m, case.scheme, case.bc_kind, case.bc_data, weights=weights) as d:
        d.upload(u0)
        ref = d.march(case.cfl, 0.0, True, 3, max_steps=400, batch=50, orders=3.0)
        ref_state = d.download()[:, : m.n_owned_cells]
    assert (ref["invalid_cell"] is not None) == bad
    ps = PT.extract_partitions(m, weights, parts)
    ranks = PT.ThreadRanks(len(ps), timeout=300)
    members = [PT.PartitionedEuler(p, case.scheme, ranks, case.bc_kind, case.bc_data) for p in ps]
    out, errors = [None] * len(ps), []

    def run(i):
        try:
            members[i].upload(u0)
            r = members[i].march(case.cfl, 0.0, True, 3, max_steps=400, batch=50, orders=3.0)
            out[i] = (r, members[i].download())
        except BaseException as e:  # noqa: BLE001 (reported below)
            errors.append(e)
            ranks.barrier.abort()

    threads = [threading.Thread(target=run, args=(i,)) for i in range(len(ps))]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=600)
    for mb in members:
        mb.close()
    assert not errors, errors
    state = PT.gather_state(ps, [o[1] for o in out], m.n_owned_cells)
    assert same_bits(state, ref_state)
    for r, _ in out:
        assert (r["iterations"], r["steps"], r["converged"]) == (ref["iterations"], ref["steps"],
                                                                   ref["converged"])  # fmt: skip
        assert same_bits(r["last"], ref["last"])
        assert r["invalid_cell"] == ref["invalid_cell"]
