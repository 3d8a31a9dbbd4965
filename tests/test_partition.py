"""Partitioned meshes on CPU: every rank's local mesh restates its owned cells' loops of the
global mesh entry for entry (the same faces, orientation, stencil entries, weights and geometry,
in the same order), the halo plan delivers each external ghost its owning rank's record, and the
exchange and reductions of the torch.distributed backend do so over two gloo ranks (the NCCL
path's host logic)."""

import datetime
import multiprocessing as mp
import os
import socket
import sys
import threading
from pathlib import Path

import numpy as np
import pytest

from autan_b200 import mesh as M
from autan_b200 import partition as PT

REPO = Path(__file__).resolve().parent.parent


def meshes():
    return [
        ("channel", M.bump_channel(24, 12, 4)),
        ("tets", M.jittered_tets(8, 8, 2, extent=(1.0, 1.0, 0.25))),
        ("hex", M.periodic_box_hex(8, 8, 2)),
    ]


def random_parts(m, n_parts, seed):
    rng = np.random.default_rng(seed)
    parts = rng.integers(0, n_parts, m.n_owned_cells).astype(np.int32)
    parts[:n_parts] = np.arange(n_parts)  # none empty
    return parts


def check_partition(m, w, p):
    L = p.mesh
    cg, fg = p.cell_global, p.face_global
    no, ni_l = p.n_owned, L["n_interior_faces"]
    home = np.concatenate((np.arange(m.n_owned_cells), m.ghost_owner))
    # owned cells in global order, every one owned by this rank
    assert np.all(np.diff(cg[:no]) > 0)
    # faces: geometry and orientation of the global faces
    assert np.array_equal(cg[L["owner"]], m.owner[fg])
    assert np.array_equal(cg[L["neighbour"]], m.neighbour[fg[:ni_l]])
    assert np.array_equal(L["face_normal"], m.face_normal[:, fg])
    assert np.array_equal(L["face_centroid"], m.face_centroid[:, fg])
    assert np.array_equal(L["face_area_magnitude"], m.face_area_magnitude[fg])
    assert np.array_equal(L["cell_centroid"], m.cell_centroid[:, cg])
    assert np.all(fg[:ni_l] < m.n_owned_interior_faces)
    assert np.all(fg[ni_l:] >= m.n_interior_faces)
    # each owned cell: its faces and stencil entries, in the global order
    cfo, so = L["cell_face_offsets"], L["stencil_offsets"]
    gcfo, gso = m.cell_face_offsets, m.stencil_offsets
    for c in range(no):
        g = cg[c]
        lf = L["cell_faces"][cfo[c] : cfo[c + 1]]
        assert np.array_equal(fg[lf], m.cell_faces[gcfo[g] : gcfo[g + 1]])
        assert np.all(np.diff(lf) > 0)
        ls = L["stencil"][so[c] : so[c + 1]]
        gs = m.stencil[gso[g] : gso[g + 1]]
        back = np.where(ls >= 0, cg[np.maximum(ls, 0)], -(fg[np.maximum(-ls - 1, 0)] + 1))
        assert np.array_equal(back, gs)
        assert np.array_equal(p.weights[:, so[c] : so[c + 1]], w[:, gso[g] : gso[g + 1]])
    # ghosts: external first, by source rank then global cell; images of this rank's cells after
    gown = L["ghost_owner"]
    assert np.all(gown[: p.n_external] == -1)
    assert np.all(gown[p.n_external :] >= 0) and np.all(gown[p.n_external :] < no)
    assert np.array_equal(cg[gown[p.n_external :]], home[cg[no + p.n_external :]])
    return home


@pytest.mark.parametrize("how", ["blocks", "random"])
@pytest.mark.parametrize("n_parts", [2, 3, 5])
def test_local_meshes_restate_the_global_loops(how, n_parts):
    for name, m in meshes():
        w = m.gradient_weights(np.full(m.n_boundary_faces, M.BC_SLIP, np.uint8))
        parts = PT.partition_cells(m, n_parts) if how == "blocks" else random_parts(m, n_parts, 7)
        ps = PT.extract_partitions(m, w, parts)
        assert sum(p.n_owned for p in ps) == m.n_owned_cells
        owned = np.concatenate([p.cell_global[: p.n_owned] for p in ps])
        assert np.array_equal(np.sort(owned), np.arange(m.n_owned_cells))
        for p in ps:
            home = check_partition(m, w, p)
            ext = p.cell_global[p.n_owned : p.n_owned + p.n_external]
            r = parts[home[ext]]
            assert np.all(r != p.rank)
            assert np.all(np.diff(r) >= 0)  # grouped by source rank
            assert np.array_equal(np.bincount(r, minlength=n_parts), p.recv_counts)
        # the halo plan: what each rank sends is what its receivers' ghosts hold
        for q in ps:
            got = []
            for r in ps:
                first = int(r.send_counts[: q.rank].sum())
                cells = r.send_cells[first : first + int(r.send_counts[q.rank])]
                assert int(q.recv_counts[r.rank]) == cells.size
                got.append(r.cell_global[cells])
            ext = q.cell_global[q.n_owned : q.n_owned + q.n_external]
            home = np.concatenate((np.arange(m.n_owned_cells), m.ghost_owner))
            assert np.array_equal(np.concatenate(got), home[ext]), name


def test_blocks_balance_the_face_cost():
    m = M.bump_channel(48, 24, 4)
    parts = PT.partition_cells(m, 4)
    cost = PT.cell_cost(m)
    share = np.array([cost[parts == r].sum() for r in range(4)]) / cost.sum()
    assert np.all(np.abs(share - 0.25) < 0.01)
    assert np.all(np.diff(parts) >= 0)


class _Member:
    """One rank's exchange buffers on the host, standing in for a stepper."""

    def __init__(self, part):
        self.part = part
        self.buf = PT._Buffers(part, 4, "cpu")


def _fill_and_check(member, ranks, m, record_bytes, stream=None):
    """Pack each sent cell's global home id into its record, exchange, and check every external
    ghost's record; then a sum and a min of the words over the ranks."""
    import torch

    p = member.part
    home = np.concatenate((np.arange(m.n_owned_cells), m.ghost_owner))
    rows = member.buf.send_rows(int(p.send_cells.size), record_bytes)
    ids = p.cell_global[p.send_cells].astype(np.int64)
    rec = np.zeros((ids.size, record_bytes // 8), dtype=np.int64)
    rec[:, 0] = ids
    rec[:, -1] = p.rank
    rows.copy_(torch.from_numpy(rec.view(np.uint8).reshape(ids.size, record_bytes)))
    ranks.exchange(member, 0, record_bytes, stream)
    got = member.buf.recv_rows(p.n_external, record_bytes).numpy().copy().view(np.int64)
    ext = p.cell_global[p.n_owned : p.n_owned + p.n_external]
    assert np.array_equal(got[:, 0], home[ext])
    member.buf.words[:5].copy_(torch.tensor([p.rank + 1, -1, 2**62, 7 * p.rank, 3 - p.rank]))
    ranks.reduce(member, 0, 5, stream)
    n = p.n_parts
    want = [n * (n + 1) // 2, -n, (n * 2**62 + 2**63) % 2**64 - 2**63, 7 * n * (n - 1) // 2,
            sum(3 - r for r in range(n))]  # fmt: skip
    assert member.buf.words[:5].tolist() == want
    member.buf.words[:2].copy_(torch.tensor([10 + p.rank, 4 - p.rank]))
    ranks.reduce(member, 1, 2, stream)
    assert member.buf.words[:2].tolist() == [10, 4 - (n - 1)]
    assert ranks.min_host(member, 100 - p.rank) == 100 - (n - 1)


@pytest.mark.parametrize("record_bytes", [32, 96])
def test_thread_ranks_exchange_and_reduce_on_host(record_bytes):
    m = M.jittered_tets(8, 8, 2, extent=(1.0, 1.0, 0.25))
    ps = PT.extract_partitions(m, None, random_parts(m, 3, 1))
    ranks = PT.ThreadRanks(3, timeout=60)
    members = [_Member(p) for p in ps]
    for mb in members:
        ranks.join(mb)
    errors = []

    def run(mb):
        try:
            _fill_and_check(mb, ranks, m, record_bytes)
        except BaseException as e:  # noqa: BLE001 (reported below)
            errors.append(e)
            ranks.barrier.abort()

    threads = [threading.Thread(target=run, args=(mb,)) for mb in members]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=120)
    assert not errors, errors


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _torch_rank(rank: int, world: int, port: int, out) -> None:
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, str(REPO))
    import torch.distributed as dist

    from autan_b200 import mesh as M2
    from autan_b200 import partition as PT2

    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))  # fmt: skip
    try:
        m = M2.bump_channel(24, 12, 4)
        parts = random_parts(m, world, 3)
        # this rank's share alone, its send lists from the other rank's requests over the group,
        # equal to the ones one process derives from every rank's ghosts
        p = PT2.extract_partition(m, None, parts, rank)
        ranks = PT2.TorchRanks()
        ranks.set_send_lists(p)
        (q,) = PT2.extract_partitions(m, None, parts, ranks=[rank])
        assert np.array_equal(p.send_cells, q.send_cells)
        assert np.array_equal(p.send_counts, q.send_counts)
        assert np.array_equal(p.recv_counts, q.recv_counts)
        member = _Member(p)
        for rb in (32, 96):
            _fill_and_check(member, ranks, m, rb)
        dist.barrier()
        out.put((rank, "ok"))
    except BaseException as e:  # noqa: BLE001
        out.put((rank, repr(e)))
    finally:
        dist.destroy_process_group()


def test_torch_ranks_exchange_and_reduce_gloo():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_torch_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(out.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got == [(0, "ok"), (1, "ok")]


def test_one_part_keeps_only_its_images():
    """A partition into one part is the whole mesh: no external ghost, no send list, and the
    periodic images stay images of their owned cells."""
    m = M.periodic_box_hex(8, 8, 2)
    w = m.gradient_weights(np.full(m.n_boundary_faces, M.BC_SLIP, np.uint8))
    (p,) = PT.extract_partitions(m, w, np.zeros(m.n_owned_cells, np.int32))
    assert p.n_external == 0 and p.send_cells.size == 0
    assert p.n_owned == m.n_owned_cells
    assert np.all(p.mesh["ghost_owner"] >= 0)
    check_partition(m, w, p)


def test_a_request_for_a_cell_the_rank_does_not_own_is_refused():
    m = M.bump_channel(24, 12, 4)
    parts = PT.partition_cells(m, 2)
    p = PT.extract_partition(m, None, parts, 0)
    foreign = np.nonzero(parts == 1)[0][:3]
    with pytest.raises(ValueError, match="does not own"):
        PT.set_send_lists(p, [np.zeros(0, np.int64), foreign])


def test_requests_and_send_lists_pair_up():
    """What each rank requests of another (in its ghost order) is what that rank's send list
    holds for it, cell for cell."""
    m = M.jittered_tets(8, 8, 2, extent=(1.0, 1.0, 0.25))
    parts = random_parts(m, 4, 9)
    ps = PT.extract_partitions(m, None, parts)
    for q in ps:
        asked = PT.requests(q)
        for r in ps:
            first = int(r.send_counts[: q.rank].sum())
            sent = r.cell_global[r.send_cells[first : first + int(r.send_counts[q.rank])]]
            assert np.array_equal(sent, asked[r.rank])


def _oracle_cases():
    from autan_b200 import cases as K

    return [
        K.bump_channel(24, 12, 4, precision="fp32+acc64", steps=1),
        K.bump_channel(24, 12, 4, precision="fp64", steps=1),
        K.vortex_tets(8, 8, 2, steps=1, precision="fp32+acc64", extent=(10.0, 10.0, 2.5)),
        K.vortex_hex(8, 8, 2, steps=1, precision="fp64"),
    ]


@pytest.mark.parametrize("index", range(4))
def test_partitions_restate_the_whole_mesh_residual_on_the_oracle(index):
    """The CPU oracle over each rank's local mesh, its external ghosts given the values the owning
    ranks hold (the whole mesh's primitives, gradients and limiter values), gives every owned
    cell the whole mesh's residual bit for bit, second order with the limiter: the local meshes
    keep the global loop order, orientation, geometry, stencils, weights and boundary faces."""
    import oracle as O
    from autan_b200 import cases as K

    case = _oracle_cases()[index]
    case.scheme.second_order = True
    case.scheme.limiter = True
    m = case.mesh
    rng = np.random.default_rng(4)
    u = case.u0 * (1.0 + 1e-3 * rng.uniform(-1.0, 1.0, case.u0.shape))
    if m.n_cells > m.n_owned_cells:
        u[:, m.n_owned_cells :] = u[:, m.ghost_owner]
    md = K.oracle_mesh_dict(case)
    whole = O.Oracle(md, case.scheme.as_dict(), case.bc_kind, case.bc_data)
    r_whole = whole.residual(u)
    fields = whole.arrays()
    for parts in (PT.partition_cells(m, 3), random_parts(m, 4, 2)):
        for p in PT.extract_partitions(m, md["stencil_lsq_weight"], parts):
            local = dict(p.mesh, stencil_lsq_weight=p.weights)
            o = O.Oracle(local, case.scheme.as_dict(), case.bc_kind[p.bc_index],
                         case.bc_data[:, p.bc_index])  # fmt: skip
            ng = p.mesh["n_cells"] - p.n_owned
            ext = p.cell_global[p.n_owned : p.n_owned + p.n_external]

            def ghosts(a, comps):
                out = np.zeros((comps, ng))
                out[:, : p.n_external] = a[:, ext]
                return out

            o.set_external(ghosts(fields["prim"], 5), ghosts(fields["grad"], 15),
                           ghosts(fields["phi"], 5))  # fmt: skip
            r = o.residual(np.ascontiguousarray(u[:, p.cell_global]))
            want = r_whole[:, p.cell_global[: p.n_owned]]
            assert np.array_equal(r[:, : p.n_owned].view(np.int64), want.view(np.int64)), p.rank


def _oracle_step_rank(rank: int, world: int, port: int, out) -> None:
    """One gloo rank: each case's partition stepped by the CPU oracle, its ghost fills and the
    CFL step's minimum through TorchRanks (the exchange code of the NCCL path), against the whole
    mesh stepped by the oracle alone."""
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, str(REPO))
    sys.path.insert(0, str(REPO / "tests"))
    import torch
    import torch.distributed as dist

    import oracle as O
    from autan_b200 import cases as K
    from autan_b200 import partition as PT2

    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))  # fmt: skip
    try:
        results = []
        for index, case in enumerate(_oracle_cases()):
            m = case.mesh
            md = K.oracle_mesh_dict(case)
            rng = np.random.default_rng(6)
            u = case.u0 * (1.0 + 1e-3 * rng.uniform(-1.0, 1.0, case.u0.shape))
            if m.n_cells > m.n_owned_cells:
                u[:, m.n_owned_cells :] = u[:, m.ghost_owner]
            steps = 3
            whole = O.Oracle(md, case.scheme.as_dict(), case.bc_kind, case.bc_data)
            ug = np.ascontiguousarray(u.copy())
            dts = [whole.step(ug, rk=case.rk, cfl=case.cfl, local=case.local)[1] for _ in range(steps)]
            for split in ("blocks", "random"):
                parts = PT2.partition_cells(m, world) if split == "blocks" else random_parts(m, world, 5)
                p = PT2.extract_partition(m, md["stencil_lsq_weight"], parts, rank)
                ranks = PT2.TorchRanks()
                ranks.set_send_lists(p)
                o = O.Oracle(dict(p.mesh, stencil_lsq_weight=p.weights), case.scheme.as_dict(),
                             case.bc_kind[p.bc_index], case.bc_data[:, p.bc_index])  # fmt: skip

                def halo(kind, send, recv, p=p, ranks=ranks):
                    comps = send.shape[0]
                    rows = torch.from_numpy(np.ascontiguousarray(send[:, p.send_cells].T))
                    got = torch.zeros((p.n_external, comps), dtype=torch.float64)
                    ranks.exchange_rows(p, rows, got)
                    recv[:, : p.n_external] = got.numpy().T

                def minimum(x):
                    t = torch.tensor([x], dtype=torch.float64)
                    dist.all_reduce(t, op=dist.ReduceOp.MIN)
                    return float(t.item())

                o.set_ranks(halo, minimum)
                ul = np.ascontiguousarray(u[:, p.cell_global])
                got_dt = [o.step(ul, rk=case.rk, cfl=case.cfl, local=case.local)[1]
                          for _ in range(steps)]  # fmt: skip
                want = ug[:, p.cell_global[: p.n_owned]]
                same = np.array_equal(ul[:, : p.n_owned].view(np.int64), want.view(np.int64))
                results.append((index, split, bool(same), got_dt == dts, p.n_external))
        out.put((rank, results))
    except BaseException as e:  # noqa: BLE001
        out.put((rank, repr(e)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_partitioned_oracle_steps_over_gloo_ranks(world):
    """Gloo ranks step their partitions on the CPU oracle, exchanging ghost values and the step's
    minimum through TorchRanks: three steps of the channel (fp32+acc64 and fp64, local steps),
    the periodic tets (global CFL step) and the periodic hex (first order, RK4) equal the whole
    mesh's bit for bit, over block and random partitions."""
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_oracle_step_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    got = sorted((out.get(timeout=300) for _ in procs), key=lambda x: x[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, results in got:
        assert isinstance(results, list), results
        assert len(results) == 8
        for index, split, same, same_dt, n_ext in results:
            assert n_ext > 0, (rank, index, split)
            assert same and same_dt, (rank, index, split)


def test_a_rank_that_fails_or_never_arrives_ends_the_others_exchange():
    """Failure detection among thread ranks, on the host: a rank that raises before its exchange
    aborts the barrier, and a rank that never arrives lets the barrier's timeout run out; either
    way the waiting ranks leave their exchange with an error instead of hanging."""
    import time

    m = M.jittered_tets(8, 8, 2, extent=(1.0, 1.0, 0.25))
    ps = PT.extract_partitions(m, None, random_parts(m, 3, 1))
    for failure in ("raises", "absent"):
        ranks = PT.ThreadRanks(3, timeout=1.0 if failure == "absent" else 60.0)
        members = [_Member(p) for p in ps]
        for mb in members:
            ranks.join(mb)
        errors, started = [], time.monotonic()

        def run(mb):
            try:
                if mb.part.rank == 2:
                    if failure == "raises":
                        ranks.barrier.abort()  # what a failed rank's error path does
                        raise RuntimeError("rank 2 failed")
                    return  # rank 2 never comes to the exchange
                ranks.exchange(mb, 0, 32, None)
            except BaseException as e:  # noqa: BLE001 (checked below)
                errors.append((mb.part.rank, type(e).__name__))

        threads = [threading.Thread(target=run, args=(mb,)) for mb in members]
        for t in threads:
            t.start()
        for t in threads:
            t.join(timeout=30)
        assert all(not t.is_alive() for t in threads)
        waiting = sorted(r for r, name in errors if name == "BrokenBarrierError")
        assert waiting == [0, 1], (failure, errors)
        assert time.monotonic() - started < 20


def _departing_rank(rank: int, world: int, port: int, out) -> None:
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, str(REPO))
    import time

    import torch
    import torch.distributed as dist

    from autan_b200 import mesh as M2
    from autan_b200 import partition as PT2

    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=5))  # fmt: skip
    m = M2.bump_channel(24, 12, 4)
    parts = PT2.partition_cells(m, world)
    p = PT2.extract_partition(m, None, parts, rank)
    ranks = PT2.TorchRanks()
    ranks.set_send_lists(p)
    dist.barrier()
    if rank == 1:
        out.put((rank, "left"))
        out.close()
        out.join_thread()  # the message out before the abrupt exit
        os._exit(0)  # leaves between steps, without its exchange
    started = time.monotonic()
    try:
        send = torch.zeros((p.send_cells.size, 4), dtype=torch.float64)
        recv = torch.zeros((p.n_external, 4), dtype=torch.float64)
        ranks.exchange_rows(p, send, recv)
        out.put((rank, "no error"))
    except BaseException as e:  # noqa: BLE001
        out.put((rank, f"error after {time.monotonic() - started:.0f} s: {type(e).__name__}"))
    out.close()
    out.join_thread()
    os._exit(0)


def test_a_departed_rank_ends_the_torch_exchange_with_an_error():
    """A gloo rank leaves between steps; the other rank's next exchange fails (the process group's
    short timeout or the closed connection) instead of waiting forever."""
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_departing_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    assert got[1] == "left"
    assert got[0].startswith("error after"), got[0]
