"""One mesh stepped by several ranks: the partition of its owned cells, each rank's local mesh
with its ghosts, and the forward ghost exchange and reductions a partitioned step makes.

    partition_cells(mesh, n_parts)          (partition/include/autan/partition/partition.hpp:38-53)
    extract_partition(mesh, weights, ...)   extract_partition (partition.hpp:132-145), one rank;
    extract_partitions                      every rank in one process
    Partition.send_cells / recv_counts      HaloPattern (partition.hpp:94-110); the send side set
                                            from the other ranks' requests (set_send_lists,
                                            TorchRanks.set_send_lists over a group)
    ThreadRanks, TorchRanks                 HaloExchange forward (halo_exchange.hpp:14-66) and
                                            Ranks::sum / min
    PartitionedEuler                        the device stepper of one rank (autan_euler_ranks)

A local mesh keeps the global mesh's geometry bit for bit and its order: owned cells in global
order, their interior faces in global order with the global orientation, then their boundary
faces, then the boundary faces of ghost cells that owned cells' stencils name; each owned cell's
faces and stencil entries in their global order. Every loop of the device path therefore adds the
same terms in the same order as on the whole mesh, and a partitioned step gives the whole mesh's
bits (the reference's reproducibility under global keys, physics/src/euler.cpp:85-88).

Ghosts: every cell an owned cell's stencil, faces or stencil boundary faces name that this rank
does not own. A periodic image whose owner is this rank's stays an image ghost (ghost_owner its
local owner); every other ghost is external (ghost_owner -1): its records come from the rank
that owns it (for an image, the owner of its owned cell), ordered by that rank, then by global
cell. The send list of a rank is, for each receiving rank in ascending order, the cells whose
records that rank's external ghosts take, in the receiver's ghost order (a cell is repeated
where a receiver holds it twice, as itself and as an image).
"""

from __future__ import annotations

import ctypes as C
import threading
from dataclasses import dataclass, field

import numpy as np

from autan_b200 import _native as N
from autan_b200.euler import EulerDevice, Scheme, StepResult
from autan_b200.mesh import Mesh

PRIM_WORDS, RECON_WORDS = 8, 24  # words of a primitive record and of a reconstruction record
NORM_WORDS = 5 * 71  # the exact-sum words of the five residual norms


def cell_cost(mesh: Mesh) -> np.ndarray:
    """Faces of each owned cell: the cost of its face and gradient loops
    (cell_cost_weights, partition.hpp:36-38)."""
    off = mesh.cell_face_offsets
    return np.diff(off[: mesh.n_owned_cells + 1]).astype(np.int64)


def partition_cells(mesh: Mesh, n_parts: int) -> np.ndarray:
    """Part in [0, n_parts) of every owned cell: consecutive runs of the mesh's cell order (RCM or
    Z-order on the generators here, so that runs are compact) of about equal cost. The reference
    cuts the dual graph with METIS (partition_cells, partition.hpp:40-53); any partition gives the
    same results here, only the ghost counts differ."""
    n = mesh.n_owned_cells
    if n_parts < 1 or n_parts > n:
        raise ValueError("n_parts must be between 1 and the owned cells")
    cost = np.cumsum(cell_cost(mesh))
    bounds = np.searchsorted(cost, cost[-1] * np.arange(1, n_parts) / n_parts, side="left")
    parts = np.zeros(n, dtype=np.int32)
    for b in bounds:
        parts[b + 1 :] += 1
    if np.bincount(parts, minlength=n_parts).min() == 0:
        raise ValueError("a part came out empty")
    return parts


def _rows(offsets: np.ndarray, cells: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """The entry indices of the CSR rows of `cells`, concatenated, and each row's length."""
    start = offsets[cells].astype(np.int64)
    length = (offsets[cells + 1] - offsets[cells]).astype(np.int64)
    total = int(length.sum())
    if total == 0:
        return np.zeros(0, dtype=np.int64), length
    first = np.repeat(start - np.concatenate(([0], np.cumsum(length)[:-1])), length)
    return first + np.arange(total, dtype=np.int64), length


@dataclass
class Partition:
    """One rank's share of a partitioned mesh: the local mesh (a dict of the arrays
    `autan_euler_mesh` takes), its LSQ weights, the global index of each local cell and boundary
    face, and the halo (HaloPattern, partition.hpp:94-110)."""

    rank: int
    n_parts: int
    mesh: dict = field(repr=False)
    weights: np.ndarray = field(repr=False)
    cell_global: np.ndarray = field(repr=False)  # local cell -> global cell
    bface_global: np.ndarray = field(repr=False)  # local boundary face -> global boundary face
    face_global: np.ndarray = field(default=None, repr=False)  # local face -> global face
    n_external: int = 0
    recv_counts: np.ndarray = field(default=None, repr=False)  # external ghosts from each rank
    send_cells: np.ndarray = field(default=None, repr=False)  # local owned cells, by receiver
    send_counts: np.ndarray = field(default=None, repr=False)  # records sent to each rank
    global_cells: int = 0
    _sources: np.ndarray = field(default=None, repr=False)  # global owned cell of each external

    @property
    def n_owned(self) -> int:
        return int(self.mesh["n_owned_cells"])

    @property
    def bc_index(self) -> np.ndarray:
        """The global boundary face of each local boundary face (indices into the global mesh's
        boundary codes and data)."""
        return self.bface_global


def _extract(mesh: Mesh, weights: np.ndarray | None, parts: np.ndarray, rank: int) -> Partition:
    """The local mesh of `rank` (without its send list)."""
    no, nc, ni = mesh.n_owned_cells, mesh.n_cells, mesh.n_interior_faces
    nf = mesh.n_faces
    owner, neighbour = mesh.owner, mesh.neighbour
    gowner = mesh.ghost_owner
    home = np.concatenate((np.arange(no, dtype=np.int64), gowner.astype(np.int64)))  # owned cell
    owned = np.nonzero(parts == rank)[0].astype(np.int64)
    if owned.size == 0:
        raise ValueError(f"rank {rank} owns no cell")
    # faces of the owned cells, in global order
    fidx, flen = _rows(mesh.cell_face_offsets, owned)
    faces = np.unique(mesh.cell_faces[fidx]).astype(np.int64)
    f_int = faces[faces < ni]
    f_bnd = faces[faces >= ni]
    # stencil rows of the owned cells
    sidx, slen = _rows(mesh.stencil_offsets, owned)
    sent = mesh.stencil[sidx].astype(np.int64)
    s_cells = sent[sent >= 0]
    s_bnd = -sent[sent < 0] - 1
    extra_bnd = np.setdiff1d(np.unique(s_bnd), f_bnd)
    # every cell a loop of the owned cells reads
    named = np.unique(np.concatenate((owner[f_int], neighbour[f_int], s_cells, owner[extra_bnd]))).astype(np.int64)
    mine = np.zeros(nc, dtype=bool)
    mine[owned] = True
    ghosts = named[~mine[named]]
    gh_home = home[ghosts]
    gh_rank = parts[gh_home]
    is_ext = gh_rank != rank
    ext = ghosts[is_ext]
    ext_rank = gh_rank[is_ext]
    order = np.lexsort((ext, ext_rank))  # by source rank, then global cell
    ext, ext_rank = ext[order], ext_rank[order]
    img = ghosts[~is_ext]  # ascending
    cell_global = np.concatenate((owned, ext, img))
    n_loc, n_ext = owned.size, ext.size
    cmap = np.full(nc, -1, dtype=np.int64)
    cmap[cell_global] = np.arange(cell_global.size)
    # faces: owned cells' interior faces, their boundary faces, then the named boundary faces of
    # ghost cells
    face_global = np.concatenate((f_int, f_bnd, extra_bnd))
    fmap = np.full(nf, -1, dtype=np.int64)
    fmap[face_global] = np.arange(face_global.size)
    ni_l = f_int.size
    local = {
        "n_cells": int(cell_global.size),
        "n_owned_cells": int(n_loc),
        "n_faces": int(face_global.size),
        "n_interior_faces": int(ni_l),
        "n_owned_interior_faces": int(ni_l),
        "n_owned_faces": int(ni_l + f_bnd.size),
    }
    local["owner"] = cmap[owner[face_global]].astype(np.int32)
    local["neighbour"] = cmap[neighbour[f_int]].astype(np.int32)
    cfo = np.zeros(cell_global.size + 1, dtype=np.int64)
    cfo[1 : n_loc + 1] = np.cumsum(flen)
    cfo[n_loc + 1 :] = cfo[n_loc]
    local["cell_face_offsets"] = cfo
    local["cell_faces"] = fmap[mesh.cell_faces[fidx]].astype(np.int32)
    gown = np.full(cell_global.size - n_loc, -1, dtype=np.int32)
    gown[n_ext:] = cmap[home[img]]
    local["ghost_owner"] = gown
    for k in ("face_normal", "face_centroid"):
        local[k] = np.ascontiguousarray(getattr(mesh, k)[:, face_global])
    local["face_area_magnitude"] = mesh.face_area_magnitude[face_global].copy()
    fm = mesh.face_moment
    local["face_moment"] = (np.ascontiguousarray(fm.reshape(9, nf)[:, face_global]) if fm.size
                            else np.zeros(0))  # fmt: skip
    local["cell_centroid"] = np.ascontiguousarray(mesh.cell_centroid[:, cell_global])
    local["cell_volume"] = mesh.cell_volume[cell_global].copy()
    so = np.zeros(cell_global.size + 1, dtype=np.int64)
    so[1 : n_loc + 1] = np.cumsum(slen)
    so[n_loc + 1 :] = so[n_loc]
    local["stencil_offsets"] = so
    st = np.where(sent >= 0, cmap[np.maximum(sent, 0)], -(fmap[np.maximum(-sent - 1, 0)] + 1))
    if st.size and (st[sent >= 0] < 0).any():
        raise AssertionError("a stencil cell missing from the local mesh")
    local["stencil"] = st.astype(np.int32)
    w = None if weights is None else np.ascontiguousarray(weights.reshape(3, -1)[:, sidx])
    counts = np.bincount(ext_rank, minlength=int(parts.max()) + 1).astype(np.int64)
    return Partition(rank=rank, n_parts=int(parts.max()) + 1, mesh=local, weights=w,
                     cell_global=cell_global, bface_global=face_global[ni_l:] - ni,
                     face_global=face_global,
                     n_external=int(n_ext), recv_counts=counts, global_cells=no,
                     _sources=home[ext])  # fmt: skip


def _check_parts(mesh: Mesh, parts) -> np.ndarray:
    parts = np.ascontiguousarray(parts, dtype=np.int32)
    if parts.size != mesh.n_owned_cells or parts.min() < 0:
        raise ValueError("one part per owned cell, from 0")
    return parts


def extract_partition(mesh: Mesh, weights: np.ndarray | None, parts: np.ndarray,
                      rank: int) -> Partition:  # fmt: skip
    """The local mesh of `rank` with its receive side (the ghosts it needs from each rank), but no
    send list yet: `set_send_lists` completes it from the other ranks' requests, which
    `TorchRanks.set_send_lists` gathers over a process group. `weights`: the global mesh's LSQ
    weights (3 x stencil entries) for its boundary kinds."""
    parts = _check_parts(mesh, parts)
    p = _extract(mesh, weights, parts, rank)
    p.n_parts = int(parts.max()) + 1
    if p.recv_counts.size < p.n_parts:
        p.recv_counts = np.pad(p.recv_counts, (0, p.n_parts - p.recv_counts.size))
    return p


def requests(part: Partition) -> list[np.ndarray]:
    """Per rank r, the global owned cells whose records this rank's external ghosts take from r,
    in ghost order (the receive side of the halo)."""
    ends = np.cumsum(part.recv_counts)
    return [part._sources[e - c : e] for c, e in zip(part.recv_counts, ends)]


def set_send_lists(part: Partition, wanted: list[np.ndarray]) -> None:
    """The send side of the halo from each rank q's request to this rank (`wanted[q]`: global
    owned cells of this rank, in q's ghost order): send_cells as local cells, by receiver."""
    owned = part.cell_global[: part.n_owned]  # ascending
    cells, counts = [], np.zeros(part.n_parts, dtype=np.int64)
    for q, g in enumerate(wanted):
        g = np.asarray(g, dtype=np.int64)
        at = np.searchsorted(owned, g)
        if g.size and (at.max() >= owned.size or not np.array_equal(owned[at], g)):
            raise ValueError(f"rank {q} asks for a cell rank {part.rank} does not own")
        cells.append(at)
        counts[q] = g.size
    part.send_cells = (np.concatenate(cells) if cells else np.zeros(0)).astype(np.int32)
    part.send_counts = counts


def extract_partitions(mesh: Mesh, weights: np.ndarray | None, parts: np.ndarray,
                       ranks=None) -> list[Partition]:  # fmt: skip
    """The local meshes of `ranks` (default: every part) with their send lists, all built in
    this process: every part's receive side is derived to build the send lists. A rank of a
    process group builds only its own (`extract_partition`, then `TorchRanks.set_send_lists`)."""
    parts = _check_parts(mesh, parts)
    n_parts = int(parts.max()) + 1
    every = [extract_partition(mesh, weights, parts, r) for r in range(n_parts)]
    asked = [requests(p) for p in every]  # asked[q][r]: what q wants from r
    want = range(n_parts) if ranks is None else ranks
    out = []
    for r in want:
        set_send_lists(every[r], [asked[q][r] for q in range(n_parts)])
        out.append(every[r])
    return out


# ---------------------------------------------------------------- exchange backends


class _Buffers:
    """One rank's exchange buffers: packed send records, received ghost records (bytes, 16-byte
    aligned rows) and the reduction words, as torch tensors on the rank's device."""

    def __init__(self, part: Partition, word_bytes: int, device):
        import torch

        rec = RECON_WORDS * word_bytes
        self.send = torch.zeros(max(int(part.send_cells.size), 1) * rec, dtype=torch.uint8, device=device)
        self.recv = torch.zeros(max(part.n_external, 1) * rec, dtype=torch.uint8, device=device)
        self.words = torch.zeros(NORM_WORDS + 1, dtype=torch.int64, device=device)

    def send_rows(self, n: int, record_bytes: int):
        return self.send[: n * record_bytes].view(n, record_bytes)

    def recv_rows(self, n: int, record_bytes: int):
        return self.recv[: n * record_bytes].view(n, record_bytes)


class ThreadRanks:
    """The ranks of one process, each stepping in a thread of its own (on one GPU or several):
    exchanges and reductions meet at a barrier, after each rank's stream has finished the work
    before them. The ranks' kernels never wait on each other; only their host threads do."""

    def __init__(self, n_ranks: int, timeout: float = 120.0):
        self.n = n_ranks
        self.barrier = threading.Barrier(n_ranks, timeout=timeout)
        self.members: list = [None] * n_ranks
        self.slots: list = [None] * n_ranks

    def join(self, member: "PartitionedEuler") -> "ThreadRanks":
        self.members[member.part.rank] = member
        return self

    @staticmethod
    def _stream(stream):
        """The stepper's stream (None: host tensors, nothing to wait for)."""
        import torch

        return torch.cuda.ExternalStream(stream) if stream else None

    @staticmethod
    def _on(s):
        import contextlib

        import torch

        return torch.cuda.stream(s) if s is not None else contextlib.nullcontext()

    @staticmethod
    def _sync(s) -> None:
        if s is not None:
            s.synchronize()

    def exchange(self, member, what: int, record_bytes: int, stream) -> None:
        if self.n == 1:
            return  # one rank: no ghost of another rank, nothing to wait for
        s = self._stream(stream)
        self._sync(s)  # the packing
        self.barrier.wait()
        p = member.part
        recv = member.buf.recv_rows(p.n_external, record_bytes)
        with self._on(s):
            at = 0
            for r in range(self.n):
                cnt = int(p.recv_counts[r])
                if cnt == 0:
                    continue
                peer = self.members[r]
                first = int(peer.part.send_counts[: p.rank].sum())
                src = peer.buf.send_rows(int(peer.part.send_cells.size), record_bytes)
                recv[at : at + cnt].copy_(src[first : first + cnt])
                at += cnt
        self._sync(s)
        self.barrier.wait()  # nobody packs again while a peer still reads its buffer

    def reduce(self, member, op: int, count: int, stream) -> None:
        if self.n == 1:
            return  # the sum and the minimum over one rank are its own words
        s = self._stream(stream)
        self._sync(s)
        mine = member.buf.words[:count].cpu().numpy().view(np.uint64)
        self.slots[member.part.rank] = mine
        self.barrier.wait()
        vals = [self.slots[r] for r in range(self.n)]
        if op == 0:
            out = np.zeros(count, dtype=np.uint64)
            for v in vals:  # ascending rank; modulo 2^64
                out += v
        else:
            out = np.min(np.stack([v.view(np.int64) for v in vals]), axis=0).view(np.uint64)
        self.barrier.wait()
        import torch

        with self._on(s):
            member.buf.words[:count].copy_(torch.from_numpy(out.view(np.int64)))
        self._sync(s)

    def min_host(self, member, value: int) -> int:
        if self.n == 1:
            return int(value)
        self.slots[member.part.rank] = int(value)
        self.barrier.wait()
        out = min(self.slots)
        self.barrier.wait()
        return out


class TorchRanks:
    """The ranks of a torch.distributed group, one process each (NCCL on GPUs; any backend with
    point-to-point operations): the exchange as send/receive pairs with every neighbour in one
    batch, the reductions as all-reduces, all on the stepper's stream."""

    def __init__(self, group=None):
        self.group = group

    def join(self, member):
        return self

    def set_send_lists(self, part: Partition, device=None) -> Partition:
        """Completes `part` (from extract_partition) with its send lists: every rank's requests
        gathered over the group (counts by all-gather, the cells by point-to-point pairs), so
        that no rank derives another's ghosts. `device`: where the group's tensors live (a CUDA
        device for NCCL, None for the CPU)."""
        import torch
        import torch.distributed as dist

        n = part.n_parts
        asked = requests(part)
        mine = torch.tensor([a.size for a in asked], dtype=torch.int64, device=device)
        table = [torch.zeros_like(mine) for _ in range(n)]
        dist.all_gather(table, mine, group=self.group)
        from_q = [int(table[q][part.rank]) for q in range(n)]  # what q asks of this rank
        recv = [torch.zeros(c, dtype=torch.int64, device=device) for c in from_q]
        ops = []
        for q in range(n):
            if q == part.rank:
                continue
            if from_q[q]:
                ops.append(dist.P2POp(dist.irecv, recv[q], q, self.group))
            if asked[q].size:
                t = torch.from_numpy(np.ascontiguousarray(asked[q], dtype=np.int64)).to(device or "cpu")
                ops.append(dist.P2POp(dist.isend, t, q, self.group))
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()
        set_send_lists(part, [r.cpu().numpy() for r in recv])
        return part

    @staticmethod
    def _ctx(stream):
        import contextlib

        import torch

        if stream and torch.cuda.is_available():
            return torch.cuda.stream(torch.cuda.ExternalStream(stream))
        return contextlib.nullcontext()

    def exchange(self, member, what: int, record_bytes: int, stream) -> None:
        p = member.part
        send = member.buf.send_rows(int(p.send_cells.size), record_bytes)
        recv = member.buf.recv_rows(p.n_external, record_bytes)
        with self._ctx(stream):
            self.exchange_rows(p, send, recv)

    def exchange_rows(self, part: Partition, send, recv) -> None:
        """The forward halo exchange of one row per cell: `send` holds the rows of
        part.send_cells (by receiver), `recv` receives the external ghosts' rows (by source rank,
        ghost order); tensors of any dtype and row width on the group's device."""
        import torch.distributed as dist

        ops = []
        s_at = r_at = 0
        for q in range(part.n_parts):
            sc, rc = int(part.send_counts[q]), int(part.recv_counts[q])
            if rc:
                ops.append(dist.P2POp(dist.irecv, recv[r_at : r_at + rc], q, self.group))
            if sc:
                ops.append(dist.P2POp(dist.isend, send[s_at : s_at + sc], q, self.group))
            s_at += sc
            r_at += rc
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()

    def reduce(self, member, op: int, count: int, stream) -> None:
        import torch.distributed as dist

        with self._ctx(stream):
            dist.all_reduce(member.buf.words[:count],
                            op=dist.ReduceOp.SUM if op == 0 else dist.ReduceOp.MIN,
                            group=self.group)  # fmt: skip

    def min_host(self, member, value: int) -> int:
        import torch
        import torch.distributed as dist

        t = torch.tensor([int(value)], dtype=torch.int64, device=member.buf.words.device)
        dist.all_reduce(t, op=dist.ReduceOp.MIN, group=self.group)
        return int(t.item())


# ---------------------------------------------------------------- one rank's stepper


_NONE = np.iinfo(np.int64).max


class PartitionedEuler:
    """The device stepper of one rank of a partitioned mesh (DeviceStepper<P> constructed with
    the rank's GhostFill and Ranks, physics/src/euler_device.cu:8-23): an EulerDevice over the
    local mesh whose steps call the backend's exchange and reductions through autan_euler_ranks.

    `bc_kind`, `bc_data`: the global mesh's boundary codes and data (one per global boundary
    face). Arrays in and out are global where the method says so."""

    def __init__(self, part: Partition, scheme: Scheme, ranks, bc_kind=None, bc_data=None,
                 device: int = 0):  # fmt: skip
        import torch

        if part.weights is None and scheme.second_order:
            raise ValueError("a second-order scheme needs the partition's LSQ weights")
        if part.send_cells is None:
            raise ValueError("the partition has no send lists yet (set_send_lists)")
        self.part = part
        kind = None if bc_kind is None else np.asarray(bc_kind, dtype=np.uint8)[part.bc_index]
        data = None if bc_data is None else np.asarray(bc_data, dtype=np.float64).reshape(5, -1)[:, part.bc_index]
        self.dev = EulerDevice(part.mesh, scheme, bc_kind=kind, bc_data=data, weights=part.weights,
                               device=device)  # fmt: skip
        word = 4 if scheme.precision == "fp32+acc64" else 8
        self.buf = _Buffers(part, word, torch.device("cuda", device) if device >= 0 else "cuda")
        self.ranks = ranks.join(self)
        self._error: BaseException | None = None

        def exchange(user, what, record_bytes, stream):
            return self._guard(self.ranks.exchange, self, int(what), int(record_bytes), stream)

        def reduce(user, op, count, stream):
            return self._guard(self.ranks.reduce, self, int(op), int(count), stream)

        self._fns = (N.EXCHANGE_FN(exchange), N.REDUCE_FN(reduce))
        self._send = np.ascontiguousarray(part.send_cells, dtype=np.int32)
        r = N.Ranks()
        r.user = None
        r.exchange, r.reduce = self._fns
        r.send = self.buf.send.data_ptr()
        r.recv = self.buf.recv.data_ptr()
        r.words = self.buf.words.data_ptr()
        r.n_send = int(self._send.size)
        r.send_cells = N.ptr(self._send, C.c_int32) if self._send.size else None
        r.global_cells = float(part.global_cells)
        self._ranks = r
        self.dev._call("autan_euler_device_set_ranks", C.byref(r))

    def _guard(self, fn, *args) -> int:
        try:
            fn(*args)
            return 0
        except BaseException as e:  # reported by the library as E1301, re-raised below
            self._error = e
            return 1

    def _native(self, call):
        try:
            return call()
        except N.NativeError:
            if self._error is not None:
                e, self._error = self._error, None
                raise RuntimeError("the ranks' exchange failed") from e
            raise

    def upload(self, u_global) -> None:
        """The local cells' entries of a global FP64 state (5 x global cells)."""
        u = np.asarray(u_global, dtype=np.float64).reshape(5, -1)
        self.dev.upload(np.ascontiguousarray(u[:, self.part.cell_global]))

    def download(self) -> np.ndarray:
        """The owned cells' FP64 state, 5 x owned cells (global cells part.cell_global[:n_owned])."""
        return self.dev.download()[:, : self.part.n_owned]

    def _global_invalid(self, r: StepResult) -> StepResult:
        bad = _NONE if r.invalid_cell is None else int(self.part.cell_global[r.invalid_cell])
        least = self.ranks.min_host(self, bad)
        r.invalid_cell = None if least == _NONE else least
        return r

    def step(self, cfl: float = 0.8, dt: float = 0.0, local: bool = False, rk: int = 3,
             n_steps: int = 1) -> StepResult:  # fmt: skip
        """n_steps steps of every rank (all ranks call it alike); the residual norms and the step
        are the whole mesh's, invalid_cell the least global cell of all ranks. The least invalid
        cell is that of the last step, as on one rank."""
        r = self._native(lambda: self.dev.step(cfl, dt, local, rk, n_steps, graph=False))
        return self._global_invalid(r)

    def evaluate(self) -> StepResult:
        r = self._native(lambda: self.dev.evaluate())
        return self._global_invalid(r)

    def history(self, count: int):
        return self.dev.history(count)

    def march(self, cfl: float = 0.8, dt: float = 0.0, local: bool = False, rk: int = 3,
              max_steps: int = 1000, batch: int = 50, orders: float = 8.0, floors=None) -> dict:  # fmt: skip
        """EulerDevice.march on every rank together: the whole mesh's norms drive the same
        convergence decision on every rank, so all take the same steps; invalid_cell global."""
        out = self._native(lambda: self.dev.march(cfl, dt, local, rk, max_steps, batch, orders,
                                                  floors))  # fmt: skip
        bad = out["invalid_cell"]
        least = self.ranks.min_host(self, _NONE if bad is None else int(self.part.cell_global[bad]))
        out["invalid_cell"] = None if least == _NONE else least
        return out

    def autotune(self, cfl: float = 0.8, dt: float = 0.0, local: bool = False, rk: int = 3,
                 trial_steps: int = 2) -> tuple[dict, float]:  # fmt: skip
        """The autotuner on this rank's mesh. Every rank calls it together: its trials step and
        so exchange; each rank keeps its own fastest choices (no result depends on them)."""
        return self._native(lambda: self.dev.autotune(cfl, dt, local, rk, trial_steps))

    def kernel_times(self, cfl: float = 0.8, dt: float = 0.0, local: bool = False, rk: int = 3,
                     n_steps: int = 1) -> dict:  # fmt: skip
        """EulerDevice.kernel_times of this rank (every rank calls it together)."""
        return self._native(lambda: self.dev.kernel_times(cfl, dt, local, rk, n_steps))

    def close(self) -> None:
        if getattr(self, "dev", None) is not None:
            try:
                self.dev._call("autan_euler_device_set_ranks", None)
            except Exception:
                pass
            self.dev.close()
            self.dev = None


def gather_state(parts: list[Partition], owned: list[np.ndarray], n_global: int) -> np.ndarray:
    """The global owned cells' state (5 x n_global) from each rank's owned state."""
    out = np.zeros((5, n_global))
    for p, u in zip(parts, owned):
        out[:, p.cell_global[: p.n_owned]] = u
    return out
