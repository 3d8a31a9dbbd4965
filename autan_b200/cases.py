"""The explicit-step workloads of the path: the convected isentropic vortex on periodic meshes.

- `vortex_hex`: 64 x 64 x 2 hexahedra on [0,10] x [0,10] x [0,0.3125] (8192 cells), periodic in x
  and y, symmetry (slip) in z; first-order Roe, classical RK4, CFL 0.5, FP64.
- `bump_channel`: steady subsonic flow (inlet Mach 0.5) through the hybrid hexahedral / prismatic /
  polyhedral channel over the bump 0.05 exp(-25 (x - 1.5)^2) on [0,3] x [0,1] x [0,0.5]; AUSM+-up
  (M_co = 0.5), second order with the Venkatakrishnan limiter (K = 5), total-pressure inlet,
  static-pressure outlet, slip walls, SSP-RK3 with local steps at CFL 1.5, fp32+acc64.
- `vortex_tets`: Kuhn tetrahedra of a 240 x 240 x 6 lattice on [0,10]^2 x [0,0.25] (2 073 600
  cells) whose nodes move by U(-0.2, 0.2) h (seed 0); second-order LSQ face2 gradient with the
  Venkatakrishnan limiter (K = 5), HLLC, SSP-RK3, CFL 0.8; FP64 or fp32+acc64.

Initial field: Shu's isentropic vortex of strength beta = 5 centred at (5, 5) on the freestream
rho = p = 1, u = v = 1, w = 0, gamma = 1.4 (Shu 1998, Lecture Notes in Mathematics 1697, section
5.2; the reference's vv/src/autan_vv/oracles/inviscid.py:105-181 states the same vortex scaled to
c = 1): du = beta / (2 pi) e^((1 - r^2) / 2) (-dy, dx), T = 1 - (gamma - 1) beta^2 / (8 gamma pi^2)
e^(1 - r^2), rho = T^(1 / (gamma - 1)), p = rho T, evaluated at the cell centroids.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from autan_b200 import mesh as M
from autan_b200.euler import Scheme

GAMMA = 1.4
FREESTREAM = (1.0, 1.0, 1.0, 0.0, 1.0)  # rho, u, v, w, p


def conserved(rho, u, v, w, p, gamma=GAMMA):
    return np.stack([rho, rho * u, rho * v, rho * w, p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v + w * w)])


def freestream_reference(gamma=GAMMA):
    rho, u, v, w, p = FREESTREAM
    return tuple(float(x) for x in conserved(np.array(rho), np.array(u), np.array(v), np.array(w),
                                             np.array(p), gamma))  # fmt: skip


def isentropic_vortex(mesh: M.Mesh, beta=5.0, centre=(5.0, 5.0), gamma=GAMMA) -> np.ndarray:
    """The conserved state (5 x n_cells, images copied from their cells)."""
    x = mesh.cell_centroid[0] - centre[0]
    y = mesh.cell_centroid[1] - centre[1]
    r2 = x * x + y * y
    f = beta / (2.0 * np.pi) * np.exp(0.5 * (1.0 - r2))
    u = FREESTREAM[1] - f * y
    v = FREESTREAM[2] + f * x
    t = 1.0 - (gamma - 1.0) * beta * beta / (8.0 * gamma * np.pi * np.pi) * np.exp(1.0 - r2)
    rho = t ** (1.0 / (gamma - 1.0))
    p = rho * t
    U = conserved(rho, u, v, np.zeros_like(u), p, gamma)
    if mesh.n_cells > mesh.n_owned_cells:
        U[:, mesh.n_owned_cells :] = U[:, mesh.ghost_owner]
    return np.ascontiguousarray(U)


@dataclass
class Case:
    name: str
    mesh: M.Mesh
    scheme: Scheme
    bc_kind: np.ndarray
    bc_data: np.ndarray
    u0: np.ndarray
    rk: int
    cfl: float
    steps: int
    local: bool = False

    @property
    def n_cells(self) -> int:
        return self.mesh.n_owned_cells


def vortex_hex(nx=64, ny=64, nz=2, steps=200, precision="fp64") -> Case:
    h = 10.0 / nx
    mesh = M.periodic_box_hex(nx, ny, nz, extent=(10.0, 10.0 * ny / nx, h * nz))
    scheme = Scheme(flux="roe", second_order=False, limiter=False, reference=freestream_reference(),
                    precision=precision, planar=bool(mesh.all_planar))  # fmt: skip
    kind = np.full(mesh.n_boundary_faces, M.BC_SLIP, dtype=np.uint8)
    return Case("vortex-hex", mesh, scheme, kind, np.zeros((5, mesh.n_boundary_faces)),
                isentropic_vortex(mesh), rk=4, cfl=0.5, steps=steps)  # fmt: skip


def vortex_tets(nx=240, ny=240, nz=6, steps=100, precision="fp32+acc64", rcm="morton",
                extent=None) -> Case:  # fmt: skip
    """The jittered-tetrahedra vortex; smaller lattices keep the cell size (h = 10 / 240) unless
    `extent` is given, so that parity cases are the same problem on a smaller periodic box. Cells
    in Morton order of their centres by default (`rcm`: see mesh.lattice)."""
    if extent is None:
        h = 10.0 / 240
        extent = (nx * h, ny * h, nz * h)
    mesh = M.jittered_tets(nx, ny, nz, extent=extent, rcm=rcm)
    speed = float(np.hypot(FREESTREAM[1], FREESTREAM[2]))
    scheme = Scheme(flux="hllc", second_order=True, limiter=True, venkat_k=5.0, length=1.0,
                    scale=(FREESTREAM[0], speed, speed, speed, FREESTREAM[4]),
                    reference=freestream_reference(), precision=precision,
                    planar=bool(mesh.all_planar))  # fmt: skip
    kind = np.full(mesh.n_boundary_faces, M.BC_SLIP, dtype=np.uint8)
    centre = (extent[0] / 2.0, extent[1] / 2.0)
    return Case("vortex-tets", mesh, scheme, kind, np.zeros((5, mesh.n_boundary_faces)),
                isentropic_vortex(mesh, centre=centre), rk=3, cfl=0.8, steps=steps)  # fmt: skip


def oracle_mesh_dict(case: Case) -> dict:
    """The case's mesh arrays with its gradient weights, as the oracle takes them."""
    m = case.mesh
    d = {k: getattr(m, k) for k in ("n_cells", "n_owned_cells", "n_faces", "n_interior_faces",
                                    "n_owned_interior_faces", "n_owned_faces")}  # fmt: skip
    for k in ("owner", "neighbour", "cell_face_offsets", "cell_faces", "ghost_owner",
              "face_normal", "face_area_magnitude", "face_centroid", "face_moment",
              "cell_centroid", "cell_volume", "stencil_offsets", "stencil"):  # fmt: skip
        d[k] = getattr(m, k)
    d["stencil_lsq_weight"] = m.gradient_weights(case.bc_kind)
    return d


def bump_channel(nx=480, ny=150, nz=100, mach=0.5, precision="fp32+acc64", steps=100,
                 order="morton") -> Case:  # fmt: skip
    """The steady bump channel (480 x 150 x 100 boxes: 8.0 M cells by default). Freestream
    rho = 1, p = 1 / gamma (unit sound speed), u = mach along x; gas constant 1 / gamma (T = 1).
    Inlet: total pressure and temperature of the freestream; outlet: its static pressure; bump,
    top and z sides slip. Starts from the uniform freestream."""
    mesh = M.bump_channel(nx, ny, nz, order=order)
    g = GAMMA
    rho, p = 1.0, 1.0 / g
    rgas = 1.0 / g
    t = p / (rho * rgas)
    fac = 1.0 + 0.5 * (g - 1.0) * mach * mach
    p0, t0 = p * fac ** (g / (g - 1.0)), t * fac
    kind = np.full(mesh.n_boundary_faces, M.BC_SLIP, dtype=np.uint8)
    data = np.zeros((5, mesh.n_boundary_faces))
    zone = mesh.boundary_zone
    kind[zone == M.ZONE_INLET] = M.BC_INLET
    data[0, zone == M.ZONE_INLET] = p0
    data[1, zone == M.ZONE_INLET] = t0
    kind[zone == M.ZONE_OUTLET] = M.BC_OUTLET
    data[4, zone == M.ZONE_OUTLET] = p
    free = conserved(np.array(rho), np.array(mach), np.array(0.0), np.array(0.0), np.array(p), g)
    scheme = Scheme(flux="ausm", second_order=True, limiter=True, venkat_k=5.0, length=1.0,
                    gamma=g, gas_constant=rgas, mach_ref=mach,
                    scale=(rho, mach, mach, mach, p), reference=tuple(float(x) for x in free),
                    precision=precision, planar=bool(mesh.all_planar))  # fmt: skip
    u0 = np.ascontiguousarray(np.repeat(free[:, None], mesh.n_cells, axis=1))
    return Case("bump-channel", mesh, scheme, kind, data, u0, rk=3, cfl=1.5, steps=steps,
                local=True)  # fmt: skip


MESH_KEYS = ("n_cells", "n_owned_cells", "n_faces", "n_interior_faces", "n_owned_interior_faces",
             "n_owned_faces")  # fmt: skip


UNION_KEYS = ("owner", "neighbour", "face_zone", "face_area_magnitude", "face_normal",
              "face_centroid", "face_area", "face_moment", "cell_face_offsets", "cell_faces",
              "cell_centroid", "cell_volume", "stencil_offsets", "stencil")  # fmt: skip


def compact(m: M.Mesh, moments: bool = True) -> "SimpleNamespace":
    """The arrays of a mesh that a union needs, detached from its native handle (closed here)."""
    from types import SimpleNamespace

    keys = UNION_KEYS if moments else tuple(k for k in UNION_KEYS if k != "face_moment")
    out = SimpleNamespace(**{k: getattr(m, k) for k in keys},
                          **{k: getattr(m, k) for k in MESH_KEYS}, all_planar=m.all_planar)  # fmt: skip
    if not moments:
        out.face_moment = None
    m.close()
    return out


def union(meshes, weights) -> tuple[dict, np.ndarray, np.ndarray]:
    """The disjoint union of meshes without ghost cells, in the mesh contract's layout: cells of
    mesh k after those of meshes < k; interior faces of every mesh (in mesh order), then boundary
    faces of every mesh; each cell's faces still in increasing order. meshes: Mesh objects or their
    compact() arrays (face_moment None: all planar, left out); weights: each mesh's LSQ weights
    (3 x its stencil entries). Returns the mesh arrays (a dict, as EulerDevice and the oracle take
    them), the concatenated weights and the cell offsets of the meshes."""
    for m in meshes:
        if m.n_cells != m.n_owned_cells:
            raise ValueError("union: meshes with ghost cells are not supported")
    moments = all(getattr(m, "face_moment", None) is not None for m in meshes)
    nc = np.array([m.n_cells for m in meshes])
    ni = np.array([m.n_interior_faces for m in meshes])
    nb = np.array([m.n_faces - m.n_interior_faces for m in meshes])
    coff = np.concatenate([[0], np.cumsum(nc)])
    ioff = np.concatenate([[0], np.cumsum(ni)])
    boff = np.concatenate([[0], np.cumsum(nb)])
    NI, NF = int(ioff[-1]), int(ioff[-1] + boff[-1])

    def new_face(k, f):
        f = np.asarray(f, dtype=np.int64)
        return np.where(f < ni[k], f + ioff[k], NI + boff[k] + (f - ni[k]))

    owner = np.empty(NF, dtype=np.int32)
    neighbour = np.empty(NI, dtype=np.int32)
    face_zone = np.empty(NF, dtype=np.int32)
    shapes = [("face_normal", 3), ("face_centroid", 3), ("face_area", 3)]
    if moments:
        shapes.append(("face_moment", 9))
    vec = {key: np.empty((d, NF)) for key, d in shapes}
    area = np.empty(NF)
    for k, m in enumerate(meshes):
        src_i = slice(0, ni[k])
        dst_i = slice(ioff[k], ioff[k + 1])
        src_b = slice(ni[k], ni[k] + nb[k])
        dst_b = slice(NI + boff[k], NI + boff[k + 1])
        for src, dst in ((src_i, dst_i), (src_b, dst_b)):
            owner[dst] = m.owner[src] + coff[k]
            face_zone[dst] = m.face_zone[src]
            area[dst] = m.face_area_magnitude[src]
            for key in vec:
                vec[key][:, dst] = getattr(m, key).reshape(vec[key].shape[0], -1)[:, src]
        neighbour[dst_i] = m.neighbour + coff[k]
    cfo, cf, so, st = [np.zeros(1, dtype=np.int64)], [], [np.zeros(1, dtype=np.int64)], []
    for k, m in enumerate(meshes):
        cfo.append(m.cell_face_offsets[1:] + cfo[-1][-1])
        cf.append(new_face(k, m.cell_faces).astype(np.int32))
        so.append(m.stencil_offsets[1:] + so[-1][-1])
        e = m.stencil.astype(np.int64)
        st.append(np.where(e >= 0, e + coff[k], -(new_face(k, -e - 1) + 1)).astype(np.int32))
    d = dict(n_cells=int(coff[-1]), n_owned_cells=int(coff[-1]), n_faces=NF, n_interior_faces=NI,
             n_owned_interior_faces=NI, n_owned_faces=NF, owner=owner, neighbour=neighbour,
             face_zone=face_zone, face_area_magnitude=area,
             cell_face_offsets=np.concatenate(cfo), cell_faces=np.concatenate(cf),
             ghost_owner=np.zeros(0, dtype=np.int32),
             cell_centroid=np.concatenate([m.cell_centroid for m in meshes], axis=1),
             cell_volume=np.concatenate([m.cell_volume for m in meshes]),
             stencil_offsets=np.concatenate(so), stencil=np.concatenate(st))  # fmt: skip
    d.update(vec)
    d["face_moment"] = d["face_moment"].reshape(-1) if moments else np.zeros(0)
    w = np.concatenate([np.asarray(x).reshape(3, -1) for x in weights], axis=1)
    d["stencil_lsq_weight"] = w
    d["all_planar"] = all(m.all_planar for m in meshes)
    d["boundary_offsets"] = boff.astype(np.int64)  # each mesh's first boundary face, from NI
    return d, w, coff


@dataclass
class Batch:
    """Many steady bump-channel cases as one union mesh (autan_euler_device_set_cases)."""

    mesh: dict
    weights: np.ndarray
    cell_offsets: np.ndarray
    scheme: Scheme
    bc_kind: np.ndarray
    bc_data: np.ndarray
    u0: np.ndarray
    params: list  # per case: dict(cells, mach, angle, bump, boxes)
    cfl: float = 1.5
    rk: int = 3

    @property
    def n_cells(self) -> int:
        return int(self.mesh["n_owned_cells"])

    @property
    def mach_ref(self) -> np.ndarray:
        """Per case, its AUSM+-up cut-off Mach number: the case's own freestream Mach, as a run of
        the case alone sets Scheme::mach_ref."""
        return np.array([p["mach"] for p in self.params], dtype=np.float64)

    def open(self, device: int = 0):
        """The batch on the device: an EulerDevice of the union mesh with the cases and their
        cut-off Mach numbers set (the caller uploads a state)."""
        from autan_b200.euler import EulerDevice

        dev = EulerDevice(self.mesh, self.scheme, self.bc_kind, self.bc_data, weights=self.weights,
                          device=device)  # fmt: skip
        dev.set_cases(self.cell_offsets)
        dev.set_case_mach_ref(self.mach_ref)
        return dev


def batch_parameters(n_cases, seed, cells) -> list[dict]:
    """The seeded per-case draws of bump_batch (numpy default_rng(seed)), in case order: target
    cells (log-uniform in `cells`), Mach, flow angle (degrees), bump height, and the boxes."""
    rng = np.random.default_rng(seed)
    lo, hi = np.log(cells[0]), np.log(cells[1])
    out = []
    for _ in range(n_cases):
        target = float(np.exp(rng.uniform(lo, hi)))
        mach = float(rng.uniform(0.3, 0.75))
        angle = float(rng.uniform(-4.0, 4.0))
        bump = float(rng.uniform(0.02, 0.10))
        # cells ~ 1.111 nx ny nz with nx = 6 a, ny = 2 a, nz = a
        a = max(2, int(round((target / (1.111 * 12.0)) ** (1.0 / 3.0))))
        out.append(dict(target=target, mach=mach, angle=angle, bump=bump, boxes=(6 * a, 2 * a, a)))
    return out


def shard_cases(params: list[dict], ranks: int) -> list[list[int]]:
    """Whole cases to ranks, greedy by cell count (largest first to the least loaded rank, ties to
    the lower rank): each rank's case indices in increasing order."""
    size = [1.111 * np.prod(p["boxes"]) for p in params]
    load = [0.0] * ranks
    out = [[] for _ in range(ranks)]
    for k in sorted(range(len(params)), key=lambda i: (-size[i], i)):
        r = min(range(ranks), key=lambda q: (load[q], q))
        out[r].append(k)
        load[r] += size[k]
    return [sorted(o) for o in out]


def bump_batch(n_cases=256, seed=0, cells=(20_000, 500_000), flux="roe", precision="fp32+acc64",
               inlet="farfield", walls=False, select=None) -> Batch:  # fmt: skip
    """Batched steady bump channels: per case (numpy default_rng(seed)) a cell count log-uniform
    in `cells`, Mach ~ U(0.3, 0.75), flow angle ~ U(-4, 4) degrees, bump height ~ U(0.02, 0.10).
    Each case's channel has about the requested cells (boxes in the ratio 3 : 1 : 1 / 2 of the
    channel's extent, hybrid rows as bump_channel). Inflow and outflow faces take the farfield
    state of the case's freestream (rho = 1, p = 1 / gamma, speed Mach, at the flow angle in the
    x-y plane); bump, top and z sides slip. walls: keep each case's bump-wall triangles
    (params[k]["wall"], t x 9, as WallSurface builds them) for the wall distance. A common scheme (second order, Venkatakrishnan K = 5,
    limiter scales and reference state of Mach 0.5 along x) serves every case, except the AUSM+-up
    cut-off Mach number, which is each case's own (Batch.mach_ref, set by Batch.open: with one
    shared cut-off above their Mach number, cases at Mach 0.30-0.42 stall in a limit cycle three
    decades above their round-off band); local steps make the cases independent. inlet="state": the inflow faces take the freestream as a given state and the
    outflow faces its static pressure (no exp/log on the path, for bit-exact tests). select: the
    case indices to build (default all), the draws being those of all n_cases."""
    draws = batch_parameters(n_cases, seed, cells)
    g = GAMMA
    p = 1.0 / g
    meshes, weights, kinds, datas, u0s, params = [], [], [], [], [], []
    for k in range(n_cases) if select is None else select:
        d0 = draws[k]
        mach, angle, bump = d0["mach"], d0["angle"], d0["bump"]
        nx, ny, nz = d0["boxes"]
        m = M.bump_channel(nx, ny, nz, bump=bump)
        zone = m.boundary_zone
        kind = np.full(m.n_boundary_faces, M.BC_SLIP, dtype=np.uint8)
        data = np.zeros((5, m.n_boundary_faces))
        t = np.radians(angle)
        w = np.array([1.0, mach * np.cos(t), mach * np.sin(t), 0.0, p])
        io = (zone == M.ZONE_INLET) | (zone == M.ZONE_OUTLET)
        if inlet == "state":
            kind[zone == M.ZONE_INLET] = M.BC_STATE
            data[:, zone == M.ZONE_INLET] = w[:, None]
            kind[zone == M.ZONE_OUTLET] = M.BC_OUTLET
            data[4, zone == M.ZONE_OUTLET] = p
        else:
            kind[io] = M.BC_FARFIELD
            data[:, io] = w[:, None]
        weights.append(m.gradient_weights(kind))
        kinds.append(kind)
        datas.append(data)
        free = conserved(*(np.array(x) for x in w), g)
        u0s.append(np.repeat(free[:, None], m.n_cells, axis=1))
        from autan_b200.euler import residual_scales

        params.append(dict(cells=m.n_cells, mach=mach, angle=angle, bump=bump, boxes=(nx, ny, nz),
                           phi=residual_scales(m, 1.0, p, mach, g), case=k))  # fmt: skip
        if walls:
            from autan_b200.warmstart import wall_triangles

            params[-1]["wall"] = wall_triangles(m, M.ZONE_BUMP)
        meshes.append(compact(m, moments=not m.all_planar))
    d, wts, coff = union(meshes, weights)
    ref = conserved(np.array(1.0), np.array(0.5), np.array(0.0), np.array(0.0), np.array(p), g)
    scheme = Scheme(flux=flux, second_order=True, limiter=True, venkat_k=5.0, length=1.0, gamma=g,
                    gas_constant=1.0 / g, mach_ref=0.5, scale=(1.0, 0.5, 0.5, 0.5, p),
                    reference=tuple(float(x) for x in ref), precision=precision,
                    planar=bool(d["all_planar"]))  # fmt: skip
    return Batch(d, wts, coff, scheme, np.concatenate(kinds), np.concatenate(datas, axis=1),
                 np.ascontiguousarray(np.concatenate(u0s, axis=1)), params)  # fmt: skip
