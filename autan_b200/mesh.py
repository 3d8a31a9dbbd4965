"""Meshes for the explicit Euler path, in the layouts of Autan's face-based mesh contract
(docs/contracts/mesh.md): built by the native set-up library (include/autan_b200_setup.h) and held
as numpy arrays.

Generators for the workloads of the path:
- `periodic_box_hex`: the n_x x n_y x n_z hexahedral box, periodic in x and y, symmetry in z;
- `jittered_tets`: a lattice whose nodes are moved by a seeded uniform jitter (tangentially only
  on boundary planes, identically on both sides of a periodic pair, as
  vv/src/autan_vv/meshes/vortex.py:41-60 moves its lattice), each box split into 6 Kuhn
  tetrahedra (tests/core/fixtures.cpp BoxFill::tetra).
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from autan_b200 import _native as N

# Boundary condition codes (kernels/euler.py:55-60, physics/include/autan/physics/euler.hpp:31-38).
BC_STATE, BC_FARFIELD, BC_SLIP, BC_INLET, BC_OUTLET, BC_WALL = range(6)
ORDERS = {"none": 0, "rcm": 1, "morton": 2}

_DTYPES = {("int32", 4): np.int32, ("int64", 8): np.int64, ("float64", 8): np.float64}
_INT32 = {"owner", "neighbour", "cell_faces", "face_zone", "stencil", "ghost_owner", "face_nodes",
          "owned_order"}  # fmt: skip
_INT64 = {"cell_face_offsets", "stencil_offsets", "face_node_offsets"}
_FLOAT = {"points", "face_area", "face_area_magnitude", "face_normal", "face_centroid",
          "face_moment", "cell_centroid", "cell_volume", "ghost_translation"}  # fmt: skip


@dataclass
class Mesh:
    """An assembled mesh with its FP64 geometry and face2 stencil (arrays copied out of the
    native handle). Component c of entity i of a vector array is at [c, i]."""

    n_cells: int
    n_owned_cells: int
    n_faces: int
    n_interior_faces: int
    n_owned_interior_faces: int
    n_owned_faces: int
    all_planar: bool
    arrays: dict[str, np.ndarray] = field(repr=False)
    _handle: int | None = field(default=None, repr=False)

    def __getattr__(self, name: str) -> np.ndarray:
        arrays = self.__dict__.get("arrays")
        if arrays is not None and name in arrays:
            return arrays[name]
        raise AttributeError(name)

    @property
    def n_boundary_faces(self) -> int:
        return self.n_faces - self.n_interior_faces

    @property
    def n_stencil(self) -> int:
        return int(self.arrays["stencil"].size)

    @property
    def boundary_zone(self) -> np.ndarray:
        """Zone of each boundary face (n_boundary_faces)."""
        return self.arrays["face_zone"][self.n_interior_faces :]

    def gradient_weights(self, bc_kind: np.ndarray) -> np.ndarray:
        """LSQ weights over the face2 stencil for the given boundary codes, 3 x n_stencil FP64
        (Euler::Impl::compute_gradient_weights, physics/src/euler.cpp:340-416)."""
        kind = np.ascontiguousarray(bc_kind, dtype=np.uint8)
        if kind.size != self.n_boundary_faces:
            raise ValueError("one boundary code per boundary face")
        out = np.zeros((3, self.n_stencil), dtype=np.float64)
        err = N.errbuf()
        N.check(
            N.lib().autan_mesh_gradient_weights(
                self._handle, N.ptr(kind, C.c_uint8), N.ptr(out, C.c_double), err, len(err)
            ),
            err,
        )
        return out

    def close(self) -> None:
        if self._handle is not None:
            N.lib().autan_mesh_free(self._handle)
            self._handle = None

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:
            pass


def _from_handle(handle: int) -> Mesh:
    lib = N.lib()
    counts = (C.c_int64 * 12)()
    lib.autan_mesh_counts(handle, counts)
    arrays: dict[str, np.ndarray] = {}
    for name in sorted(_INT32 | _INT64 | _FLOAT):
        p, n, es = C.c_void_p(), C.c_int64(), C.c_int32()
        if lib.autan_mesh_array(handle, name.encode(), C.byref(p), C.byref(n), C.byref(es)) != 0:
            raise N.NativeError(f"E1100: array {name} missing")
        dt = np.int32 if name in _INT32 else np.int64 if name in _INT64 else np.float64
        if n.value == 0:
            arrays[name] = np.zeros(0, dtype=dt)
            continue
        buf = (C.c_char * (n.value * es.value)).from_address(p.value)
        arrays[name] = np.frombuffer(buf, dtype=dt).copy()
    nc, nf, ng, npt = int(counts[1]), int(counts[3]), int(counts[10]), int(counts[0])
    shapes = {
        "points": (3, npt),
        "face_area": (3, nf),
        "face_normal": (3, nf),
        "face_centroid": (3, nf),
        "face_moment": (9, nf),
        "cell_centroid": (3, nc),
        "ghost_translation": (3, ng),
    }
    for k, s in shapes.items():
        arrays[k] = arrays[k].reshape(s)
    return Mesh(
        n_cells=nc,
        n_owned_cells=int(counts[2]),
        n_faces=nf,
        n_interior_faces=int(counts[4]),
        n_owned_interior_faces=int(counts[5]),
        n_owned_faces=int(counts[6]),
        all_planar=bool(counts[9]),
        arrays=arrays,
        _handle=handle,
    )


def lattice(
    fill: str,
    n: tuple[int, int, int],
    origin=(0.0, 0.0, 0.0),
    extent=(1.0, 1.0, 1.0),
    periodic=(False, False, False),
    zones=(0, 1, 2, 3, 4, 5),
    displacement: np.ndarray | None = None,
    rcm: bool | int = False,
) -> Mesh:
    """A lattice mesh of hexahedra (`fill="hexa"`) or Kuhn tetrahedra (`fill="tetra"`).
    `zones`: boundary zone of the sides x-, x+, y-, y+, z-, z+ (ignored on periodic axes).
    `displacement`: 3 x (nx+1)(ny+1)(nz+1) node moves, node (i, j, k) at i + (nx+1)(j + (ny+1) k).
    `rcm`: owned cell order, False/0 the generator's, True/1 reverse Cuthill-McKee, 2 or "morton"
    the Z-order of the cell centres."""
    spec = N.Lattice()
    spec.fill = {"hexa": 0, "tetra": 1}[fill]
    spec.nx, spec.ny, spec.nz = n
    spec.origin[:] = origin
    spec.extent[:] = extent
    spec.periodic[:] = [int(bool(p)) for p in periodic]
    spec.zone[:] = zones
    disp = None
    if displacement is not None:
        disp = np.ascontiguousarray(displacement, dtype=np.float64)
        if disp.size != 3 * (n[0] + 1) * (n[1] + 1) * (n[2] + 1):
            raise ValueError("displacement must hold 3 values per lattice node")
        spec.displacement = N.ptr(disp, C.c_double)
    spec.rcm = ORDERS.get(rcm, rcm) if isinstance(rcm, str) else int(rcm)
    handle = C.c_void_p()
    err = N.errbuf()
    N.check(N.lib().autan_mesh_build_lattice(C.byref(spec), C.byref(handle), err, len(err)), err)
    return _from_handle(handle.value)


def from_cells(points, cell_face_offsets, face_node_offsets, face_nodes, face_zone, rcm=False):
    """A mesh from cells given by outward face loops (autan_mesh_build_cells)."""
    pts = np.ascontiguousarray(points, dtype=np.float64)
    cfo = np.ascontiguousarray(cell_face_offsets, dtype=np.int64)
    fno = np.ascontiguousarray(face_node_offsets, dtype=np.int64)
    fn = np.ascontiguousarray(face_nodes, dtype=np.int32)
    fz = np.ascontiguousarray(face_zone, dtype=np.int32)
    handle = C.c_void_p()
    err = N.errbuf()
    N.check(
        N.lib().autan_mesh_build_cells(
            pts.shape[-1], N.ptr(pts, C.c_double), cfo.size - 1, N.ptr(cfo, C.c_int64),
            N.ptr(fno, C.c_int64), N.ptr(fn, C.c_int32), N.ptr(fz, C.c_int32),
        ORDERS.get(rcm, 0) if isinstance(rcm, str) else int(rcm),
            C.byref(handle), err, len(err),
        ),
        err,
    )  # fmt: skip
    return _from_handle(handle.value)


# Boundary zones of the bump channel (autan_mesh_build_bump_channel).
ZONE_INLET, ZONE_OUTLET, ZONE_BUMP, ZONE_TOP, ZONE_ZMIN, ZONE_ZMAX = range(6)


def bump_channel(nx: int, ny: int, nz: int, extent=(3.0, 1.0, 0.5), bump=0.05, ratio=1.1,
                 stretched=None, prism_rows=None, brick_rows=None, brick_cols=None,
                 order="morton") -> Mesh:  # fmt: skip
    """The hybrid hexahedral / prismatic / polyhedral channel over the bump
    y_w = bump exp(-25 (x - 1.5)^2) (autan_mesh_build_bump_channel). Defaults: spacings grow by
    `ratio` over the first ny / 4 layers; prisms in rows [ny / 3, ny / 2); polyhedral bricks in
    rows [2 ny / 3, ny) over the middle third of the columns."""
    spec = N.BumpChannel()
    spec.nx, spec.ny, spec.nz = nx, ny, nz
    spec.extent[:] = extent
    spec.bump = bump
    spec.ratio = ratio
    spec.stretched = ny // 4 if stretched is None else stretched
    spec.prism_rows[:] = (ny // 3, ny // 2) if prism_rows is None else prism_rows
    spec.brick_rows[:] = (2 * ny // 3, ny) if brick_rows is None else brick_rows
    spec.brick_cols[:] = (nx // 3, 2 * nx // 3) if brick_cols is None else brick_cols
    spec.order = ORDERS.get(order, order) if isinstance(order, str) else int(order)
    handle = C.c_void_p()
    err = N.errbuf()
    N.check(N.lib().autan_mesh_build_bump_channel(C.byref(spec), C.byref(handle), err, len(err)),
            err)  # fmt: skip
    return _from_handle(handle.value)


def periodic_box_hex(nx=64, ny=64, nz=2, extent=(10.0, 10.0, 0.3125), origin=(0.0, 0.0, 0.0),
                     rcm=False) -> Mesh:  # fmt: skip
    """Hexahedral box periodic in x and y (image ghosts), zones 4 (z-) and 5 (z+) in z."""
    return lattice("hexa", (nx, ny, nz), origin, extent, (True, True, False), rcm=rcm)


def vortex_jitter(n: tuple[int, int, int], extent, amplitude=0.2, seed=0) -> np.ndarray:
    """Node displacement U(-a, a) h per axis (numpy default_rng(seed)), one draw per node of the
    periodic lattice in x and y, so that both sides of a periodic pair move alike; nodes on x
    lattice planes of the period boundary do not move along x (likewise y), and nodes on the z
    bounding planes do not move along z (tangential moves only, vv/src/autan_vv/meshes/vortex.py:
    41-60). Returns 3 x (nx+1)(ny+1)(nz+1)."""
    nx, ny, nz = n
    h = np.array(extent, dtype=np.float64) / np.array(n, dtype=np.float64)
    rng = np.random.default_rng(seed)
    jit = rng.uniform(-amplitude, amplitude, size=(3, nz + 1, ny, nx))
    k, j, i = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
    d = jit[:, k, j % ny, i % nx] * h[:, None, None, None]
    d[0] = np.where(i % nx == 0, 0.0, d[0])
    d[1] = np.where(j % ny == 0, 0.0, d[1])
    d[2] = np.where((k == 0) | (k == nz), 0.0, d[2])
    return d.reshape(3, -1)


def jittered_tets(nx=240, ny=240, nz=6, extent=(10.0, 10.0, 0.25), amplitude=0.2, seed=0,
                  rcm="morton") -> Mesh:  # fmt: skip
    """Kuhn tetrahedra of a jittered lattice, periodic in x and y, zones 4 (z-) and 5 (z+)."""
    disp = vortex_jitter((nx, ny, nz), extent, amplitude, seed)
    return lattice("tetra", (nx, ny, nz), (0.0, 0.0, 0.0), extent, (True, True, False),
                   displacement=disp, rcm=rcm)  # fmt: skip
