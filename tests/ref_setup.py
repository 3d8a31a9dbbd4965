"""ctypes binding of oracle/_ref/libref_setup.so: the reference's own mesh assembly, FP64 geometry
and face2 stencil (core/src/mesh.cpp:273 assemble, core/src/geometry.cpp:120 compute_geometry,
codegen/cpp/geometry.cpp:166 pack_geometry and :432 cell_stencil), compiled from the reference's
sources by `make -C oracle ref` (oracle/ref_setup_shim.cpp). Test infrastructure."""

from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB = Path(__file__).resolve().parent.parent / "oracle" / "_ref" / "libref_setup.so"
_lib = None


def available() -> bool:
    return LIB.exists()


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(str(LIB))
        _lib.ref_setup.restype = C.c_int
        _lib.ref_setup.argtypes = [C.c_int64, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32,
                                   C.c_int32, C.c_void_p, C.POINTER(C.c_void_p), C.c_char_p,
                                   C.c_size_t]  # fmt: skip
        _lib.ref_count.restype = C.c_int64
        _lib.ref_count.argtypes = [C.c_void_p, C.c_char_p, C.POINTER(C.c_int32)]
        _lib.ref_copy.restype = C.c_int
        _lib.ref_copy.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p]
        _lib.ref_free.restype = None
        _lib.ref_free.argtypes = [C.c_void_p]
    return _lib


NAMES = ["face_source", "face_reversed", "owner", "neighbour", "cell_face_offsets", "cell_faces",
         "counts", "face_area", "face_area_magnitude", "face_centroid", "cell_volume",
         "cell_centroid", "face_normal", "face_moment", "stencil_offsets", "stencil",
         "stencil_lsq_weight"]  # fmt: skip


def reference_setup(mesh) -> dict[str, np.ndarray]:
    """The reference's set-up of the product mesh `mesh` (autan_b200.mesh.Mesh): its faces given
    face by face with the product's owner / neighbour and node loops, its ghost cells as the
    reference's halo cells (their centroids the product's, as a partitioner supplies them)."""
    nf, ni = mesh.n_faces, mesh.n_interior_faces
    c1 = np.full(nf, -1, dtype=np.int32)
    c1[:ni] = mesh.neighbour
    gc = None
    if mesh.n_cells > mesh.n_owned_cells:
        gc = mesh.cell_centroid[:, mesh.n_owned_cells:]
    return reference_setup_arrays(mesh.points, mesh.face_node_offsets, mesh.face_nodes, mesh.owner,
                                  c1, mesh.face_zone, mesh.n_cells,
                                  mesh.n_cells - mesh.n_owned_cells, gc)  # fmt: skip


def reference_setup_arrays(points, face_node_offsets, face_nodes, cell0, cell1, face_zone,
                           n_cells: int, n_ghost: int, ghost_centroid=None) -> dict[str, np.ndarray]:
    """The reference's set-up of a mesh given face by face: points 3 x n_points, each face's node
    loop, the cells on its two sides (cell1 -1 on a boundary face), the boundary zone of each
    boundary face, the last n_ghost cells periodic images (ghost_centroid 3 x n_ghost, their
    centroids, or None)."""
    l = lib()
    pts = np.ascontiguousarray(points, dtype=np.float64)
    fno = np.ascontiguousarray(face_node_offsets, dtype=np.int64)
    fn = np.ascontiguousarray(face_nodes, dtype=np.int32)
    c0 = np.ascontiguousarray(cell0, dtype=np.int32)
    c1 = np.ascontiguousarray(cell1, dtype=np.int32)
    nf = c0.size
    zone = np.ascontiguousarray(face_zone, dtype=np.int32)
    n_zones = int(max(zone.max(initial=-1) + 1, 1))
    gc = None if ghost_centroid is None else np.ascontiguousarray(ghost_centroid, dtype=np.float64)
    h = C.c_void_p()
    err = C.create_string_buffer(1024)
    rc = l.ref_setup(pts.shape[1], pts.ctypes.data, nf, fno.ctypes.data, fn.ctypes.data,
                     c0.ctypes.data, c1.ctypes.data, zone.ctypes.data, n_zones, int(n_cells),
                     int(n_ghost), None if gc is None else gc.ctypes.data, C.byref(h), err,
                     len(err))  # fmt: skip
    if rc != 0:
        raise RuntimeError(err.value.decode())
    out = {}
    try:
        for name in NAMES:
            is_int = C.c_int32()
            n = l.ref_count(h, name.encode(), C.byref(is_int))
            if n < 0:
                raise KeyError(name)
            a = np.zeros(n, dtype=np.int64 if is_int.value else np.float64)
            if n:
                l.ref_copy(h, name.encode(), a.ctypes.data)
            out[name] = a
    finally:
        l.ref_free(h)
    nc = int(n_cells)
    for k, rows, cols in (("face_area", 3, nf), ("face_centroid", 3, nf), ("face_normal", 3, nf),
                          ("face_moment", 9, nf), ("cell_centroid", 3, nc)):  # fmt: skip
        out[k] = out[k].reshape(rows, cols)
    out["stencil_lsq_weight"] = out["stencil_lsq_weight"].reshape(3, -1)
    return out
