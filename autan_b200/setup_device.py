"""The gradient set-up on the GPU (include/autan_b200_setup.h, autan_setup_device_*): the face2
stencil of every cell and the least-squares weights of the owned cells, computed by kernels with
the same per-cell rules as the host set-up, so both give the same bits."""

from __future__ import annotations

import ctypes as C

import numpy as np

from autan_b200 import _native as N


class DeviceSetup:
    """The stencil of `mesh` (an autan_b200.mesh.Mesh, or any object with its arrays and counts)
    computed on `device` at construction; `weights(bc_kind)` computes the weights there."""

    def __init__(self, mesh, device: int = 0):
        self._arrays = {
            "cell_face_offsets": np.ascontiguousarray(mesh.cell_face_offsets, dtype=np.int64),
            "cell_faces": np.ascontiguousarray(mesh.cell_faces, dtype=np.int32),
            "owner": np.ascontiguousarray(mesh.owner, dtype=np.int32),
            "neighbour": np.ascontiguousarray(mesh.neighbour, dtype=np.int32),
            "cell_centroid": np.ascontiguousarray(mesh.cell_centroid, dtype=np.float64),
            "face_centroid": np.ascontiguousarray(mesh.face_centroid, dtype=np.float64),
        }
        a = self._arrays
        m = N.SetupMesh()
        m.n_cells, m.n_owned_cells = mesh.n_cells, mesh.n_owned_cells
        m.n_faces, m.n_interior_faces = mesh.n_faces, mesh.n_interior_faces
        m.cell_face_offsets = N.ptr(a["cell_face_offsets"], C.c_int64)
        m.cell_faces = N.ptr(a["cell_faces"], C.c_int32)
        m.owner = N.ptr(a["owner"], C.c_int32)
        m.neighbour = N.ptr(a["neighbour"], C.c_int32)
        m.cell_centroid = N.ptr(a["cell_centroid"], C.c_double)
        m.face_centroid = N.ptr(a["face_centroid"], C.c_double)
        self.n_cells = mesh.n_cells
        self.n_boundary = mesh.n_faces - mesh.n_interior_faces
        self._handle = C.c_void_p()
        n = C.c_int64()
        err = N.errbuf()
        N.check(N.lib().autan_setup_device_create(C.byref(m), device, C.byref(self._handle),
                                                  C.byref(n), err, len(err)), err)  # fmt: skip
        self.n_stencil = int(n.value)

    def stencil(self) -> tuple[np.ndarray, np.ndarray]:
        """(offsets n_cells + 1, entries n_stencil) as the mesh contract writes them."""
        off = np.zeros(self.n_cells + 1, dtype=np.int64)
        ent = np.zeros(self.n_stencil, dtype=np.int32)
        err = N.errbuf()
        N.check(N.lib().autan_setup_device_download(self._handle, N.ptr(off, C.c_int64),
                                                    N.ptr(ent, C.c_int32), None, err, len(err)),
                err)  # fmt: skip
        return off, ent

    def weights(self, bc_kind) -> tuple[np.ndarray, int]:
        """The weights (3 x n_stencil FP64) for the boundary codes, and the number of cells that
        needed every boundary face in their fit."""
        kind = np.ascontiguousarray(bc_kind, dtype=np.uint8)
        if kind.size != self.n_boundary:
            raise ValueError("one boundary code per boundary face")
        retried = C.c_int64()
        err = N.errbuf()
        N.check(N.lib().autan_setup_device_weights(self._handle, N.ptr(kind, C.c_uint8),
                                                   C.byref(retried), err, len(err)), err)  # fmt: skip
        w = np.zeros((3, self.n_stencil), dtype=np.float64)
        N.check(N.lib().autan_setup_device_download(self._handle, None, None,
                                                    N.ptr(w, C.c_double), err, len(err)), err)  # fmt: skip
        return w, int(retried.value)

    def times(self) -> dict:
        """Device milliseconds: mesh arrays copied in, stencil, last weights."""
        ms = (C.c_double * 3)()
        N.lib().autan_setup_device_times(self._handle, ms)
        return {"copy_ms": ms[0], "stencil_ms": ms[1], "weights_ms": ms[2]}

    def close(self) -> None:
        if self._handle:
            N.lib().autan_setup_device_free(self._handle)
            self._handle = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
