"""The product's set-up against the reference's own code run on the same meshes (oracle/_ref, built
from the reference's sources by `make -C oracle ref`): the face order and orientation of the mesh
contract (core/src/mesh.cpp:273 assemble), the FP64 geometry (core/src/geometry.cpp:120
compute_geometry: face area vectors, areas, centroids; owned cells' volumes and centroids), the
packed unit normals and face moments (codegen/cpp/geometry.cpp:166 pack_geometry) and the face2
stencil of every cell, ghosts included (codegen/cpp/geometry.cpp:432 cell_stencil): bit for bit.
The least-squares weights (physics/src/euler.cpp:340-416, restated in
autan_b200/csrc/setup_rules.cuh) against the reference's own face2 least-squares weights
(codegen/cpp/geometry.cpp:70 store_lsq_weights) with every boundary face in the fit: the same
normal matrix and weight formula, the inverse formed as cofactors times 1/det there and over det
here, and offsets within 64 ulps zeroed only here, so within 1e-12 of each cell's largest weight.
Meshes: periodic jittered Kuhn tetrahedra (ghost images), a jittered hexahedral box (warped faces:
non-zero moments), the hybrid bump channel (hexahedra, prisms, polyhedral bricks) and the periodic
hexahedral box. Skipped where oracle/_ref is not built."""

import numpy as np
import pytest

import ref_setup as R
from autan_b200 import cases
from autan_b200 import mesh as M

pytestmark = pytest.mark.skipif(not R.available(), reason="oracle/_ref not built")


def warped_hex():
    n, ext = (8, 6, 4), (1.0, 0.8, 0.5)
    return M.lattice("hexa", n, extent=ext, displacement=M.vortex_jitter(n, ext, 0.15, seed=3))


MESHES = {
    "tets": lambda: cases.vortex_tets(8, 8, 4).mesh,
    "warped_hex": warped_hex,
    "channel": lambda: cases.bump_channel(24, 10, 4).mesh,
    "periodic_hex": lambda: cases.vortex_hex(16, 16, 2).mesh,
}


def same_bits(a, b):
    a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
    return a.shape == b.shape and np.array_equal(a.view(np.uint64), b.view(np.uint64))


@pytest.fixture(scope="module", params=sorted(MESHES))
def pair(request):
    m = MESHES[request.param]()
    return request.param, m, R.reference_setup(m)


def test_assembly_order_and_topology(pair):
    _, m, r = pair
    assert np.array_equal(r["face_source"], np.arange(m.n_faces))
    assert not r["face_reversed"].any()
    assert list(r["counts"]) == [m.n_cells, m.n_owned_cells, m.n_faces, m.n_interior_faces,
                                 m.n_owned_interior_faces, m.n_owned_faces]  # fmt: skip
    for k in ("owner", "neighbour", "cell_face_offsets", "cell_faces"):
        assert np.array_equal(getattr(m, k), r[k]), k


def test_geometry_bit_for_bit(pair):
    name, m, r = pair
    for k in ("face_area", "face_area_magnitude", "face_centroid", "face_normal", "face_moment"):
        assert same_bits(getattr(m, k), r[k]), k
    no = m.n_owned_cells
    assert same_bits(m.cell_volume[:no], r["cell_volume"][:no])
    assert same_bits(m.cell_centroid[:, :no], r["cell_centroid"][:, :no])
    if name == "warped_hex":
        assert np.abs(r["face_moment"]).max() > 0.0  # the moments are exercised


def test_face2_stencil_bit_for_bit(pair):
    _, m, r = pair
    assert np.array_equal(m.stencil_offsets, r["stencil_offsets"])
    assert np.array_equal(m.stencil, r["stencil"])


def test_weights_against_the_reference_least_squares(pair):
    _, m, r = pair
    w = m.gradient_weights(np.zeros(m.n_boundary_faces, np.uint8))
    wr = r["stencil_lsq_weight"]
    so = m.stencil_offsets
    worst = 0.0
    for c in range(m.n_owned_cells):
        a, b = so[c], so[c + 1]
        scale = np.abs(wr[:, a:b]).max()
        worst = max(worst, float(np.abs(w[:, a:b] - wr[:, a:b]).max() / scale))
    assert worst <= 1e-12, worst
