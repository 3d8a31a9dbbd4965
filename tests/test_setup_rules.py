"""The boundary rule of the least-squares weights (physics/src/euler.cpp:340-416, restated in
autan_b200/csrc/setup_rules.cuh): a boundary face enters a cell's fit only where its condition
fixes the state there (kind 0), unless the cell's other entries leave the fit singular, in which
case every boundary face enters. Checked on the hybrid channel with its own conditions (inlet,
outlet, slip walls) and with the slip walls made state faces, against a numpy fit of the same
entries; the kept fits reproduce linear fields."""

import numpy as np
import pytest

from autan_b200 import cases


def offsets(m, c, k):
    e = m.stencil[k]
    x = m.cell_centroid[:, e] if e >= 0 else m.face_centroid[:, -e - 1]
    return x - m.cell_centroid[:, c]


def singular(ds):
    a = np.zeros((3, 3))
    for d in ds:
        a += np.outer(d, d) / (d @ d)
    return not abs(np.linalg.det(a)) > 1e-10 * abs(a[0, 0] * a[1, 1] * a[2, 2])


@pytest.mark.parametrize("walls_as_state", [False, True])
def test_boundary_faces_enter_the_fit_by_their_condition(walls_as_state):
    case = cases.bump_channel(30, 12, 4)
    m = case.mesh
    kind = np.ascontiguousarray(case.bc_kind, np.uint8).copy()
    if walls_as_state:
        kind[kind == 2] = 0
    w = m.gradient_weights(kind)
    ni = m.n_interior_faces
    so = m.stencil_offsets
    a = np.array([0.3, -1.2, 0.7])
    retried = 0
    for c in range(m.n_owned_cells):
        ks = range(so[c], so[c + 1])
        excluded = [k for k in ks if m.stencil[k] < 0 and kind[-m.stencil[k] - 1 - ni] != 0]
        kept = [k for k in ks if k not in excluded]
        if any(np.any(w[:, k] != 0) for k in excluded):
            # the retry: only where the fit without those faces is singular
            assert singular([offsets(m, c, k) for k in kept])
            retried += 1
            kept = list(ks)
        g = sum((a @ offsets(m, c, k)) * w[:, k] for k in kept)
        assert np.allclose(g, a, rtol=1e-9, atol=1e-9)
    print("cells that needed every boundary face:", retried)


def test_one_layer_slab_retries_with_every_boundary_face():
    """A one-cell-thick slab with slip faces on every side: without its boundary faces a cell's fit
    has no offset across the layer and is singular, so every cell takes all of them."""
    from autan_b200 import mesh as M

    m = M.lattice("hexa", (5, 4, 1), extent=(1.0, 0.8, 0.2))
    kind = np.full(m.n_boundary_faces, 2, dtype=np.uint8)
    w = m.gradient_weights(kind)
    so = m.stencil_offsets
    a = np.array([0.3, -1.2, 0.7])
    for c in range(m.n_owned_cells):
        ks = range(so[c], so[c + 1])
        cells_only = [k for k in ks if m.stencil[k] >= 0]
        assert singular([offsets(m, c, k) for k in cells_only])
        assert any(np.any(w[:, k] != 0) for k in ks if m.stencil[k] < 0)
        g = sum((a @ offsets(m, c, k)) * w[:, k] for k in ks)
        assert np.allclose(g, a, rtol=1e-9, atol=1e-9)
