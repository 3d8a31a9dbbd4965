"""The gradient set-up on the GPU (autan_setup_device_*) against the host set-up: the face2
stencil and the least-squares weights bit for bit, on the periodic tetrahedra (ghost cells), the
hybrid bump channel (boundary faces excluded from and retried into the fits) and the hexahedral
box, and on the full 2 073 600-cell benchmark lattice."""

import numpy as np
import pytest

from autan_b200 import cases
from autan_b200.setup_device import DeviceSetup

pytestmark = pytest.mark.gpu


def same_bits(a, b):
    return a.shape == b.shape and np.array_equal(a.view(np.uint64), b.view(np.uint64))


@pytest.mark.parametrize("which", ["tets", "channel", "hex", "tets_full"])
def test_device_setup_equals_the_host(which):
    case = {"tets": lambda: cases.vortex_tets(12, 12, 6),
            "channel": lambda: cases.bump_channel(40, 16, 6),
            "hex": lambda: cases.vortex_hex(16, 16, 2),
            "tets_full": lambda: cases.vortex_tets()}[which]()
    m = case.mesh
    with DeviceSetup(m) as s:
        off, ent = s.stencil()
        assert np.array_equal(off, m.stencil_offsets)
        assert np.array_equal(ent, m.stencil)
        for kind in (np.ascontiguousarray(case.bc_kind, np.uint8),
                     np.zeros(m.n_boundary_faces, np.uint8)):
            w, _ = s.weights(kind)
            assert same_bits(w, m.gradient_weights(kind))


def test_device_setup_retries_as_the_host():
    """A one-cell-thick slab with slip faces all round: every cell's first fit is singular and the
    retry with every boundary face gives the host's weights on the device too."""
    from autan_b200 import mesh as M

    m = M.lattice("hexa", (9, 7, 1), extent=(1.0, 0.8, 0.2))
    kind = np.full(m.n_boundary_faces, 2, dtype=np.uint8)
    with DeviceSetup(m) as s:
        w, retried = s.weights(kind)
    assert retried == m.n_owned_cells
    assert same_bits(w, m.gradient_weights(kind))
