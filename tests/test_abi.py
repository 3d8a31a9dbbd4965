"""The native library without a GPU: it loads, exports every entry point its headers declare, and
its host set-up builds meshes that satisfy the mesh contract."""

import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from autan_b200 import _native as N
from autan_b200 import mesh as M

INCLUDE = Path(__file__).resolve().parent.parent / "include"


def declared(header: Path) -> list[str]:
    text = re.sub(r"/\*.*?\*/", "", header.read_text(), flags=re.S)
    return sorted(set(re.findall(r"\b(autan_[a-z0-9_]+)\s*\(", text)))


@pytest.mark.parametrize("header", sorted(INCLUDE.glob("*.h")), ids=lambda p: p.name)
def test_exports_every_declared_symbol(header):
    lib = C.CDLL(str(N.LIB_PATH))
    names = declared(header)
    assert names
    for n in names:
        assert hasattr(lib, n), n


def test_create_without_device_reports_an_error():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    m = M.periodic_box_hex(4, 4, 2, extent=(1, 1, 0.5))
    from autan_b200.euler import EulerDevice, Scheme

    with pytest.raises(N.NativeError) as e:
        EulerDevice(m, Scheme(second_order=False))
    assert str(e.value).startswith("E1")


def test_lattice_contract():
    m = M.jittered_tets(6, 5, 3, extent=(1.2, 1.0, 0.6), rcm=True)
    ni, nf, no = m.n_interior_faces, m.n_faces, m.n_owned_cells
    own, nei = m.owner, m.neighbour
    assert np.all(own[:ni] < nei)
    key = own[:ni].astype(np.int64) * m.n_cells + nei
    assert np.all(np.diff(key) >= 0)
    assert np.all(own[: m.n_owned_interior_faces] < no)
    assert np.all(own[m.n_owned_interior_faces : ni] >= no)
    assert np.all(own[ni : m.n_owned_faces] < no) and np.all(own[m.n_owned_faces :] >= no)
    # every cell's faces in increasing order
    off, cf = m.cell_face_offsets, m.cell_faces
    for c in range(m.n_cells):
        assert np.all(np.diff(cf[off[c] : off[c + 1]]) > 0)
    # closed owned cells
    acc = np.zeros((3, m.n_cells))
    np.add.at(acc, (slice(None), own), m.face_area)
    np.add.at(acc, (slice(None), nei), -m.face_area[:, :ni])
    assert np.abs(acc[:, :no]).max() < 1e-14
    # images: the owned cell's centroid shifted by the translation
    g = m.ghost_owner
    shifted = m.cell_centroid[:, g] + m.ghost_translation
    assert np.array_equal(m.cell_centroid[:, no:], shifted)
    assert m.cell_volume[:no].sum() == pytest.approx(1.2 * 1.0 * 0.6, rel=1e-12)


def test_face2_stencil_and_weights_reproduce_linear_fields():
    """The LSQ weights are exact for linear fields (every cell's fit keeps enough entries)."""
    m = M.jittered_tets(5, 5, 3, extent=(1.0, 1.0, 0.6))
    kind = np.zeros(m.n_boundary_faces, dtype=np.uint8)  # `state` faces: kept in the fits
    w = m.gradient_weights(kind)
    a = np.array([0.3, -1.2, 0.7])
    xc = m.cell_centroid
    xf = m.face_centroid
    so, st = m.stencil_offsets, m.stencil
    for c in range(m.n_owned_cells):
        g = np.zeros(3)
        for k in range(so[c], so[c + 1]):
            e = st[k]
            x = xc[:, e] if e >= 0 else xf[:, -e - 1]
            g += (a @ (x - xc[:, c])) * w[:, k]
        assert np.allclose(g, a, rtol=1e-9, atol=1e-9)


def test_boundary_code_out_of_range():
    m = M.periodic_box_hex(4, 4, 2, extent=(1, 1, 0.5))
    with pytest.raises(N.NativeError):
        m.gradient_weights(np.full(m.n_boundary_faces, 9, dtype=np.uint8))


def test_bump_channel_contract():
    """The hybrid channel: closed cells of positive volume filling the channel, hexahedra, prisms
    and polyhedral bricks present, planar faces, zones on the six sides, LSQ weights exact for
    linear fields with every boundary face kept."""
    m = M.bump_channel(18, 12, 3, order="morton")
    ni, no = m.n_interior_faces, m.n_owned_cells
    assert m.n_cells == no and m.all_planar
    nfaces = np.diff(m.cell_face_offsets)
    # 6 faces: hex; 5: prism; 8 to 10: bricks (one or two faces per side, hexagonal ends)
    assert set(np.unique(nfaces)) >= {5, 6} and nfaces.max() >= 8
    acc = np.zeros((3, m.n_cells))
    np.add.at(acc, (slice(None), m.owner), m.face_area)
    np.add.at(acc, (slice(None), m.neighbour), -m.face_area[:, :ni])
    assert np.abs(acc).max() < 1e-14
    assert np.all(m.cell_volume > 0)
    xs = np.linspace(0.0, 3.0, 200001)
    area = np.trapezoid(1.0 - 0.05 * np.exp(-25 * (xs - 1.5) ** 2), xs)
    assert m.cell_volume.sum() == pytest.approx(0.5 * area, rel=1e-4)
    assert set(np.unique(m.boundary_zone)) == {0, 1, 2, 3, 4, 5}
    kind = np.zeros(m.n_boundary_faces, dtype=np.uint8)
    w = m.gradient_weights(kind)
    a = np.array([0.3, -1.2, 0.7])
    xc, xf = m.cell_centroid, m.face_centroid
    so, st = m.stencil_offsets, m.stencil
    for c in range(no):
        g = np.zeros(3)
        for k in range(so[c], so[c + 1]):
            e = st[k]
            x = xc[:, e] if e >= 0 else xf[:, -e - 1]
            g += (a @ (x - xc[:, c])) * w[:, k]
        assert np.allclose(g, a, rtol=1e-9, atol=1e-9)
