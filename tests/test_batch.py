"""Batched cases as one union mesh (cases.union, cases.bump_batch), on the oracle (CPU): the union
keeps the mesh contract, and its residual is each case's own residual, bit for bit."""

import numpy as np

import oracle as O
from autan_b200 import cases
from autan_b200 import mesh as M


def small_batch(precision="fp64"):
    return cases.bump_batch(3, seed=2, cells=(800, 3000), precision=precision, inlet="state")


def test_union_keeps_the_mesh_contract():
    b = small_batch()
    m = b.mesh
    ni, nf = m["n_interior_faces"], m["n_faces"]
    own, nei = m["owner"], m["neighbour"]
    assert np.all(own[:ni] < nei)
    key = own[:ni].astype(np.int64) * m["n_cells"] + nei
    assert np.all(np.diff(key) > 0)
    off, cf = m["cell_face_offsets"], m["cell_faces"]
    for c in range(m["n_cells"]):
        faces = cf[off[c] : off[c + 1]]
        assert np.all(np.diff(faces) > 0)
        assert np.all((own[faces] == c) | ((faces < ni) & (nei[np.minimum(faces, ni - 1)] == c)))
    acc = np.zeros((3, m["n_cells"]))
    np.add.at(acc, (slice(None), own), m["face_area"])
    np.add.at(acc, (slice(None), nei), -m["face_area"][:, :ni])
    assert np.abs(acc).max() < 1e-14
    st = m["stencil"]
    assert np.all(st < m["n_cells"]) and np.all(-st - 1 < nf)
    assert np.all((-st[st < 0] - 1) >= ni)  # boundary entries name boundary faces
    assert b.weights.shape == (3, st.size)


def test_union_residual_is_each_cases_residual():
    b = small_batch()
    o = O.Oracle(b.mesh, b.scheme.as_dict(), b.bc_kind, b.bc_data)
    u = b.u0 * (1.0 + 1e-3 * np.sin(np.arange(b.n_cells))[None, :])
    res = o.residual(u)
    nb_off = 0
    for k in range(3):
        c0, c1 = b.cell_offsets[k], b.cell_offsets[k + 1]
        p = b.params[k]
        m = M.bump_channel(*p["boxes"], bump=p["bump"])
        nb = m.n_boundary_faces
        kind = b.bc_kind[nb_off : nb_off + nb]
        data = b.bc_data[:, nb_off : nb_off + nb]
        nb_off += nb
        md = cases.oracle_mesh_dict(cases.Case("k", m, b.scheme, kind, data, u[:, c0:c1], 3, 1.5,
                                               1, True))  # fmt: skip
        ok = O.Oracle(md, b.scheme.as_dict(), kind, data)
        want = ok.residual(np.ascontiguousarray(u[:, c0:c1]))
        assert np.array_equal(res[:, c0:c1].view(np.int64), want.view(np.int64))


def test_oracle_takes_no_moments_for_a_planar_union():
    """A planar batch's union mesh carries no face moments (an empty array); the oracle must get a
    NULL pointer for them, not a stand-in element: its set-up reads 9 x n_faces moments from any
    pointer it is given."""
    b = cases.bump_batch(2, seed=0, cells=(300, 500))
    assert b.mesh["all_planar"] and np.asarray(b.mesh["face_moment"]).size == 0
    o = O.Oracle(b.mesh, b.scheme.as_dict(), b.bc_kind, b.bc_data)
    assert not o.mesh.face_moment  # NULL
    u = b.u0.copy()
    o.step(u, rk=3, cfl=b.cfl, local=True)
    assert np.all(np.isfinite(u))
