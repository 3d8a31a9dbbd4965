"""The meshes and cases of the CPU baseline samples, written once as compact face-based inputs
(tests/golden/samples/cpu_sample_<name>.npz) so that the reference arm of bench.py and its CPU
baseline build their problem without this repository's native library: at run time the reference's own
mesh assembly, geometry and face2 stencil (oracle/_ref) and the oracle's least-squares weights
set the sample up from these arrays, and the oracle steps it.

    python tests/golden/make_cpu_samples.py

Samples (one per benchmark workload, the same generators and schemes at a size one host thread
steps in seconds):
  channel  the hybrid bump channel of 60 x 20 x 10 boxes (the 8.0 M-cell workload's generator and
           scheme: AUSM+-up, total-pressure inlet, static-pressure outlet, slip walls, local steps)
  tets     a 60 x 24 x 6 periodic slab of the jittered Kuhn-tetrahedra lattice at its cell size
           (HLLC, SSP-RK3, CFL 0.8), the vortex centred in the slab
  hex      the 8 192-cell periodic hexahedral vortex (first-order Roe, classical RK4, fp64)
  batch    the first channel of the batched workload (seed 0) drawn at 20 000 cells (Roe,
           farfield inflow and outflow)
Each file: points (3 x n_points), face_node_offsets, face_nodes, cell0 / cell1 per face (cell1 -1
on boundary faces), face_zone, n_cells, n_ghost, ghost_owner, ghost_translation (3 x n_ghost),
the scheme (JSON), bc_kind, bc_data (5 x boundary faces), rk, cfl, local, and the start: uniform
(5 conserved values) or the isentropic vortex (beta, centre)."""

import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

from autan_b200 import cases  # noqa: E402


def write(name: str, case, start: dict) -> None:
    m = case.mesh
    cell1 = np.full(m.n_faces, -1, dtype=np.int32)
    cell1[: m.n_interior_faces] = m.neighbour
    n_ghost = m.n_cells - m.n_owned_cells
    np.savez_compressed(
        HERE / "samples" / f"cpu_sample_{name}.npz",
        points=m.points, face_node_offsets=m.face_node_offsets, face_nodes=m.face_nodes,
        cell0=m.owner, cell1=cell1, face_zone=m.face_zone, n_cells=m.n_cells, n_ghost=n_ghost,
        ghost_owner=m.ghost_owner if n_ghost else np.zeros(0, np.int32),
        ghost_translation=m.ghost_translation if n_ghost else np.zeros((3, 0)),
        scheme=json.dumps(case.scheme.as_dict()), bc_kind=case.bc_kind, bc_data=case.bc_data,
        rk=case.rk, cfl=case.cfl, local=case.local, start=json.dumps(start),
    )  # fmt: skip


def main() -> None:
    ch = cases.bump_channel(60, 20, 10, steps=1)
    write("channel", ch, {"uniform": [float(x) for x in ch.u0[:, 0]]})
    t = cases.vortex_tets(60, 24, 6, steps=1, precision="fp32+acc64")
    h = 10.0 / 240
    write("tets", t, {"vortex": {"beta": 5.0, "centre": [60 * h / 2, 24 * h / 2]}})
    x = cases.vortex_hex(steps=1)
    write("hex", x, {"vortex": {"beta": 5.0, "centre": [5.0, 5.0]}})
    b = cases.bump_batch(1, seed=0, cells=(20_000, 20_000))
    p = b.params[0]
    from autan_b200 import mesh as M

    m = M.bump_channel(*p["boxes"], bump=p["bump"])
    bc = cases.Case("batch", m, b.scheme, b.bc_kind, b.bc_data, b.u0, rk=b.rk, cfl=b.cfl, steps=1,
                    local=True)  # fmt: skip
    write("batch", bc, {"uniform": [float(v) for v in b.u0[:, 0]]})


if __name__ == "__main__":
    main()
