"""The CPU samples of bench.py's reference arm and CPU baseline (bench.cpu_sample): built from the
committed compact meshes by the reference's own set-up code and the oracle's weights, they are the
same problems as the product's generators give (topology, geometry, stencil and weights bit for
bit), and the reference arm runs without loading this repository's native library."""

import json
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

import ref_setup as R

REPO = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(REPO))

pytestmark = pytest.mark.skipif(not R.available(), reason="oracle/_ref not built")


@pytest.mark.parametrize("workload", ["channel", "tets", "hex", "batch"])
def test_sample_equals_the_product_set_up(workload):
    import bench
    from autan_b200 import cases
    from autan_b200 import mesh as M

    md, sch, kind, data, u0, rk, cfl, local, owned = bench.cpu_sample(workload)
    if workload == "channel":
        case = cases.bump_channel(60, 20, 10, steps=1)
    elif workload == "tets":
        case = cases.vortex_tets(60, 24, 6, steps=1)
    elif workload == "hex":
        case = cases.vortex_hex(steps=1)
    else:
        b = cases.bump_batch(1, seed=0, cells=(20_000, 20_000))
        p = b.params[0]
        case = cases.Case("b", M.bump_channel(*p["boxes"], bump=p["bump"]), b.scheme, b.bc_kind,
                          b.bc_data, b.u0, rk=b.rk, cfl=b.cfl, steps=1, local=True)  # fmt: skip
    want = cases.oracle_mesh_dict(case)
    for k in ("owner", "neighbour", "cell_face_offsets", "cell_faces", "stencil_offsets", "stencil",
              "face_normal", "face_area_magnitude", "face_centroid", "cell_centroid",
              "cell_volume", "stencil_lsq_weight"):  # fmt: skip
        a, b_ = np.asarray(md[k]), np.asarray(want[k])
        assert a.shape == b_.shape, k
        if a.dtype.kind == "f":
            assert np.array_equal(a.view(np.uint64), b_.astype(np.float64).view(np.uint64)), k
        else:
            assert np.array_equal(a, b_), k
    assert sch == case.scheme.as_dict()
    assert np.array_equal(kind, case.bc_kind) and np.array_equal(data, case.bc_data)
    assert (rk, cfl, local) == (case.rk, case.cfl, case.local)
    assert np.allclose(u0[:, :owned], case.u0[:, :owned], rtol=1e-15, atol=1e-15)


def test_reference_arm_loads_no_native_library():
    code = ("import sys; sys.argv = ['bench.py', '--impl', 'reference', '--workload', 'hex', "
            "'--steps', '1', '--warmup', '3', '--cpu-threads', '1']; import bench; bench.main(); "
            "print('MAPS', 'libautan_b200' in open('/proc/self/maps').read())")  # fmt: skip
    r = subprocess.run([sys.executable, "-c", code], cwd=REPO, capture_output=True, text=True,
                       timeout=600)  # fmt: skip
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads([x for x in r.stdout.splitlines() if x.startswith("{")][0])
    assert line["impl"] == "reference" and line["value"] > 0
    assert "MAPS False" in r.stdout
