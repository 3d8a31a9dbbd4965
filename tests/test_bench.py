"""bench.py's host-side bookkeeping that needs no GPU: the committed DRAM traffic per launch,
looked up by kernel kind and mesh family and scaled to the workload's cells."""

import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(REPO))

import bench  # noqa: E402


def test_traffic_is_per_mesh_family_and_scales_with_cells():
    tets = bench.committed_traffic("gradients", 1_016_064, "tets")
    channel = bench.committed_traffic("gradients", 994_600, "channel")
    assert tets == pytest.approx(445_897_813)
    assert channel == pytest.approx(664_242_005)
    # the channel's longer stencils (about 23 entries per cell, 13.8 on the tets) read more
    assert channel / 994_600 > 1.4 * tets / 1_016_064
    assert bench.committed_traffic("gradients", 2 * 994_600, "channel") == pytest.approx(2 * channel)
    assert bench.committed_traffic("faces", 1000, "tets") is None
    assert bench.committed_traffic("gradients", 1000, "hex") is None
