"""The ctypes mirrors of the C ABI's structures (autan_b200/_native.py) against the headers: every
field's offset and every structure's size as a C compiler lays them out (gcc on the headers in
include/), so that a field added or moved on one side only fails here, on the CPU."""

import ctypes as C
import subprocess
from pathlib import Path

import pytest

from autan_b200 import _native as N

REPO = Path(__file__).resolve().parent.parent

PAIRS = {
    "autan_lattice": (N.Lattice, "autan_b200_setup.h"),
    "autan_bump_channel": (N.BumpChannel, "autan_b200_setup.h"),
    "autan_setup_mesh": (N.SetupMesh, "autan_b200_setup.h"),
    "autan_euler_scheme": (N.Scheme, "autan_euler_device.h"),
    "autan_euler_mesh": (N.MeshArrays, "autan_euler_device.h"),
    "autan_euler_step_result": (N.StepResult, "autan_euler_device.h"),
    "autan_march_result": (N.MarchResult, "autan_euler_device.h"),
    "autan_euler_ranks": (N.Ranks, "autan_euler_device.h"),
}


@pytest.fixture(scope="module")
def c_layout(tmp_path_factory):
    """struct -> (sizeof, {field: offsetof}) from a C program compiled against the headers."""
    lines = ["#include <stddef.h>", "#include <stdio.h>"]
    for h in sorted({h for _, h in PAIRS.values()}):
        lines.append(f'#include "{h}"')
    lines.append("int main(void) {")
    for name, (cls, _) in PAIRS.items():
        lines.append(f'  printf("{name} size %zu\\n", sizeof(struct {name}));')
        for field, *_ in cls._fields_:
            lines.append(f'  printf("{name} {field} %zu\\n", offsetof(struct {name}, {field}));')
    lines.append("  return 0;\n}")
    d = tmp_path_factory.mktemp("abi")
    src, exe = d / "layout.c", d / "layout"
    src.write_text("\n".join(lines) + "\n")
    subprocess.run(["gcc", "-std=c11", f"-I{REPO / 'include'}", str(src), "-o", str(exe)],
                   check=True)  # fmt: skip
    out: dict = {}
    for line in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines():
        name, field, value = line.split()
        size, fields = out.setdefault(name, [None, {}])
        if field == "size":
            out[name][0] = int(value)
        else:
            fields[field] = int(value)
    return out


@pytest.mark.parametrize("name", list(PAIRS))
def test_ctypes_mirror_matches_the_header(name, c_layout):
    cls, _ = PAIRS[name]
    size, fields = c_layout[name]
    assert C.sizeof(cls) == size, name
    for field, *_ in cls._fields_:
        assert getattr(cls, field).offset == fields[field], (name, field)
