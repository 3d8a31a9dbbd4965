"""The reference-side DeviceStepper<P> adapter (autan_b200/adapter/euler_device_b200.cpp) compiles
against the reference's own headers (physics/include/autan/physics/euler_device.hpp and what it
includes), syntax only, both precision policies instantiated: `make -C oracle adapter-check`.
Skipped where the reference tree is absent."""

import subprocess
from pathlib import Path

import pytest

ORACLE = Path(__file__).resolve().parent.parent / "oracle"


def reference_present() -> bool:
    out = subprocess.run(["make", "-s", "-C", str(ORACLE), "has-ref"], capture_output=True, text=True)
    return out.stdout.strip() == "1"


@pytest.mark.skipif(not reference_present(), reason="the reference tree is not here")
def test_adapter_compiles_against_the_reference_headers():
    out = subprocess.run(["make", "-s", "-C", str(ORACLE), "adapter-check"], capture_output=True,
                         text=True)  # fmt: skip
    assert out.returncode == 0, out.stderr[-2000:]
