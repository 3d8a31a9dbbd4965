"""autan_exact_rms_static, the exact-sum RMS whose scratch is module-level device memory: its
argument checks (no GPU needed), and on the GPU two calls in a row against the residual norms of
autan_euler_device_evaluate on the same residual, bit for bit. The file is named to be collected
last, so that the GPU test also runs after every other test has used the device."""

import ctypes as C

import numpy as np
import pytest

from autan_b200 import _native as N
from autan_b200 import cases
from autan_b200.euler import EulerDevice


def call(values, n, stride, components, rms, stream=None):
    err = N.errbuf()
    rc = N.lib().autan_exact_rms_static(values, n, stride, components, rms, stream, err, len(err))
    return rc, err.value.decode()


@pytest.mark.parametrize(
    "n, stride, components, code",
    [
        (0, 0, 5, "E1101: n must be positive"),
        ((1 << 30) + 1, (1 << 30) + 1, 5, "E1101: n above 2^30"),
        (10, 10, 0, "E1101: components must be 1 to 8"),
        (10, 10, 9, "E1101: components must be 1 to 8"),
        (10, 9, 2, "E1101: stride below n"),
    ],
)
def test_limits_are_refused_before_device_work(n, stride, components, code):
    # The pointers are never dereferenced: every case fails its checks first.
    rc, msg = call(C.c_void_p(16), n, stride, components, C.c_void_p(16))
    assert rc == 1
    assert msg.startswith(code), msg


def test_null_pointers_are_refused():
    rc, msg = call(None, 10, 10, 5, C.c_void_p(16))
    assert rc == 1 and msg.startswith("E1101: null argument")


@pytest.mark.gpu
@pytest.mark.parametrize("which", ["hex_fp64", "tets_fp32"])
def test_static_rms_matches_evaluate_twice(which):
    import torch

    case = cases.vortex_hex(16, 16, 2) if which == "hex_fp64" else cases.vortex_tets(24, 24, 6)
    with EulerDevice(case.mesh, case.scheme, bc_kind=case.bc_kind, bc_data=case.bc_data) as dev:
        dev.upload(case.u0)
        expected = np.array(dev.evaluate().residuals)
        res = dev.residual(case.u0)  # 5 x n_cells, images' rows zero
    n, nc = case.mesh.n_owned_cells, case.mesh.n_cells
    values = torch.from_numpy(np.ascontiguousarray(res)).to("cuda:0")
    out = torch.full((2, 5), -1.0, dtype=torch.float64, device="cuda:0")
    stream = torch.cuda.current_stream(0).cuda_stream
    for k in range(2):
        rc, msg = call(C.c_void_p(values.data_ptr()), n, nc, 5,
                       C.c_void_p(out[k].data_ptr()), C.c_void_p(stream))  # fmt: skip
        assert rc == 0, msg
    torch.cuda.synchronize(0)
    got = out.cpu().numpy()
    assert np.count_nonzero(expected) >= 4  # z-momentum is zero on the hexahedral box
    for k in range(2):
        assert np.array_equal(got[k], expected), (got[k], expected)
