"""ctypes binding of the in-tree native library (autan_b200/_lib/libautan_b200.so).

There is no fallback: a missing library is an error, so that nothing runs on another code path
by accident. Build it with `python -m autan_b200.build`.
"""

from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

# The in-tree build, or another build of the same sources named by AUTAN_B200_LIB.
LIB_PATH = Path(os.environ.get("AUTAN_B200_LIB") or
                Path(__file__).resolve().parent / "_lib" / "libautan_b200.so")

_lib: C.CDLL | None = None

i32, i64, u8, f64, vp, sz = C.c_int32, C.c_int64, C.c_uint8, C.c_double, C.c_void_p, C.c_size_t
P = C.POINTER


class NativeError(RuntimeError):
    """An error reported through the C ABI ("Exxxx: message")."""


class Lattice(C.Structure):
    _fields_ = [
        ("fill", i32),
        ("nx", i32),
        ("ny", i32),
        ("nz", i32),
        ("origin", f64 * 3),
        ("extent", f64 * 3),
        ("periodic", i32 * 3),
        ("zone", i32 * 6),
        ("displacement", P(f64)),
        ("rcm", i32),
    ]


class BumpChannel(C.Structure):
    """struct autan_bump_channel of include/autan_b200_setup.h."""

    _fields_ = [
        ("nx", i32),
        ("ny", i32),
        ("nz", i32),
        ("extent", f64 * 3),
        ("bump", f64),
        ("ratio", f64),
        ("stretched", i32),
        ("prism_rows", i32 * 2),
        ("brick_rows", i32 * 2),
        ("brick_cols", i32 * 2),
        ("order", i32),
    ]


class Scheme(C.Structure):
    """struct autan_euler_scheme of include/autan_euler_device.h."""

    _fields_ = [
        ("flux", i32),
        ("second_order", i32),
        ("limiter", i32),
        ("precision", i32),
        ("planar", i32),
        ("gamma", f64),
        ("gas_constant", f64),
        ("venkat_k", f64),
        ("length", f64),
        ("mach_ref", f64),
        ("scale", f64 * 5),
        ("reference", f64 * 5),
    ]


class SetupMesh(C.Structure):
    """struct autan_setup_mesh of include/autan_b200_setup.h."""

    _fields_ = [
        ("n_cells", i32),
        ("n_owned_cells", i32),
        ("n_faces", i32),
        ("n_interior_faces", i32),
        ("cell_face_offsets", P(i64)),
        ("cell_faces", P(i32)),
        ("owner", P(i32)),
        ("neighbour", P(i32)),
        ("cell_centroid", P(f64)),
        ("face_centroid", P(f64)),
    ]


class MeshArrays(C.Structure):
    """struct autan_euler_mesh of include/autan_euler_device.h."""

    _fields_ = [
        ("n_cells", i32),
        ("n_owned_cells", i32),
        ("n_faces", i32),
        ("n_interior_faces", i32),
        ("n_owned_interior_faces", i32),
        ("n_owned_faces", i32),
        ("owner", P(i32)),
        ("neighbour", P(i32)),
        ("cell_face_offsets", P(i64)),
        ("cell_faces", P(i32)),
        ("ghost_owner", P(i32)),
        ("face_normal", P(f64)),
        ("face_area_magnitude", P(f64)),
        ("face_centroid", P(f64)),
        ("face_moment", P(f64)),
        ("cell_centroid", P(f64)),
        ("cell_volume", P(f64)),
        ("stencil_offsets", P(i64)),
        ("stencil", P(i32)),
        ("stencil_lsq_weight", P(f64)),
    ]


class StepResult(C.Structure):
    """struct autan_euler_step_result of include/autan_euler_device.h."""

    _fields_ = [
        ("residuals", f64 * 5),
        ("time_step", f64),
        ("invalid_cell", i64),
        ("steps", i64),
    ]


class MarchResult(C.Structure):
    """struct autan_march_result of include/autan_euler_device.h."""

    _fields_ = [
        ("iterations", i64),
        ("steps", i64),
        ("converged", i32),
        ("plateau_mask", i32),
        ("first", f64 * 5),
        ("last", f64 * 5),
        ("time_step", f64),
        ("gpu_ms", f64),
        ("invalid_cell", i64),
    ]


# Callbacks of struct autan_euler_ranks.
EXCHANGE_FN = C.CFUNCTYPE(i32, vp, i32, i64, vp)
REDUCE_FN = C.CFUNCTYPE(i32, vp, i32, i64, vp)


class Ranks(C.Structure):
    """struct autan_euler_ranks of include/autan_euler_device.h."""

    _fields_ = [
        ("user", vp),
        ("exchange", EXCHANGE_FN),
        ("reduce", REDUCE_FN),
        ("send", vp),
        ("recv", vp),
        ("words", vp),
        ("n_send", i64),
        ("send_cells", P(i32)),
        ("global_cells", f64),
    ]


def _bind(lib: C.CDLL) -> None:
    def fn(name: str, res, *args):
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = list(args)

    fn("autan_mesh_build_lattice", C.c_int, P(Lattice), P(vp), C.c_char_p, sz)
    fn("autan_mesh_build_cells", C.c_int, i64, P(f64), i64, P(i64), P(i64), P(i32), P(i32), i32,
       P(vp), C.c_char_p, sz)  # fmt: skip
    fn("autan_mesh_build_bump_channel", C.c_int, P(BumpChannel), P(vp), C.c_char_p, sz)
    fn("autan_mesh_free", None, vp)
    fn("autan_convergence_iteration", C.c_int, P(f64), i64, f64, P(f64), P(i64), P(i32), C.c_char_p,
       sz)  # fmt: skip
    fn("autan_mesh_counts", None, vp, P(i64))
    fn("autan_mesh_array", C.c_int, vp, C.c_char_p, P(vp), P(i64), P(i32))
    fn("autan_mesh_gradient_weights", C.c_int, vp, P(u8), P(f64), C.c_char_p, sz)
    if hasattr(lib, "autan_euler_device_create"):
        fn("autan_euler_device_create", C.c_int, P(MeshArrays), P(Scheme), i32, vp, P(vp),
           C.c_char_p, sz)  # fmt: skip
        fn("autan_euler_device_destroy", None, vp)
        fn("autan_euler_device_set_boundary", C.c_int, vp, P(u8), P(f64), i64, C.c_char_p, sz)
        fn("autan_euler_device_set_boundary_data", C.c_int, vp, P(f64), i64, C.c_char_p, sz)
        fn("autan_euler_device_set_source", C.c_int, vp, P(f64), C.c_char_p, sz)
        fn("autan_euler_device_set_second_order", C.c_int, vp, i32, C.c_char_p, sz)
        fn("autan_euler_device_upload", C.c_int, vp, P(f64), C.c_char_p, sz)
        fn("autan_euler_device_download", C.c_int, vp, P(f64), C.c_char_p, sz)
        fn("autan_euler_device_residual", C.c_int, vp, P(f64), P(f64), C.c_char_p, sz)
        fn("autan_euler_device_step", C.c_int, vp, f64, f64, i32, i32, i64, i32, P(StepResult),
           C.c_char_p, sz)  # fmt: skip
        fn("autan_euler_device_evaluate", C.c_int, vp, P(StepResult), C.c_char_p, sz)
        fn("autan_euler_device_sync", C.c_int, vp, C.c_char_p, sz)
        fn("autan_euler_device_set_stall_test", C.c_int, vp, i32, C.c_char_p, sz)
        fn("autan_euler_device_set_ranks", C.c_int, vp, P(Ranks), C.c_char_p, sz)
        fn("autan_euler_device_external_ghosts", C.c_int, vp, P(i64), C.c_char_p, sz)
        fn("autan_euler_device_stream", vp, vp)
        fn("autan_euler_device_counters", C.c_int, vp, P(i64), C.c_char_p, sz)
        fn("autan_euler_device_gradients", C.c_int, vp, P(f64), P(f64), C.c_char_p, sz)
        fn("autan_euler_device_time_steps", C.c_int, vp, f64, P(f64), C.c_char_p, sz)
        fn("autan_euler_device_history", C.c_int, vp, i64, P(f64), P(f64), C.c_char_p, sz)
        fn("autan_euler_device_set_tuning", C.c_int, vp, P(i32), i32, C.c_char_p, sz)
        fn("autan_euler_device_get_tuning", C.c_int, vp, P(i32), i32, C.c_char_p, sz)
        fn("autan_euler_device_autotune", C.c_int, vp, f64, f64, i32, i32, i32, P(i32), P(f64),
           C.c_char_p, sz)  # fmt: skip
        fn("autan_euler_device_kernel_times", C.c_int, vp, f64, f64, i32, i32, i64, P(f64), P(i64),
           C.c_char_p, sz)  # fmt: skip
        fn("autan_euler_device_face_parts", C.c_int, vp, P(f64), P(f64), P(f64), C.c_char_p, sz)
        fn("autan_euler_device_boundary_pressure", C.c_int, vp, P(f64), P(f64), P(f64), C.c_char_p,
           sz)  # fmt: skip
        fn("autan_euler_device_conservation", C.c_int, vp, P(f64), P(i32), C.c_char_p, sz)
        fn("autan_euler_device_march", C.c_int, vp, f64, f64, i32, i32, i64, i32, f64, P(f64),
           P(MarchResult), C.c_char_p, sz)  # fmt: skip
        fn("autan_euler_device_set_cases", C.c_int, vp, i32, P(i64), C.c_char_p, sz)
        fn("autan_euler_device_set_active", C.c_int, vp, P(u8), C.c_char_p, sz)
        fn("autan_euler_device_set_case_mach_ref", C.c_int, vp, P(f64), C.c_char_p, sz)
        fn("autan_euler_device_case_history", C.c_int, vp, i64, P(f64), C.c_char_p, sz)
        fn("autan_euler_device_march_cases", C.c_int, vp, f64, f64, i32, i32, i64, i32, f64, P(f64),
           P(f64), P(i64), P(i32), P(f64), P(i64), P(f64), P(f64), C.c_char_p, sz)  # fmt: skip
    if hasattr(lib, "autan_setup_device_create"):
        fn("autan_setup_device_create", C.c_int, P(SetupMesh), i32, P(vp), P(i64), C.c_char_p, sz)
        fn("autan_setup_device_weights", C.c_int, vp, P(u8), P(i64), C.c_char_p, sz)
        fn("autan_setup_device_download", C.c_int, vp, P(i64), P(i32), P(f64), C.c_char_p, sz)
        fn("autan_setup_device_times", None, vp, P(f64))
        fn("autan_setup_device_free", None, vp)
    if hasattr(lib, "autan_exact_rms_static"):
        fn("autan_exact_rms_static", C.c_int, vp, i64, i64, i32, vp, vp, C.c_char_p, sz)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise NativeError(
                f"E1104: native library missing at {LIB_PATH}; build it with "
                "`python -m autan_b200.build`"
            )
        _lib = C.CDLL(str(LIB_PATH))
        _bind(_lib)
    return _lib


def check(rc: int, err: C.Array) -> None:
    if rc != 0:
        raise NativeError(err.value.decode(errors="replace") or f"native call failed ({rc})")


def errbuf() -> C.Array:
    return C.create_string_buffer(512)


def ptr(a, ctype):
    """Pointer to a contiguous numpy array's data (None for None)."""
    if a is None:
        return None
    return a.ctypes.data_as(P(ctype))
