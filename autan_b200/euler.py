"""Python mirror of the reference's device stepper interface over the C ABI of
include/autan_euler_device.h.

    physics::Scheme, Gas           (physics/include/autan/physics/euler.hpp:40-71)  -> Scheme
    DeviceStepper<P>                (physics/include/autan/physics/euler_device.hpp:22-41)
                                                                                     -> EulerDevice
    make_device_stepper<P>(...)     (euler_device.hpp:49-54)                         -> EulerDevice(...)

Every call goes to the native library; there is no other code path. Arrays are FP64 numpy arrays
in the reference's layout: component c of cell i at [c, i] (5 x n_cells), ghost cells included.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from autan_b200 import _native as N
from autan_b200.mesh import Mesh

FLUXES = {"roe": 0, "hllc": 1, "ausm_up": 2, "ausm": 2}
PRECISIONS = {"fp64": 0, "fp32+acc64": 1}


@dataclass
class Scheme:
    """physics::Scheme and physics::Gas, with the precision policy and the planar-loop choice."""

    flux: str = "roe"
    second_order: bool = True
    limiter: bool = True
    venkat_k: float = 10.0
    length: float = 1.0
    scale: tuple = (1.0, 1.0, 1.0, 1.0, 1.0)
    mach_ref: float = 0.3
    reference: tuple = (1.0, 0.0, 0.0, 0.0, 2.5)
    gamma: float = 1.4
    gas_constant: float = 287.0
    precision: str = "fp64"
    planar: bool = True

    def native(self) -> N.Scheme:
        s = N.Scheme()
        s.flux = FLUXES[self.flux]
        s.second_order = int(self.second_order)
        s.limiter = int(self.limiter)
        s.precision = PRECISIONS[self.precision]
        s.planar = int(self.planar)
        s.gamma = self.gamma
        s.gas_constant = self.gas_constant
        s.venkat_k = self.venkat_k
        s.length = self.length
        s.mach_ref = self.mach_ref
        s.scale[:] = [float(x) for x in self.scale]
        s.reference[:] = [float(x) for x in self.reference]
        return s

    @classmethod
    def from_dict(cls, d: dict) -> "Scheme":
        """A scheme from the oracle's dictionary form (flux and precision as codes)."""
        inv_f = {0: "roe", 1: "hllc", 2: "ausm_up"}
        inv_p = {0: "fp64", 1: "fp32+acc64"}
        return cls(flux=inv_f[int(d["flux"])], second_order=bool(d["second_order"]),
                   limiter=bool(d["limiter"]), venkat_k=float(d["venkat_k"]),
                   length=float(d["length"]), scale=tuple(d["scale"]),
                   mach_ref=float(d["mach_ref"]), reference=tuple(d["reference"]),
                   gamma=float(d["gamma"]), gas_constant=float(d["gas_constant"]),
                   precision=inv_p[int(d["precision"])], planar=bool(d["planar"]))  # fmt: skip

    def as_dict(self) -> dict:
        """The scheme in the oracle's dictionary form."""
        n = self.native()
        return dict(flux=n.flux, second_order=n.second_order, limiter=n.limiter,
                    precision=n.precision, planar=n.planar, gamma=n.gamma,
                    gas_constant=n.gas_constant, venkat_k=n.venkat_k, length=n.length,
                    mach_ref=n.mach_ref, scale=list(n.scale), reference=list(n.reference))  # fmt: skip


@dataclass
class StepResult:
    """DeviceStepper<P>::Result (euler_device.hpp:25-29)."""

    residuals: np.ndarray
    time_step: float
    invalid_cell: int | None
    steps: int


def mesh_arrays(mesh: Mesh | dict, weights: np.ndarray | None) -> tuple[N.MeshArrays, list]:
    """struct autan_euler_mesh over a Mesh (or a dict of the same arrays); returns the struct and
    the arrays it points into (keep them alive while the struct is used)."""
    get = (lambda k: mesh[k]) if isinstance(mesh, dict) else (lambda k: getattr(mesh, k))
    keep = []
    m = N.MeshArrays()
    for k in ("n_cells", "n_owned_cells", "n_faces", "n_interior_faces", "n_owned_interior_faces",
              "n_owned_faces"):  # fmt: skip
        setattr(m, k, int(get(k)))
    spec = {
        "owner": C.c_int32, "neighbour": C.c_int32, "cell_face_offsets": C.c_int64,
        "cell_faces": C.c_int32, "ghost_owner": C.c_int32, "face_normal": C.c_double,
        "face_area_magnitude": C.c_double, "face_centroid": C.c_double,
        "face_moment": C.c_double, "cell_centroid": C.c_double, "cell_volume": C.c_double,
        "stencil_offsets": C.c_int64, "stencil": C.c_int32,
    }  # fmt: skip
    np_t = {C.c_int32: np.int32, C.c_int64: np.int64, C.c_double: np.float64}
    for k, t in spec.items():
        a = np.ascontiguousarray(get(k), dtype=np_t[t])
        if a.size == 0 and k == "face_moment":
            m.face_moment = None  # no moments: every face planar (the ABI's NULL)
            continue
        if a.size == 0:
            a = np.zeros(1, dtype=np_t[t])
        keep.append(a)
        setattr(m, k, N.ptr(a, t))
    if weights is not None:
        w = np.ascontiguousarray(weights, dtype=np.float64)
        keep.append(w)
        m.stencil_lsq_weight = N.ptr(w, C.c_double)
    return m, keep


class EulerDevice:
    """The explicit Euler path of one mesh on one GPU (DeviceStepper<P> + Euler<P>'s set-up calls).

    `weights`: the stencil's LSQ weights for the boundary kinds (Euler<P>::gradient_weights);
    computed from `bc_kind` by the mesh when not given.
    """

    def __init__(self, mesh: Mesh | dict, scheme: Scheme, bc_kind=None, bc_data=None,
                 weights=None, device: int = 0, stream: int | None = None):  # fmt: skip
        self.lib = N.lib()
        if not hasattr(self.lib, "autan_euler_device_create"):
            raise N.NativeError("E1104: the native library was built without its CUDA path")
        get = (lambda k: mesh[k]) if isinstance(mesh, dict) else (lambda k: getattr(mesh, k))
        self.n_cells = int(get("n_cells"))
        self.n_owned_cells = int(get("n_owned_cells"))
        self.n_faces = int(get("n_faces"))
        self.n_boundary = int(get("n_faces")) - int(get("n_interior_faces"))
        self.scheme = scheme
        if bc_kind is None:
            bc_kind = np.full(self.n_boundary, 2, dtype=np.uint8)
        bc_kind = np.ascontiguousarray(bc_kind, dtype=np.uint8)
        if weights is None and isinstance(mesh, Mesh):
            weights = mesh.gradient_weights(bc_kind)
        m, self._keep = mesh_arrays(mesh, weights)
        s = scheme.native()
        h = C.c_void_p()
        err = N.errbuf()
        N.check(self.lib.autan_euler_device_create(C.byref(m), C.byref(s), device, stream,
                                                   C.byref(h), err, len(err)), err)  # fmt: skip
        self.h = h.value
        if bc_data is None:
            bc_data = np.zeros((5, self.n_boundary))
        self.set_boundary(bc_kind, bc_data)

    # -- set-up (Euler<P>::set_boundary, set_boundary_data, set_source; set_second_order)
    def _call(self, name, *args):
        err = N.errbuf()
        N.check(getattr(self.lib, name)(self.h, *args, err, len(err)), err)

    def set_boundary(self, kind, data):
        k = np.ascontiguousarray(kind, dtype=np.uint8)
        d = np.ascontiguousarray(data, dtype=np.float64).reshape(5, -1)
        if k.size != self.n_boundary or d.shape[1] != self.n_boundary:
            raise ValueError("one code and 5 values per boundary face")
        self._call("autan_euler_device_set_boundary", N.ptr(k, C.c_uint8), N.ptr(d, C.c_double),
                   self.n_boundary)  # fmt: skip

    def set_boundary_data(self, data):
        d = np.ascontiguousarray(data, dtype=np.float64).reshape(5, -1)
        self._call("autan_euler_device_set_boundary_data", N.ptr(d, C.c_double), self.n_boundary)

    def set_source(self, source):
        s = np.ascontiguousarray(source, dtype=np.float64).reshape(5, self.n_cells)
        self._call("autan_euler_device_set_source", N.ptr(s, C.c_double))

    def set_second_order(self, on: bool):
        self._call("autan_euler_device_set_second_order", int(on))

    # -- state
    def upload(self, u):
        a = np.ascontiguousarray(u, dtype=np.float64).reshape(5, self.n_cells)
        self._call("autan_euler_device_upload", N.ptr(a, C.c_double))

    def download(self, out: np.ndarray | None = None) -> np.ndarray:
        """The FP64 state (5 x n_cells); into `out` (C-contiguous FP64, e.g. pinned) if given."""
        a = np.zeros((5, self.n_cells)) if out is None else out
        if a.dtype != np.float64 or not a.flags.c_contiguous or a.size != 5 * self.n_cells:
            raise ValueError("out must be a C-contiguous float64 array of 5 x n_cells")
        self._call("autan_euler_device_download", N.ptr(a, C.c_double))
        return a

    # -- evaluation (DeviceStepper<P>::residual, step, evaluate)
    def residual(self, u) -> np.ndarray:
        a = np.ascontiguousarray(u, dtype=np.float64).reshape(5, self.n_cells)
        r = np.zeros((5, self.n_cells))
        self._call("autan_euler_device_residual", N.ptr(a, C.c_double), N.ptr(r, C.c_double))
        return r

    def step(self, cfl: float = 0.8, dt: float = 0.0, local: bool = False, rk: int = 3,
             n_steps: int = 1, graph: bool = True) -> StepResult:  # fmt: skip
        out = N.StepResult()
        self._call("autan_euler_device_step", float(cfl), float(dt), int(local), int(rk),
                   int(n_steps), int(graph), C.byref(out))  # fmt: skip
        return _result(out)

    def evaluate(self) -> StepResult:
        out = N.StepResult()
        self._call("autan_euler_device_evaluate", C.byref(out))
        return _result(out)

    def face_parts(self, u=None) -> tuple[np.ndarray, np.ndarray]:
        """Euler<P>::face_parts of the host state u (or of the device state): the residual's face
        part (5 x n_cells) and every owned face's flux (5 x n_faces)."""
        rf = np.zeros((5, self.n_cells))
        ff = np.zeros((5, self.n_faces))
        self._call("autan_euler_device_face_parts", self._state_ptr(u), N.ptr(rf, C.c_double),
                   N.ptr(ff, C.c_double))  # fmt: skip
        return rf, ff

    def boundary_pressure(self, u=None) -> tuple[np.ndarray, np.ndarray]:
        """Euler<P>::boundary_pressure after evaluating u (or the device state): the face pressure
        of every boundary face and its force p_f S + phi_p M^T grad p (3 x n_boundary)."""
        p = np.zeros(self.n_boundary)
        force = np.zeros((3, self.n_boundary))
        self._call("autan_euler_device_boundary_pressure", self._state_ptr(u),
                   N.ptr(p, C.c_double), N.ptr(force, C.c_double))  # fmt: skip
        return p, force

    def conservation(self) -> tuple[np.ndarray, int]:
        """check_conservation's exact sums on the device state: rows E, D, boundary, faces (one
        column per equation), and the most faces of a cell."""
        sums = np.zeros((4, 5))
        d = C.c_int32()
        self._call("autan_euler_device_conservation", N.ptr(sums, C.c_double), C.byref(d))
        return sums, int(d.value)

    def _state_ptr(self, u):
        if u is None:
            return None
        self._u_keep = np.ascontiguousarray(u, dtype=np.float64).reshape(5, self.n_cells)
        return N.ptr(self._u_keep, C.c_double)

    def march(self, cfl: float = 0.8, dt: float = 0.0, local: bool = False, rk: int = 3,
              max_steps: int = 1000, batch: int = 50, orders: float = 8.0,
              floors=None) -> dict:  # fmt: skip
        """A steady march to the convergence rule (autan_euler_device_march): steps until every
        equation's RMS has dropped `orders` decades (or sits on a round-off plateau at most 10
        `floors` high), at most max_steps."""
        out = N.MarchResult()
        fl = None if floors is None else np.ascontiguousarray(floors, dtype=np.float64)
        self._call("autan_euler_device_march", float(cfl), float(dt), int(local), int(rk),
                   int(max_steps), int(batch), float(orders),
                   None if fl is None else N.ptr(fl, C.c_double), C.byref(out))  # fmt: skip
        return dict(iterations=int(out.iterations), steps=int(out.steps),
                    converged=bool(out.converged), plateau_mask=int(out.plateau_mask),
                    first=np.array(out.first[:]), last=np.array(out.last[:]),
                    time_step=float(out.time_step), gpu_ms=float(out.gpu_ms),
                    invalid_cell=None if out.invalid_cell < 0 else int(out.invalid_cell))  # fmt: skip

    # -- batched cases
    def set_cases(self, cell_offsets) -> None:
        """Case k = owned cells [cell_offsets[k], cell_offsets[k + 1]) of the union mesh."""
        off = np.ascontiguousarray(cell_offsets, dtype=np.int64)
        self.n_cases = off.size - 1
        self._call("autan_euler_device_set_cases", int(self.n_cases), N.ptr(off, C.c_int64))

    def set_case_mach_ref(self, mach_ref) -> None:
        """Per case, the AUSM+-up cut-off Mach number (n_cases values) in place of the scheme's."""
        m = np.ascontiguousarray(mach_ref, dtype=np.float64)
        if m.size != self.n_cases:
            raise ValueError("one cut-off Mach number per case")
        self._call("autan_euler_device_set_case_mach_ref", N.ptr(m, C.c_double))

    def set_active(self, active) -> None:
        a = np.ascontiguousarray(active, dtype=np.uint8)
        self._call("autan_euler_device_set_active", N.ptr(a, C.c_uint8))

    def case_history(self, count: int) -> np.ndarray:
        """Per-case RMS of the last `count` steps of the last step call: count x cases x 5."""
        out = np.zeros((count, self.n_cases, 5))
        self._call("autan_euler_device_case_history", int(count), N.ptr(out, C.c_double))
        return out

    def march_cases(self, cfl: float = 0.8, dt: float = 0.0, local: bool = True, rk: int = 3,
                    max_steps: int = 1000, batch: int = 50, orders: float = 8.0,
                    floors=None, reference=None) -> dict:  # fmt: skip
        """The batched march (autan_euler_device_march_cases): each case to the convergence rule
        (drops from `reference`, n_cases x 5, else from its first iteration), stopping at the end
        of the batch in which it converged."""
        it = np.zeros(self.n_cases, dtype=np.int64)
        conv = np.zeros(self.n_cases, dtype=np.int32)
        first = np.zeros((self.n_cases, 5))
        steps = C.c_int64()
        ms = C.c_double()
        stop = np.zeros(self.n_cases)
        fl = None if floors is None else np.ascontiguousarray(floors, dtype=np.float64)
        rf = None if reference is None else np.ascontiguousarray(reference, dtype=np.float64)
        self._call("autan_euler_device_march_cases", float(cfl), float(dt), int(local), int(rk),
                   int(max_steps), int(batch), float(orders),
                   None if fl is None else N.ptr(fl, C.c_double),
                   None if rf is None else N.ptr(rf, C.c_double), N.ptr(it, C.c_int64),
                   N.ptr(conv, C.c_int32), N.ptr(first, C.c_double), C.byref(steps),
                   C.byref(ms), N.ptr(stop, C.c_double))  # fmt: skip
        return dict(iterations=it, converged=conv.astype(bool), first=first,
                    steps=int(steps.value), gpu_ms=float(ms.value), stop_ms=stop)

    def history(self, count: int) -> tuple[np.ndarray, np.ndarray]:
        rms = np.zeros((count, 5))
        dt = np.zeros(count)
        self._call("autan_euler_device_history", int(count), N.ptr(rms, C.c_double),
                   N.ptr(dt, C.c_double))  # fmt: skip
        return rms, dt

    def gradients(self) -> tuple[np.ndarray, np.ndarray]:
        g = np.zeros((15, self.n_owned_cells))
        p = np.zeros((5, self.n_owned_cells))
        self._call("autan_euler_device_gradients", N.ptr(g, C.c_double), N.ptr(p, C.c_double))
        return g, p

    def time_steps(self, cfl: float) -> np.ndarray:
        dt = np.zeros(self.n_owned_cells)
        self._call("autan_euler_device_time_steps", float(cfl), N.ptr(dt, C.c_double))
        return dt

    KERNEL_KINDS = ("boundary_states", "gradients", "spectral", "faces", "norms", "control")

    def kernel_times(self, cfl: float = 0.8, dt: float = 0.0, local: bool = False, rk: int = 3,
                     n_steps: int = 1) -> dict:  # fmt: skip
        """Per kernel kind: (total ms, launches) over n_steps eager steps timed with CUDA events."""
        ms = np.zeros(6)
        n = np.zeros(6, dtype=np.int64)
        self._call("autan_euler_device_kernel_times", float(cfl), float(dt), int(local), int(rk),
                   int(n_steps), N.ptr(ms, C.c_double), N.ptr(n, C.c_int64))  # fmt: skip
        return {k: (float(ms[i]), int(n[i])) for i, k in enumerate(self.KERNEL_KINDS)}

    TUNING_KEYS = ("grad_chunk", "grad_block", "face_mode", "face_block", "gather_block",
                   "grad_mode", "grad_widen", "grad_narrow", "grad_minb", "grad_depth")

    def tuning(self) -> dict:
        p = np.zeros(len(self.TUNING_KEYS), dtype=np.int32)
        self._call("autan_euler_device_get_tuning", N.ptr(p, C.c_int32), len(p))
        return dict(zip(self.TUNING_KEYS, map(int, p)))

    def set_tuning(self, **kw) -> None:
        t = self.tuning()
        t.update(kw)
        p = np.array([t[k] for k in self.TUNING_KEYS], dtype=np.int32)
        self._call("autan_euler_device_set_tuning", N.ptr(p, C.c_int32), len(p))

    def autotune(self, cfl: float = 0.8, dt: float = 0.0, local: bool = False, rk: int = 3,
                 trial_steps: int = 2) -> tuple[dict, float]:  # fmt: skip
        """Picks the fastest launch choices on this case; returns them and the ms per step."""
        p = np.zeros(len(self.TUNING_KEYS), dtype=np.int32)
        ms = C.c_double()
        self._call("autan_euler_device_autotune", float(cfl), float(dt), int(local), int(rk),
                   int(trial_steps), N.ptr(p, C.c_int32), C.byref(ms))  # fmt: skip
        return dict(zip(self.TUNING_KEYS, map(int, p))), float(ms.value)

    def set_stall_test(self, polls: int) -> None:
        """Test hook of the failure detection: with polls > 0 the mode-5 gradient kernel's warps
        also wait on a barrier nothing arrives on, at most `polls` polls, so the next step call
        fails with E1201; 0 turns it off."""
        self._call("autan_euler_device_set_stall_test", int(polls))

    def sync(self):
        self._call("autan_euler_device_sync")

    @property
    def stream(self) -> int:
        return self.lib.autan_euler_device_stream(self.h)

    def counters(self) -> dict:
        c = (C.c_int64 * 4)()
        self._call("autan_euler_device_counters", c)
        return dict(launches=c[0], steps=c[1], residuals=c[2], device_bytes=c[3])

    def close(self):
        if getattr(self, "h", None):
            self.lib.autan_euler_device_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _result(out: N.StepResult) -> StepResult:
    return StepResult(
        residuals=np.array(out.residuals[:]),
        time_step=float(out.time_step),
        invalid_cell=None if out.invalid_cell < 0 else int(out.invalid_cell),
        steps=int(out.steps),
    )


# runtime/include/autan/runtime/physics.hpp: round_off_floor = 2^-24 (half an FP32 ulp at 1).
ROUND_OFF_FLOOR = 0.5 * 2.0**-23


def residual_scales(mesh: Mesh, density: float, pressure: float, speed: float,
                    gamma: float = 1.4) -> np.ndarray:  # fmt: skip
    """Phi_k, the constant flux scales of the Euler residual (EulerPhysics::residual_scales,
    physics/src/euler_physics.cpp:440-476): the RMS over owned cells of each cell's total face
    area (exact sums), times rho q, rho q^2 (three momenta) and rho q h, q = |u| + c,
    h = c^2 / (gamma - 1) + |u|^2 / 2."""
    import math

    nf, ni = mesh.n_faces, mesh.n_interior_faces
    area = mesh.face_area_magnitude
    surface = np.zeros(mesh.n_cells)
    np.add.at(surface, mesh.owner[:nf], area[:nf])
    np.add.at(surface, mesh.neighbour[:ni], area[:ni])
    own = surface[: mesh.n_owned_cells]
    rms_area = math.sqrt(math.fsum(own * own) / math.fsum(np.ones(own.size)))
    c = math.sqrt(gamma * pressure / density)
    q = speed + c
    h = c * c / (gamma - 1.0) + 0.5 * speed * speed
    mass = density * q * rms_area
    momentum = mass * q
    return np.array([mass, momentum, momentum, momentum, mass * h])


def convergence_iteration(residuals, orders: float, floors=None) -> tuple[int, int]:
    """The convergence rule on a residual history (autan_convergence_iteration): the first
    1-based iteration at which it holds (0: none) and its plateau mask."""
    r = np.ascontiguousarray(residuals, dtype=np.float64).reshape(-1, 5)
    fl = None if floors is None else np.ascontiguousarray(floors, dtype=np.float64)
    it = C.c_int64()
    mask = C.c_int32()
    err = N.errbuf()
    N.check(N.lib().autan_convergence_iteration(N.ptr(r, C.c_double), r.shape[0], float(orders),
                                                None if fl is None else N.ptr(fl, C.c_double),
                                                C.byref(it), C.byref(mask), err, len(err)), err)  # fmt: skip
    return int(it.value), int(mask.value)
