"""ctypes binding of the CPU oracle (oracle/liboracle.so): the checker of the parity tests.

The oracle is test infrastructure; nothing in autan_b200/ imports it."""

from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB = Path(__file__).resolve().parent.parent / "oracle" / "liboracle.so"
i32, i64, f64, P = C.c_int32, C.c_int64, C.c_double, C.POINTER


class OracleMesh(C.Structure):
    _fields_ = [(n, i32) for n in ("n_cells", "n_owned_cells", "n_faces", "n_interior_faces",
                                   "n_owned_interior_faces", "n_owned_faces")] + [
        ("owner", P(i32)), ("neighbour", P(i32)), ("cell_face_offsets", P(i64)),
        ("cell_faces", P(i32)), ("ghost_owner", P(i32)), ("face_normal", P(f64)),
        ("face_area_magnitude", P(f64)), ("face_centroid", P(f64)), ("face_moment", P(f64)),
        ("cell_centroid", P(f64)), ("cell_volume", P(f64)), ("stencil_offsets", P(i64)),
        ("stencil", P(i32)), ("stencil_lsq_weight", P(f64)),
    ]  # fmt: skip


class OracleScheme(C.Structure):
    _fields_ = [(n, i32) for n in ("flux", "second_order", "limiter", "precision", "planar")] + [
        (n, f64) for n in ("gamma", "gas_constant", "venkat_k", "length", "mach_ref")
    ] + [("scale", f64 * 5), ("reference", f64 * 5)]  # fmt: skip


_lib = None

# Callbacks of oracle_set_ranks.
HALO_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_int32, C.c_int32, P(f64), P(f64))
MIN_FN = C.CFUNCTYPE(None, C.c_void_p, P(f64))


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(str(LIB))
        vp = C.c_void_p
        L.oracle_create.restype = vp
        L.oracle_create.argtypes = [P(OracleMesh), P(OracleScheme), P(C.c_uint8), P(f64), P(f64)]
        L.oracle_free.argtypes = [vp]
        L.oracle_set_second_order.argtypes = [vp, i32]
        L.oracle_residual.argtypes = [vp, P(f64), P(f64)]
        L.oracle_face_parts.argtypes = [vp, P(f64), P(f64), P(f64)]
        L.oracle_boundary_pressure.argtypes = [vp, P(f64), P(f64)]
        L.oracle_arrays.argtypes = [vp] + [P(f64)] * 6
        L.oracle_set_external.argtypes = [vp, P(f64), P(f64), P(f64)]
        L.oracle_set_ranks.argtypes = [vp, HALO_FN, MIN_FN, vp]
        L.oracle_spectral_radius.argtypes = [vp, P(f64)]
        L.oracle_step.restype = i64
        L.oracle_step.argtypes = [vp, P(f64), i32, f64, f64, i32, P(f64), P(f64)]
        L.oracle_norms.argtypes = [P(f64), i32, i32, P(f64)]
        L.oracle_exact_sum.restype = f64
        L.oracle_exact_sum.argtypes = [P(f64), i64]
        L.oracle_first_invalid.restype = i64
        L.oracle_first_invalid.argtypes = [vp, P(f64), P(f64)]
        L.oracle_gradient_weights.restype = None
        L.oracle_gradient_weights.argtypes = [P(OracleMesh), P(C.c_uint8), P(f64)]
        for n in ("oracle_flux",):
            getattr(L, n).argtypes = [P(OracleScheme), P(f64), P(f64), P(f64), P(f64)]
        L.oracle_boundary_value.argtypes = [P(OracleScheme), P(f64), f64, P(f64), P(f64), P(f64)]
        L.oracle_to_primitive.argtypes = [P(OracleScheme), P(f64), P(f64)]
        _lib = L
    return _lib


def _p(a, t=f64):
    return None if a is None else a.ctypes.data_as(P(t))


def scheme_struct(s: dict) -> OracleScheme:
    o = OracleScheme()
    for k in ("flux", "second_order", "limiter", "precision", "planar"):
        setattr(o, k, int(s.get(k, 0)))
    for k in ("gamma", "gas_constant", "venkat_k", "length", "mach_ref"):
        setattr(o, k, float(s[k]))
    o.scale[:] = [float(x) for x in s["scale"]]
    o.reference[:] = [float(x) for x in s["reference"]]
    return o


def mesh_struct(mesh: dict, keep: dict) -> OracleMesh:
    """struct oracle_mesh over the dict's arrays (kept alive in `keep`); a missing or empty
    stencil_lsq_weight is passed as a one-element stand-in, face_moment as NULL."""
    m = OracleMesh()
    for k in ("n_cells", "n_owned_cells", "n_faces", "n_interior_faces",
              "n_owned_interior_faces", "n_owned_faces"):  # fmt: skip
        setattr(m, k, int(mesh[k]))
    types = {"owner": i32, "neighbour": i32, "cell_faces": i32, "ghost_owner": i32,
             "stencil": i32, "cell_face_offsets": i64, "stencil_offsets": i64}  # fmt: skip
    for k in ("owner", "neighbour", "cell_face_offsets", "cell_faces", "ghost_owner",
              "face_normal", "face_area_magnitude", "face_centroid", "face_moment",
              "cell_centroid", "cell_volume", "stencil_offsets", "stencil",
              "stencil_lsq_weight"):  # fmt: skip
        t = types.get(k, f64)
        dt = {i32: np.int32, i64: np.int64, f64: np.float64}[t]
        a = np.ascontiguousarray(mesh.get(k, np.zeros(0)), dtype=dt)
        if a.size == 0 and k == "face_moment":
            setattr(m, k, None)
            continue
        if a.size == 0:
            a = np.zeros(1, dtype=dt)
        keep[k] = a
        setattr(m, k, _p(a, t))
    return m


def gradient_weights(mesh: dict, bc_kind) -> np.ndarray:
    """The oracle's least-squares weights (3 x n_stencil) of the mesh dict's stencil for the
    boundary codes (Euler::Impl::compute_gradient_weights, physics/src/euler.cpp:340-416)."""
    keep = {}
    m = mesh_struct(mesh, keep)
    kind = np.ascontiguousarray(bc_kind, dtype=np.uint8)
    w = np.zeros((3, int(np.asarray(mesh["stencil_offsets"])[int(mesh["n_cells"])])))
    lib().oracle_gradient_weights(C.byref(m), _p(kind, C.c_uint8), _p(w))
    return w


class Oracle:
    """The oracle over one mesh (a dict of arrays in the mesh contract's layout)."""

    def __init__(self, mesh: dict, scheme: dict, bc_kind, bc, source=None):
        self.keep = {}
        m = OracleMesh()
        for k in ("n_cells", "n_owned_cells", "n_faces", "n_interior_faces",
                  "n_owned_interior_faces", "n_owned_faces"):  # fmt: skip
            setattr(m, k, int(mesh[k]))
        types = {"owner": i32, "neighbour": i32, "cell_faces": i32, "ghost_owner": i32,
                 "stencil": i32, "cell_face_offsets": i64, "stencil_offsets": i64}  # fmt: skip
        for k in ("owner", "neighbour", "cell_face_offsets", "cell_faces", "ghost_owner",
                  "face_normal", "face_area_magnitude", "face_centroid", "face_moment",
                  "cell_centroid", "cell_volume", "stencil_offsets", "stencil",
                  "stencil_lsq_weight"):  # fmt: skip
            t = types.get(k, f64)
            dt = {i32: np.int32, i64: np.int64, f64: np.float64}[t]
            a = np.ascontiguousarray(mesh[k], dtype=dt)
            if a.size == 0 and k == "face_moment":
                # no moments (planar meshes): NULL, as the C side reads 9 x n_faces of them
                # whenever the pointer is set
                setattr(m, k, None)
                continue
            if a.size == 0:
                a = np.zeros(1, dtype=dt)
            self.keep[k] = a
            setattr(m, k, _p(a, t))
        self.mesh = m
        self.n_cells = int(mesh["n_cells"])
        self.n_faces = int(mesh["n_faces"])
        self.n_owned = int(mesh["n_owned_cells"])
        self.scheme = scheme_struct(scheme)
        kind = np.ascontiguousarray(bc_kind, dtype=np.uint8)
        bcd = np.ascontiguousarray(bc, dtype=np.float64)
        src = None if source is None else np.ascontiguousarray(source, dtype=np.float64)
        self.keep.update(kind=kind, bc=bcd, src=src)
        self.h = lib().oracle_create(C.byref(m), C.byref(self.scheme), _p(kind, C.c_uint8),
                                     _p(bcd), _p(src))  # fmt: skip

    def __del__(self):
        if getattr(self, "h", None):
            lib().oracle_free(self.h)
            self.h = None

    def set_second_order(self, on: bool):
        lib().oracle_set_second_order(self.h, int(on))

    def residual(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        res = np.zeros((5, self.n_cells))
        lib().oracle_residual(self.h, _p(u), _p(res))
        return res

    def face_parts(self, u):
        """Euler<P>::face_parts of state(u): (res_faces 5 x n_cells, face_flux 5 x n_faces)."""
        u = np.ascontiguousarray(u, dtype=np.float64)
        rf = np.zeros((5, self.n_cells))
        ff = np.zeros((5, self.n_faces))
        lib().oracle_face_parts(self.h, _p(u), _p(rf), _p(ff))
        return rf, ff

    def boundary_pressure(self):
        """Euler<P>::boundary_pressure of the last evaluation: (p nb, force 3 x nb)."""
        nb = self.n_faces - int(self.mesh.n_interior_faces)
        p = np.zeros(nb)
        force = np.zeros((3, nb))
        lib().oracle_boundary_pressure(self.h, _p(p), _p(force))
        return p, force

    def set_ranks(self, halo, minimum):
        """This oracle as one rank of a partitioned mesh: halo(kind, send, recv) fills recv
        (comps x ghosts) with the external ghosts' values from this rank's owned values send
        (comps x owned) at each ghost fill (kind 0 primitives, 1 gradients, 2 limiter values);
        minimum(x) returns the minimum of x over the ranks. An exception in either is re-raised
        by the next step."""
        no, ng = self.n_owned, self.n_cells - self.n_owned
        self.rank_errors = []

        def h(user, kind, comps, send, recv):
            try:
                sv = np.ctypeslib.as_array(send, shape=(comps * max(no, 1),))
                rv = np.ctypeslib.as_array(recv, shape=(comps * max(ng, 1),))
                halo(int(kind), sv[: comps * no].reshape(comps, no), rv[: comps * ng].reshape(comps, ng))
            except BaseException as e:  # noqa: BLE001 (re-raised by step)
                self.rank_errors.append(e)

        def mn(user, value):
            try:
                value[0] = float(minimum(float(value[0])))
            except BaseException as e:  # noqa: BLE001
                self.rank_errors.append(e)

        self.keep["ranks"] = (HALO_FN(h), MIN_FN(mn))
        lib().oracle_set_ranks(self.h, *self.keep["ranks"], None)

    def set_external(self, prim, grad, phi):
        """The external ghosts' values (5, 15, 5 x ghosts, ghost order) for the next residuals:
        what the halo exchange of a partitioned mesh delivers."""
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (prim, grad, phi)]
        self.keep["external"] = arrs
        lib().oracle_set_external(self.h, *[_p(a) for a in arrs])

    def arrays(self):
        nc, nf = self.n_cells, self.n_faces
        out = dict(prim=np.zeros((5, nc)), grad=np.zeros((15, nc)), phi=np.zeros((5, nc)),
                   wmin=np.zeros((5, nc)), wmax=np.zeros((5, nc)), prim_b=np.zeros((5, nf)))  # fmt: skip
        lib().oracle_arrays(self.h, *[_p(out[k]) for k in ("prim", "grad", "phi", "wmin", "wmax",
                                                            "prim_b")])  # fmt: skip
        return out

    def spectral_radius(self):
        lam = np.zeros(self.n_cells)
        lib().oracle_spectral_radius(self.h, _p(lam))
        return lam

    def step(self, u, rk=3, cfl=0.5, dt=0.0, local=False):
        """One step of u in place; returns (norms, dt, invalid cell or -1)."""
        assert u.flags.c_contiguous and u.dtype == np.float64
        norms = np.zeros(5)
        h = np.zeros(1)
        bad = lib().oracle_step(self.h, _p(u), rk, cfl, dt, int(local), _p(norms), _p(h))
        errors = getattr(self, "rank_errors", None)
        if errors:
            e = errors[0]
            errors.clear()
            raise RuntimeError("a rank callback failed") from e
        return norms, float(h[0]), int(bad)

    def first_invalid(self, u, res):
        return int(lib().oracle_first_invalid(self.h, _p(np.ascontiguousarray(u)),
                                              _p(np.ascontiguousarray(res))))  # fmt: skip


def conservation_sums(mesh: dict, res_faces, face_flux) -> np.ndarray:
    """The sums of EulerPhysics::check_conservation (physics/src/euler_physics.cpp:1747-1779) on
    one rank, each an ExactSum: rows E, D, boundary, faces; one column per equation."""
    n = int(mesh["n_owned_cells"])
    ni, nof = int(mesh["n_interior_faces"]), int(mesh["n_owned_faces"])
    noi = int(mesh["n_owned_interior_faces"])
    owner, neighbour = mesh["owner"], mesh["neighbour"]
    out = np.zeros((4, 5))
    for k in range(5):
        rf = res_faces[k, :n]
        fb = face_flux[k, ni:nof]
        fi = face_flux[k, :noi]
        mult = (owner[:noi] < n).astype(np.int64) + (neighbour[:noi] < n).astype(np.int64)
        d_terms = np.concatenate([np.abs(fb), np.repeat(np.abs(fi), mult)])
        out[0, k] = exact_sum(np.concatenate([rf, -fb]))
        out[1, k] = exact_sum(d_terms)
        out[2, k] = exact_sum(fb)
        out[3, k] = exact_sum(rf)
    return out


def exact_sum(terms) -> float:
    t = np.ascontiguousarray(terms, dtype=np.float64)
    return float(lib().oracle_exact_sum(_p(t), t.size))


def flux(scheme: dict, wl, wr, n):
    s = scheme_struct(scheme)
    out = np.zeros(5)
    lib().oracle_flux(C.byref(s), _p(np.ascontiguousarray(wl, dtype=np.float64)),
                      _p(np.ascontiguousarray(wr, dtype=np.float64)),
                      _p(np.ascontiguousarray(n, dtype=np.float64)), _p(out))  # fmt: skip
    return out


def boundary_value(scheme: dict, w, kind, data, n):
    s = scheme_struct(scheme)
    out = np.zeros(5)
    lib().oracle_boundary_value(C.byref(s), _p(np.ascontiguousarray(w, dtype=np.float64)),
                                float(kind), _p(np.ascontiguousarray(data, dtype=np.float64)),
                                _p(np.ascontiguousarray(n, dtype=np.float64)), _p(out))  # fmt: skip
    return out


def to_primitive(scheme: dict, dq):
    s = scheme_struct(scheme)
    out = np.zeros(5)
    lib().oracle_to_primitive(C.byref(s), _p(np.ascontiguousarray(dq, dtype=np.float64)), _p(out))
    return out


def load_case(path) -> tuple[dict, dict, dict]:
    """(mesh dict, scheme dict, everything else) of a golden case file."""
    z = dict(np.load(path))
    mesh_keys = ("n_cells", "n_owned_cells", "n_faces", "n_interior_faces",
                 "n_owned_interior_faces", "n_owned_faces", "owner", "neighbour",
                 "cell_face_offsets", "cell_faces", "ghost_owner", "face_normal",
                 "face_area_magnitude", "face_centroid", "face_moment", "cell_centroid",
                 "cell_volume", "stencil_offsets", "stencil", "stencil_lsq_weight")  # fmt: skip
    mesh = {k: z[k] for k in mesh_keys}
    for k in mesh_keys[:6]:
        mesh[k] = int(mesh[k])
    scheme = {k[len("scheme_"):]: (z[k].tolist()) for k in z if k.startswith("scheme_")}
    rest = {k: v for k, v in z.items() if k not in mesh_keys and not k.startswith("scheme_")}
    return mesh, scheme, rest


def convergence_iteration(residuals, orders, floors=None):
    """The steady convergence decision restated in Python (runtime/src/run.cpp:2351-2389,
    runtime/include/autan/runtime/round_off.hpp RoundOffExemption and ResidualPlateau): the first
    1-based iteration at which every equation met its drop or sits on a round-off plateau, and the
    plateau mask then; (0, 0) if never."""
    drop = 10.0 ** (-orders)
    first = None
    zero = exempt = None
    floor0 = 0.0
    plats = [dict(window=[0.0] * 100, ref=float("inf"), count=0, since=0) for _ in range(5)]

    def plateau_add(pl, v):
        pl["window"][pl["count"] % 100] = v
        pl["count"] += 1
        if pl["count"] >= 100:
            srt = sorted(pl["window"])
            level = (srt[49] + srt[50]) / 2
            if level < 0.9 * pl["ref"]:
                pl["ref"] = level
                pl["since"] = pl["count"]
        return pl["since"] > 0 and pl["count"] - pl["since"] >= 100

    def drop_ref(e):
        return max(first[1:4]) if 1 <= e <= 3 else first[e]

    def woken_ref(e):
        return drop_ref(e) if 1 <= e <= 3 else max(first)

    for it, r in enumerate(np.asarray(residuals, dtype=np.float64).reshape(-1, 5), start=1):
        if first is None:
            first = [float(x) for x in r]
            floor0 = 1e-12 * max(first)
            zero = [x < floor0 for x in first]
            exempt = list(zero)
        for e in range(5):
            if exempt[e] and r[e] > floor0:
                exempt[e] = False
        ok, mask = True, 0
        for e in range(5):
            flat = plateau_add(plats[e], float(r[e]))
            woken = zero[e] and not exempt[e]
            ref = woken_ref(e) if woken else drop_ref(e)
            met = exempt[e] or r[e] <= ref * drop
            plateau = floors is not None and flat and r[e] <= 10.0 * floors[e]
            if not met and plateau:
                mask |= 1 << e
            ok = ok and (met or plateau)
        if ok:
            return it, mask
    return 0, 0


# ------------------------------------------------------------------ MLP restatement (numpy)


def bf16(a):
    """Round FP32 values to BF16 (nearest, ties to even), returned as FP32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32)
    return np.where(np.isnan(a), a, out)


def _erf(x):
    from math import erf

    return np.vectorize(erf)(x)


def mlp_layers(inputs, width, layers, outputs):
    """(in, out, offset of W) per layer in the parameter vector of autan_mlp (W out x in, then b)."""
    out, off = [], 0
    for l in range(layers + 1):
        i = inputs if l == 0 else width
        o = outputs if l == layers else width
        out.append((i, o, off))
        off += o * i + o
    return out, off


def mlp_forward_backward(params, x, y, scaling, inputs=7, width=128, layers=4, outputs=5,
                         exact=False):  # fmt: skip
    """The loss and parameter gradient of the autan_mlp kernels, restated in numpy: BF16 rounding of
    the standardised inputs, the weights, the hidden activations and the backward dZ, FP32 math
    (FP64 and no rounding with exact=True, for finite-difference checks)."""
    dt = np.float64 if exact else np.float32
    rnd = (lambda a: np.asarray(a, dtype=dt)) if exact else bf16
    im, isd, om, osd = (np.asarray(v, dtype=dt) for v in scaling)
    spec, count = mlp_layers(inputs, width, layers, outputs)
    p = np.asarray(params, dtype=dt)
    W = [rnd(p[o : o + n_out * n_in].reshape(n_out, n_in)) for n_in, n_out, o in spec]
    b = [p[o + n_out * n_in : o + n_out * n_in + n_out] for n_in, n_out, o in spec]
    a = rnd((np.asarray(x, dtype=dt) - im) / isd)
    acts, zs = [a], []
    for l in range(layers + 1):
        z = (acts[-1].astype(dt) @ W[l].T.astype(dt)).astype(dt) + b[l]
        zs.append(z)
        if l < layers:
            g = (0.5 * z * (1.0 + _erf(z / np.sqrt(2.0)))).astype(dt)
            acts.append(rnd(g))
    t = (np.asarray(y, dtype=dt) - om) / osd
    pred = zs[-1]
    n = pred.shape[0]
    loss = float(np.sum((pred - t) ** 2) / (n * outputs))
    dz = (2.0 / (n * outputs)) * (pred - t)
    grad = np.zeros(count, dtype=dt)
    for l in range(layers, -1, -1):
        n_in, n_out, o = spec[l]
        dzb = rnd(dz)
        grad[o : o + n_out * n_in] = (dzb.T @ acts[l]).reshape(-1)
        grad[o + n_out * n_in : o + n_out * n_in + n_out] = dz.sum(axis=0)
        if l == 0:
            break
        da = dzb @ W[l]
        z = zs[l - 1]
        cdf = 0.5 * (1.0 + _erf(z / np.sqrt(2.0)))
        pdf = np.exp(-0.5 * z * z) / np.sqrt(2.0 * np.pi)
        dz = (da * (cdf + z * pdf)).astype(dt)
    return loss, grad


def point_triangle(p, a, b, c):
    """Distance from p to triangle (a, b, c) by the Voronoi regions of its features (Ericson,
    Real-Time Collision Detection, 2005, sec. 5.1.5), in the kernel's operation order."""
    def dot(u, v):  # left to right, no fused multiply-add (the kernel's order)
        return float(u[0]) * float(v[0]) + float(u[1]) * float(v[1]) + float(u[2]) * float(v[2])

    ab, ac, ap = b - a, c - a, p - a
    d1, d2 = dot(ab, ap), dot(ac, ap)
    if d1 <= 0.0 and d2 <= 0.0:
        q = a
    else:
        bp = p - b
        d3, d4 = dot(ab, bp), dot(ac, bp)
        cp = p - c
        d5, d6 = dot(ab, cp), dot(ac, cp)
        vc = d1 * d4 - d3 * d2
        vb = d5 * d2 - d1 * d6
        va = d3 * d6 - d5 * d4
        if d3 >= 0.0 and d4 <= d3:
            q = b
        elif vc <= 0.0 and d1 >= 0.0 and d3 <= 0.0:
            q = a + (d1 / (d1 - d3)) * ab
        elif d6 >= 0.0 and d5 <= d6:
            q = c
        elif vb <= 0.0 and d2 >= 0.0 and d6 <= 0.0:
            q = a + (d2 / (d2 - d6)) * ac
        elif va <= 0.0 and (d4 - d3) >= 0.0 and (d5 - d6) >= 0.0:
            q = b + ((d4 - d3) / ((d4 - d3) + (d5 - d6))) * (c - b)
        else:
            den = 1.0 / (va + vb + vc)
            q = (a + (vb * den) * ab) + (vc * den) * ac
    d = p - q
    return float(np.sqrt(dot(d, d)))
