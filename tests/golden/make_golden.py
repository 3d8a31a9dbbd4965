"""Golden vectors of the explicit Euler path from the reference's own kernel source.

Run with the reference tree named by the environment (the script reads its kernels/euler.py):

    AUTAN_REFERENCE=<reference checkout> python tests/golden/make_golden.py

It imports the reference's `kernels/euler.py` (the DSL module the reference's generator turns into
the CPU and GPU loops) and calls its @pointwise bodies directly in Python, with the DSL intrinsics
(Vec3, dot, @, outer, min, max, abs, sqrt, exp, log, rel) given the semantics the generator emits
(codegen/src/autan_codegen/frontend.py: dot and @ sum left to right from the first product,
min(a, b) = a if a <= b else b, max(a, b) = a if a >= b else b, abs(x) = x if x >= 0 else -x,
constants folded only between literals; emit_cpp.py: inputs converted to the compute type on first
use, rel() subtracting in FP64 before the conversion). Python floats are IEEE doubles and
math.exp/log/sqrt call the C library, so the fp64 vectors carry the bits the reference's generated
C++ computes; fp32 vectors use numpy float32 scalars and avoid exp/log (farfield and inlet states),
whose last bits differ between libraries.

The loops around the bodies restate emit_cpu.py: cell loops over owned cells; reductions over the
face2 stencil or the cell's faces with Sum in FP64 and Min/Max in the compute type (ties keep the
first entry); interior faces scattered in face order into an FP64 residual, then boundary faces;
ghost fills after primitives, gradients and limiter (physics/src/euler.cpp:113-136).

Outputs (small .npz files beside this script) hold the inputs (mesh arrays, boundary data, state)
and the reference-evaluated outputs; tests/test_oracle_golden.py checks the C oracle against them
bit for bit, and the GPU parity tests check the CUDA path against the oracle.
"""

from __future__ import annotations

import importlib.util
import math
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
if "AUTAN_REFERENCE" not in os.environ:
    raise SystemExit("set AUTAN_REFERENCE to the reference checkout")
REFERENCE = Path(os.environ["AUTAN_REFERENCE"])
sys.path.insert(0, str(REPO))


# ---------------------------------------------------------------------------- DSL intrinsics


class Arr:
    """A DSL array value: components in row-major order and a shape."""

    __slots__ = ("v", "shape")

    def __init__(self, v, shape=None):
        self.v = list(v)
        self.shape = shape if shape is not None else (len(self.v),)

    def __add__(self, o):
        assert isinstance(o, Arr) and o.shape == self.shape
        return Arr([a + b for a, b in zip(self.v, o.v)], self.shape)

    def __sub__(self, o):
        assert isinstance(o, Arr) and o.shape == self.shape
        return Arr([a - b for a, b in zip(self.v, o.v)], self.shape)

    def __mul__(self, s):
        assert not isinstance(s, Arr)
        return Arr([x * s for x in self.v], self.shape)

    def __rmul__(self, s):
        assert not isinstance(s, Arr)
        return Arr([s * x for x in self.v], self.shape)

    def __truediv__(self, s):
        assert not isinstance(s, Arr)
        return Arr([x / s for x in self.v], self.shape)

    def __neg__(self):
        return Arr([-x for x in self.v], self.shape)

    def __matmul__(self, o):
        n, m = self.shape
        cols = o.shape[1] if len(o.shape) == 2 else 1
        out = []
        for i in range(n):
            for j in range(cols):
                acc = None
                for k in range(m):
                    p = self.v[i * m + k] * o.v[k * cols + j]
                    acc = p if acc is None else acc + p
                out.append(acc)
        return Arr(out, (n, cols) if len(o.shape) == 2 else (n,))

    def __getitem__(self, i):
        if isinstance(i, tuple):
            return self.v[i[0] * self.shape[1] + i[1]]
        if len(self.shape) == 1:
            return self.v[i]
        m = self.shape[1]
        return Arr(self.v[i * m : (i + 1) * m], (m,))


def _sel_min(a, b):
    if isinstance(a, Arr):
        return Arr([x if x <= y else y for x, y in zip(a.v, b.v)], a.shape)
    return a if a <= b else b


def _sel_max(a, b):
    if isinstance(a, Arr):
        return Arr([x if x >= y else y for x, y in zip(a.v, b.v)], a.shape)
    return a if a >= b else b


def _abs(x):
    return x if x >= 0.0 else -x


def _dot(a, b):
    acc = None
    for x, y in zip(a.v, b.v):
        p = x * y
        acc = p if acc is None else acc + p
    return acc


def _outer(a, b):
    return Arr([x * y for x in a.v for y in b.v], (len(a.v), len(b.v)))


def _transpose(a):
    n, m = a.shape
    return Arr([a.v[i * m + j] for j in range(m) for i in range(n)], (m, n))


class Reference:
    """The reference's kernels/euler.py with its bodies callable, in one precision."""

    def __init__(self, fp32: bool):
        sys.path.insert(0, str(REFERENCE / "codegen" / "src"))
        from autan_codegen.dsl import Body

        spec = importlib.util.spec_from_file_location(
            f"ref_euler_{int(fp32)}", REFERENCE / "kernels" / "euler.py"
        )
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        for name, obj in list(vars(mod).items()):
            if isinstance(obj, Body):
                setattr(mod, name, obj.fn)
        self.fp32 = fp32
        cv = np.float32 if fp32 else float
        self.cv = cv
        if fp32:
            sqrt = lambda x: np.sqrt(np.float32(x))  # noqa: E731
            exp = lambda x: np.exp(np.float32(x))  # noqa: E731
            log = lambda x: np.log(np.float32(x))  # noqa: E731
        else:
            sqrt, exp, log = math.sqrt, math.exp, math.log
        mod.Vec2 = lambda *a: Arr([cv(x) for x in a])
        mod.Vec3 = lambda *a: Arr([cv(x) for x in a])
        mod.Vec5 = lambda *a: Arr([cv(x) for x in a])
        mod.dot = _dot
        mod.outer = _outer
        mod.transpose = _transpose
        mod.sqrt, mod.exp, mod.log = sqrt, exp, log
        mod.abs, mod.min, mod.max = _abs, _sel_min, _sel_max
        mod.rel = None  # replaced by explicit FP64 differences at the loops' loads
        self.m = mod


# ---------------------------------------------------------------------------- loop driver


class Driver:
    """Euler<P>::residual over a mesh with the reference bodies (emit_cpu.py semantics)."""

    def __init__(self, ref: Reference, mesh, scheme: dict, bc_kind, bc, source=None):
        self.r = ref
        self.mesh = mesh
        self.s = scheme
        fp32 = ref.fp32
        self.S = np.float32 if fp32 else np.float64  # state, grad, geometry read as values
        cv = ref.cv
        g = scheme["gamma"]
        r = scheme["reference"]
        self.ref = np.array(r, dtype=np.float64)
        p_ref = (g - 1.0) * (r[4] - 0.5 * (r[1] * r[1] + r[2] * r[2] + r[3] * r[3]) / r[0])
        k3 = (scheme["venkat_k"] / scheme["length"]) ** 3
        self.g, self.rgas, self.minf, self.pref = cv(g), cv(scheme["gas_constant"]), cv(
            scheme["mach_ref"]
        ), cv(p_ref)
        self.ur = Arr([cv(x) for x in r])
        self.scale = Arr([cv(k3 * s * s) for s in scheme["scale"]])
        nc, nf, ni = mesh["n_cells"], mesh["n_faces"], mesh["n_interior_faces"]
        self.bc_kind = np.zeros(nf)
        self.bc_kind[ni:] = bc_kind
        self.bc = np.zeros((5, nf), dtype=self.S)
        self.bc[:, ni:] = bc
        self.source = np.zeros((5, nc), dtype=self.S) if source is None else source.astype(self.S)
        self.normal = mesh["face_normal"].astype(self.S)
        self.area = mesh["face_area_magnitude"].astype(self.S)
        self.moment = mesh["face_moment"].astype(self.S)
        self.volume = mesh["cell_volume"].astype(self.S)
        self.weight = mesh["stencil_lsq_weight"].astype(self.S)
        self.prim = np.zeros((5, nc), dtype=self.S)
        self.prim_b = np.zeros((5, nf), dtype=self.S)
        self.grad = np.zeros((15, nc), dtype=self.S)
        self.wmin = np.zeros((5, nc), dtype=self.S)
        self.wmax = np.zeros((5, nc), dtype=self.S)
        self.phi = np.full((5, nc), 1.0 if scheme["second_order"] and not scheme["limiter"] else 0.0,
                           dtype=self.S)  # fmt: skip

    def vec(self, a, i, k=5):
        cv = self.r.cv
        return Arr([cv(a[j, i]) for j in range(k)])

    def mat(self, a, i, n, m):
        cv = self.r.cv
        return Arr([cv(a[j, i]) for j in range(n * m)], (n, m))

    def rel(self, xf, f, xc, c):
        cv = self.r.cv
        return Arr([cv(float(xf[a, f]) - float(xc[a, c])) for a in range(3)])

    def fill(self, arr):
        m = self.mesh
        no = m["n_owned_cells"]
        for gi, o in enumerate(m["ghost_owner"]):
            arr[:, no + gi] = arr[:, o]

    def residual(self, u):
        mod, cv, m = self.r.m, self.r.cv, self.mesh
        nc, nf, ni = m["n_cells"], m["n_faces"], m["n_interior_faces"]
        no = m["n_owned_cells"]
        s = (u - self.ref[:, None]).astype(self.S)
        # primitives
        for c in range(no):
            w = mod.primitive(self.vec(s, c), self.ur, self.g)
            self.prim[:, c] = w.v
        self.fill(self.prim)
        # boundary states, every boundary face
        for f in range(ni, nf):
            w = mod.boundary_primitive(
                self.vec(self.prim, m["owner"][f]), cv(self.bc_kind[f]), self.vec(self.bc, f),
                self.vec(self.normal, f, 3), self.g, self.rgas, self.pref,
            )  # fmt: skip
            self.prim_b[:, f] = w.v
        if self.s["second_order"]:
            so, st = m["stencil_offsets"], m["stencil"]
            for c in range(no):
                acc = [0.0] * 15
                lo = [cv(math.inf)] * 5
                hi = [cv(-math.inf)] * 5
                wc = self.vec(self.prim, c)
                for k in range(so[c], so[c + 1]):
                    e = st[k]
                    wn = self.vec(self.prim, e) if e >= 0 else self.vec(self.prim_b, -e - 1)
                    out = mod.lsq_term(wc, wn, self.vec(self.weight, k, 3))
                    for i in range(15):
                        acc[i] += float(out[0].v[i])
                    for i in range(5):
                        if out[1].v[i] < lo[i]:
                            lo[i] = out[1].v[i]
                        if out[2].v[i] > hi[i]:
                            hi[i] = out[2].v[i]
                fin = mod.include_own_value(
                    Arr([cv(a) for a in acc], (5, 3)), Arr([cv(x) for x in lo]),
                    Arr([cv(x) for x in hi]), wc,
                )  # fmt: skip
                self.grad[:, c] = fin[0].v
                self.wmin[:, c] = fin[1].v
                self.wmax[:, c] = fin[2].v
            self.fill(self.grad)
            if self.s["limiter"]:
                cfo, cf = m["cell_face_offsets"], m["cell_faces"]
                for c in range(no):
                    accm = [cv(math.inf)] * 5
                    wc, gc = self.vec(self.prim, c), self.mat(self.grad, c, 5, 3)
                    lo, hi = self.vec(self.wmin, c), self.vec(self.wmax, c)
                    vol = cv(self.volume[c])
                    for k in range(cfo[c], cfo[c + 1]):
                        f = cf[k]
                        r = self.rel(m["face_centroid"], f, m["cell_centroid"], c)
                        # limiter_term reads rel(xf, xc) through its `@`: pass the difference.
                        out = _limiter_term(mod, wc, gc, lo, hi, vol, r, self.scale)
                        for i in range(5):
                            if out.v[i] < accm[i]:
                                accm[i] = out.v[i]
                    fin = mod.at_most_one(Arr([cv(x) for x in accm]))
                    self.phi[:, c] = fin.v
                self.fill(self.phi)
        res = np.zeros((5, nc), dtype=np.float64)
        for c in range(no):
            out = mod.volume_source(self.vec(self.source, c), cv(self.volume[c]))
            res[:, c] = [float(x) for x in out.v]
        flux = ["roe", "hllc", "ausm"][self.s["flux"]]
        planar = self.s["planar"]
        face_fn = getattr(mod, f"{flux}_face_planar" if planar else f"{flux}_face")
        bnd_fn = getattr(mod, f"{flux}_boundary_planar" if planar else f"{flux}_boundary")
        owner, neigh = m["owner"], m["neighbour"]
        for f in range(m["n_owned_interior_faces"]):
            l, r_ = owner[f], neigh[f]
            args = [
                self.vec(self.prim, l), self.mat(self.grad, l, 5, 3), self.vec(self.phi, l),
                self.rel(m["face_centroid"], f, m["cell_centroid"], l),
                self.vec(self.prim, r_), self.mat(self.grad, r_, 5, 3), self.vec(self.phi, r_),
                self.rel(m["face_centroid"], f, m["cell_centroid"], r_),
                None, self.vec(self.normal, f, 3), cv(self.area[f]),
            ]  # fmt: skip
            if not planar:
                args.append(self.mat(self.moment, f, 3, 3))
            args += [self.g, self.pref]
            if flux == "ausm":
                args.append(self.minf)
            out = _face_call(mod, face_fn, args)
            for k in range(5):
                res[k, l] += float(out.v[k])
            for k in range(5):
                res[k, r_] -= float(out.v[k])
        for f in range(ni, m["n_owned_faces"]):
            l = owner[f]
            args = [
                self.vec(self.prim, l), self.mat(self.grad, l, 5, 3), self.vec(self.phi, l),
                self.rel(m["face_centroid"], f, m["cell_centroid"], l),
                cv(self.bc_kind[f]), self.vec(self.bc, f), None, self.vec(self.normal, f, 3),
                cv(self.area[f]),
            ]  # fmt: skip
            if not planar:
                args.append(self.mat(self.moment, f, 3, 3))
            args += [self.g, self.pref, self.rgas]
            if flux == "ausm":
                args.append(self.minf)
            out = _boundary_call(mod, bnd_fn, args)
            for k in range(5):
                res[k, l] += float(out.v[k])
        return res

    def spectral_radius(self):
        mod, cv, m = self.r.m, self.r.cv, self.mesh
        lam = np.zeros(m["n_cells"])
        cfo, cf = m["cell_face_offsets"], m["cell_faces"]
        for c in range(m["n_owned_cells"]):
            acc = 0.0
            wc = self.vec(self.prim, c)
            for k in range(cfo[c], cfo[c + 1]):
                f = cf[k]
                if f < m["n_interior_faces"]:
                    nb = m["neighbour"][f] if m["owner"][f] == c else m["owner"][f]
                    wn = self.vec(self.prim, nb)
                else:
                    wn = self.vec(self.prim_b, f)
                acc += float(mod.wave_speed(wc, wn, self.vec(self.normal, f, 3), cv(self.area[f]),
                                            self.g, self.pref))  # fmt: skip
            lam[c] = float(self.S(acc))
        return lam

    def step(self, u, rk, cfl):
        """One explicit step (the oracle's oracle_step, global CFL step)."""
        m = self.mesh
        no, vol = m["n_owned_cells"], m["cell_volume"]
        res = self.residual(u)
        terms = [[float(res[k, c]) ** 2 for c in range(no)] for k in range(5)]
        norms = [math.sqrt(math.fsum(t) / float(no)) for t in terms]
        lam = self.spectral_radius()
        dt = math.inf
        for c in range(no):
            dt = min(dt, cfl * vol[c] / lam[c])
        stage = u.copy()
        if rk == 3:
            w = [(0.0, 1.0), (0.75, 0.25), (1.0 / 3.0, 2.0 / 3.0)]
            for s in range(3):
                if s > 0:
                    res = self.residual(stage)
                for k in range(5):
                    for c in range(no):
                        nxt = stage[k, c] - dt / vol[c] * res[k, c]
                        stage[k, c] = w[s][0] * u[k, c] + w[s][1] * nxt
        else:
            cs = [0.5, 0.5, 1.0]
            acc = np.zeros_like(u)
            for s in range(4):
                if s > 0:
                    res = self.residual(stage)
                for k in range(5):
                    for c in range(no):
                        if s == 0:
                            acc[k, c] = res[k, c]
                        elif s < 3:
                            acc[k, c] = acc[k, c] + 2.0 * res[k, c]
                        else:
                            acc[k, c] = acc[k, c] + res[k, c]
                        if s < 3:
                            stage[k, c] = u[k, c] - cs[s] * dt / vol[c] * res[k, c]
                        else:
                            stage[k, c] = u[k, c] - dt / 6.0 / vol[c] * acc[k, c]
        out = u.copy()
        out[:, :no] = stage[:, :no]
        return out, np.array(norms), dt


def _limiter_term(mod, wc, gc, lo, hi, vol, r, scale):
    # limiter_term(wc, gc, lo, hi, vol, xf, xc, scale) computes d = gc @ rel(xf, xc); the loads
    # give rel(xf, xc) as `r`, so the body runs with rel returning it.
    mod.rel = lambda xf, xc: r
    try:
        return mod.limiter_term(wc, gc, lo, hi, vol, None, None, scale)
    finally:
        mod.rel = None


def _face_call(mod, fn, args):
    # args: wl gl pl rl wr gr pr rr xf n area [m] g pref [minf]; the bodies call rel(xf, xl) then
    # rel(xf, xr): serve the precomputed FP64 differences in that order.
    rl, rr = args[3], args[7]
    queue = [rl, rr]
    mod.rel = lambda xf, xc: queue.pop(0)
    try:
        return fn(*args)
    finally:
        mod.rel = None


def _boundary_call(mod, fn, args):
    rl = args[3]
    mod.rel = lambda xf, xc: rl
    try:
        return fn(*args)
    finally:
        mod.rel = None


# ---------------------------------------------------------------------------- cases


def mesh_dict(mesh, bc_kind):
    d = {
        "n_cells": mesh.n_cells,
        "n_owned_cells": mesh.n_owned_cells,
        "n_faces": mesh.n_faces,
        "n_interior_faces": mesh.n_interior_faces,
        "n_owned_interior_faces": mesh.n_owned_interior_faces,
        "n_owned_faces": mesh.n_owned_faces,
    }
    for k in ["owner", "neighbour", "cell_face_offsets", "cell_faces", "ghost_owner",
              "face_normal", "face_area_magnitude", "face_centroid", "face_moment",
              "cell_centroid", "cell_volume", "stencil_offsets", "stencil"]:  # fmt: skip
        d[k] = np.array(getattr(mesh, k))
    d["stencil_lsq_weight"] = mesh.gradient_weights(bc_kind)
    return d


def smooth_state(mesh, rng, amp=0.05, rho0=1.2, vel=(0.3, -0.2, 0.1), p0=1.0e5 / 1.0e5,
                 gamma=1.4):  # fmt: skip
    """A smooth perturbed conserved state on the owned cells (ghosts copied)."""
    x = mesh.cell_centroid
    k = rng.uniform(0.5, 2.0, size=3)
    ph = rng.uniform(0, 2 * np.pi, size=5)
    s = np.sin(k[0] * x[0] + ph[0]) * np.cos(k[1] * x[1] + ph[1]) + np.sin(k[2] * x[2] + ph[2])
    rho = rho0 * (1 + amp * s)
    u = vel[0] * (1 + amp * np.cos(k[1] * x[1] + ph[3]))
    v = vel[1] * (1 + amp * np.sin(k[0] * x[0] + ph[4]))
    w = vel[2] * (1 + amp * s)
    p = p0 * (1 + 2 * amp * np.cos(k[2] * x[2] + ph[2]) * np.sin(k[0] * x[0]))
    E = p / (gamma - 1) + 0.5 * rho * (u * u + v * v + w * w)
    U = np.stack([rho, rho * u, rho * v, rho * w, E])
    U[:, mesh.n_owned_cells :] = U[:, mesh.ghost_owner]
    return U


def main():
    from autan_b200 import mesh as M

    rng = np.random.default_rng(20261203)
    gamma = 1.4
    scheme_base = dict(gamma=gamma, gas_constant=287.0, venkat_k=5.0, length=1.0, mach_ref=0.3,
                       scale=[1.2, 0.4, 0.4, 0.4, 1.0],
                       reference=[1.2, 0.36, -0.24, 0.12, 1.0 / 0.4 + 0.5 * 1.2 * 0.14])  # fmt: skip

    # -- pointwise bodies: fluxes, boundary states, primitives
    out = {}
    n = 64
    for fp32 in (False, True):
        ref = Reference(fp32)
        cv = ref.cv
        tag = "f32" if fp32 else "f64"
        wl = np.stack([rng.uniform(0.5, 2.0, n), rng.uniform(-1, 1, n), rng.uniform(-1, 1, n),
                       rng.uniform(-1, 1, n), rng.uniform(-0.3, 0.3, n)])  # fmt: skip
        wr = wl * rng.uniform(0.8, 1.25, size=wl.shape)
        # some supersonic / strongly sheared pairs
        wr[1:4, :8] *= 4.0
        nn = rng.normal(size=(3, n))
        nn /= np.linalg.norm(nn, axis=0)
        if fp32:
            wl, wr, nn = wl.astype(np.float32), wr.astype(np.float32), nn.astype(np.float32)
        # p_ref as Euler<P> derives it (physics/src/euler.cpp:238-239) from the reference state
        # (1, 0, 0, 0, 2.5): (g - 1) (E - |m|^2 / (2 rho)), in FP64.
        g, pref, minf = cv(gamma), cv((gamma - 1.0) * (2.5 - 0.5 * 0.0 / 1.0)), cv(0.4)
        res = {"roe": [], "hllc": [], "ausm": []}
        for i in range(n):
            a = Arr([cv(x) for x in wl[:, i]])
            b = Arr([cv(x) for x in wr[:, i]])
            nv = Arr([cv(x) for x in nn[:, i]])
            res["roe"].append([float(x) for x in ref.m.roe(a, b, nv, g, pref).v])
            res["hllc"].append([float(x) for x in ref.m.hllc(a, b, nv, g, pref).v])
            res["ausm"].append([float(x) for x in ref.m.ausm_up(a, b, nv, g, minf, pref).v])
        out[f"flux_{tag}_wl"] = wl.astype(np.float64)
        out[f"flux_{tag}_wr"] = wr.astype(np.float64)
        out[f"flux_{tag}_n"] = nn.astype(np.float64)
        for k, v in res.items():
            out[f"flux_{tag}_{k}"] = np.array(v).T
        # boundary states: every kind (fp32: no exp/log kinds)
        kinds = [0, 1, 2, 3, 4, 5] if not fp32 else [0, 2, 4, 5]
        bv_in, bv_kind, bv_data, bv_n, bv_out = [], [], [], [], []
        for kind in kinds:
            for i in range(12):
                wg = np.array([rng.uniform(0.8, 1.5), *rng.uniform(-0.6, 0.6, 3),
                               rng.uniform(-0.2, 0.2)])  # fmt: skip
                if kind == 3:
                    data = np.array([rng.uniform(1.1, 1.4), rng.uniform(0.0035, 0.0045), 0, 0, 0])
                elif kind == 5:
                    data = np.array([rng.choice([0.0, 0.004]), 0, 0, 0, 0])
                elif kind == 4:
                    data = np.array([0, 0, 0, 0, rng.uniform(0.9, 1.1)])
                else:
                    data = np.array([rng.uniform(0.9, 1.2), *rng.uniform(-0.5, 0.5, 3),
                                     rng.uniform(0.9, 1.1)])  # fmt: skip
                nv = rng.normal(size=3)
                nv /= np.linalg.norm(nv)
                if fp32:
                    wg, data, nv = wg.astype(np.float32), data.astype(np.float32), nv.astype(np.float32)
                w = ref.m.boundary_value(Arr([cv(x) for x in wg]), cv(kind), Arr([cv(x) for x in data]),
                                         Arr([cv(x) for x in nv]), g, cv(287.0 if kind in (3, 5) else 287.0),
                                         pref)  # fmt: skip
                bv_in.append(wg.astype(np.float64))
                bv_kind.append(kind)
                bv_data.append(data.astype(np.float64))
                bv_n.append(nv.astype(np.float64))
                bv_out.append([float(x) for x in w.v])
        out[f"bv_{tag}_w"] = np.array(bv_in).T
        out[f"bv_{tag}_kind"] = np.array(bv_kind, dtype=np.float64)
        out[f"bv_{tag}_data"] = np.array(bv_data).T
        out[f"bv_{tag}_n"] = np.array(bv_n).T
        out[f"bv_{tag}_out"] = np.array(bv_out).T
        # primitives from gauge states
        ur = Arr([cv(x) for x in scheme_base["reference"]])
        dq = rng.uniform(-0.1, 0.1, size=(5, n))
        if fp32:
            dq = dq.astype(np.float32)
        prim = [[float(x) for x in ref.m.to_primitive(Arr([cv(x) for x in dq[:, i]]), ur, g).v]
                for i in range(n)]  # fmt: skip
        out[f"prim_{tag}_dq"] = dq.astype(np.float64)
        out[f"prim_{tag}_out"] = np.array(prim).T
    np.savez_compressed(HERE / "bodies.npz", **out)
    print("bodies.npz", sum(v.nbytes for v in out.values()), "bytes")

    # -- whole residuals and steps on small meshes
    cases = []
    # 1. periodic hex box, first-order Roe, fp64 (the configuration of the 8192-cell vortex)
    hexbox = M.periodic_box_hex(5, 4, 2, extent=(1.0, 0.8, 0.4))
    kind = np.full(hexbox.n_boundary_faces, 2, dtype=np.uint8)
    cases.append(("hex_roe1_f64", hexbox, kind, dict(flux=0, second_order=0, limiter=0,
                                                     precision=0, planar=1)))  # fmt: skip
    # 2. jittered periodic tets, HLLC second order + limiter, fp64 and fp32+acc64
    tets = M.jittered_tets(3, 3, 2, extent=(0.75, 0.75, 0.5), rcm=True)
    kt = np.full(tets.n_boundary_faces, 2, dtype=np.uint8)
    cases.append(("tet_hllc2_f64", tets, kt, dict(flux=1, second_order=1, limiter=1, precision=0,
                                                  planar=1)))  # fmt: skip
    cases.append(("tet_hllc2_f32", tets, kt, dict(flux=1, second_order=1, limiter=1, precision=1,
                                                  planar=1)))  # fmt: skip
    # 3. a jittered hex channel (warped faces: full loops with moments), every boundary kind,
    #    AUSM+-up and Roe second order
    nx, ny, nz = 4, 3, 2
    disp = rng.uniform(-0.08, 0.08, size=(3, (nx + 1) * (ny + 1) * (nz + 1))) * 0.25
    chan = M.lattice("hexa", (nx, ny, nz), (0, 0, 0), (1.0, 0.75, 0.5), (False, False, False),
                     zones=(0, 1, 2, 3, 4, 5), displacement=disp)  # fmt: skip
    zone_kind = np.array([3, 4, 5, 2, 1, 0], dtype=np.uint8)  # inlet outlet wall slip far state
    kc = zone_kind[chan.boundary_zone]
    cases.append(("chan_ausm2_f64", chan, kc, dict(flux=2, second_order=1, limiter=1, precision=0,
                                                   planar=0)))  # fmt: skip
    cases.append(("chan_roe2_f64", chan, kc, dict(flux=0, second_order=1, limiter=1, precision=0,
                                                  planar=0)))  # fmt: skip
    # fp32: kinds without exp/log (state, slip, outlet, wall)
    kc32 = np.array([4, 4, 5, 2, 0, 0], dtype=np.uint8)[chan.boundary_zone]
    cases.append(("chan_roe2nolim_f32", chan, kc32, dict(flux=0, second_order=1, limiter=0,
                                                         precision=1, planar=0)))  # fmt: skip
    cases.append(("chan_ausm2_f32", chan, kc32, dict(flux=2, second_order=1, limiter=1,
                                                     precision=1, planar=0)))  # fmt: skip
    for name, mesh, bkind, sch in cases:
        scheme = dict(scheme_base, **sch)
        fp32 = bool(sch["precision"])
        ref = Reference(fp32)
        md = mesh_dict(mesh, bkind)
        nb = mesh.n_boundary_faces
        bc = np.zeros((5, nb))
        for b in range(nb):
            k = bkind[b]
            if k == 3:
                bc[:, b] = [1.3, 1.3 / (1.2 * 287.0) * 1.05, 0, 0, 0]
            elif k == 4:
                bc[:, b] = [0, 0, 0, 0, 0.98]
            elif k == 5:
                bc[:, b] = [1.0 / (1.2 * 287.0), 0, 0, 0, 0]
            elif k == 1:
                bc[:, b] = [1.2, 0.3, -0.2, 0.1, 1.0]
            elif k == 0:
                bc[:, b] = [1.21, 0.31, -0.19, 0.1, 0.01]
        u = smooth_state(mesh, rng, gamma=gamma)
        source = rng.uniform(-0.01, 0.01, size=(5, mesh.n_cells))
        drv = Driver(ref, md, scheme, bkind, bc, source)
        res = drv.residual(u)
        lam = drv.spectral_radius()
        entry = dict(md)
        entry.update({f"scheme_{k}": np.array(v) for k, v in scheme.items()})
        entry.update(bc_kind=bkind, bc=bc, u=u, source=source, res=res, lam=lam,
                     prim=drv.prim.astype(np.float64), grad=drv.grad.astype(np.float64),
                     phi=drv.phi.astype(np.float64), wmin=drv.wmin.astype(np.float64),
                     wmax=drv.wmax.astype(np.float64), prim_b=drv.prim_b.astype(np.float64))  # fmt: skip
        if name not in ("chan_ausm2_f64", "chan_roe2_f64"):  # steps where no exp/log enters
            for rk in (3, 4):
                drv2 = Driver(ref, md, scheme, bkind, bc, source)
                un, norms, dt = drv2.step(u, rk, 0.5)
                entry[f"step{rk}_u"] = un
                entry[f"step{rk}_norms"] = norms
                entry[f"step{rk}_dt"] = np.array(dt)
        np.savez_compressed(HERE / f"{name}.npz", **entry)
        print(name, mesh.n_owned_cells, "cells", (HERE / f"{name}.npz").stat().st_size, "bytes")


if __name__ == "__main__":
    main()
