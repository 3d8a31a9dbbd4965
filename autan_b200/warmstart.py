"""The learned warm start of the batched steady bump channels (include/autan_mlp.h).

An MLP of 4 hidden layers of width 128 (GELU) maps a cell's features (centroid x, y, z, distance
to the bump wall, the case's Mach number, flow angle and bump height) to its conserved-variable
offsets from the case's freestream; it is trained on converged states the batched solver produces
and starts held-out cases from its prediction instead of the uniform freestream. Weights and
activations are BF16 with FP32 accumulation, in this library's own tensor-core kernels.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from autan_b200 import _native as N

FEATURES = ("x", "y", "z", "wall_distance", "mach", "angle", "bump")


def _bind():
    lib = N.lib()
    if getattr(lib, "_mlp_bound", False):
        return lib
    P, vp, sz = C.POINTER, C.c_void_p, C.c_size_t
    f32, f64, i32, i64, u64 = C.c_float, C.c_double, C.c_int32, C.c_int64, C.c_uint64

    def fn(name, res, *args):
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = list(args)

    fn("autan_mlp_create", C.c_int, i32, i32, i32, i32, u64, i32, P(vp), C.c_char_p, sz)
    fn("autan_mlp_destroy", None, vp)
    fn("autan_mlp_set_scaling", C.c_int, vp, P(f32), P(f32), P(f32), P(f32), C.c_char_p, sz)
    fn("autan_mlp_parameter_count", i64, vp)
    fn("autan_mlp_get_parameters", C.c_int, vp, P(f32), i64, C.c_char_p, sz)
    fn("autan_mlp_set_parameters", C.c_int, vp, P(f32), i64, C.c_char_p, sz)
    fn("autan_mlp_set_data", C.c_int, vp, P(f32), P(f32), i64, C.c_char_p, sz)
    fn("autan_mlp_train", C.c_int, vp, i32, i32, f32, u64, P(f32), C.c_char_p, sz)
    fn("autan_mlp_gradient", C.c_int, vp, P(f32), P(f32), i64, P(f32), P(f32), C.c_char_p, sz)
    fn("autan_mlp_predict", C.c_int, vp, P(f32), i64, P(f32), i32, C.c_char_p, sz)
    fn("autan_wall_distance", C.c_int, P(f64), P(i64), P(f64), P(i64), i32, i64, P(f64),
       C.c_char_p, sz)  # fmt: skip
    lib._mlp_bound = True
    return lib


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


class MLP:
    """autan_mlp_* on one GPU."""

    def __init__(self, inputs=7, width=128, layers=4, outputs=5, seed=0, device=0):
        self.lib = _bind()
        self.inputs, self.width, self.layers, self.outputs = inputs, width, layers, outputs
        h = C.c_void_p()
        err = N.errbuf()
        N.check(self.lib.autan_mlp_create(inputs, width, layers, outputs, seed, device,
                                          C.byref(h), err, len(err)), err)  # fmt: skip
        self.h = h.value

    def _call(self, name, *args):
        err = N.errbuf()
        N.check(getattr(self.lib, name)(self.h, *args, err, len(err)), err)

    def set_scaling(self, in_mean, in_std, out_mean, out_std):
        a = [_f32(v) for v in (in_mean, in_std, out_mean, out_std)]
        self._keep = a
        self._call("autan_mlp_set_scaling", *[N.ptr(v, C.c_float) for v in a])

    @property
    def parameter_count(self) -> int:
        return int(self.lib.autan_mlp_parameter_count(self.h))

    def parameters(self) -> np.ndarray:
        p = np.zeros(self.parameter_count, dtype=np.float32)
        self._call("autan_mlp_get_parameters", N.ptr(p, C.c_float), p.size)
        return p

    def set_parameters(self, p):
        p = _f32(p)
        self._call("autan_mlp_set_parameters", N.ptr(p, C.c_float), p.size)

    def set_data(self, x, y):
        x, y = _f32(x), _f32(y)
        self._call("autan_mlp_set_data", N.ptr(x, C.c_float), N.ptr(y, C.c_float), x.shape[0])

    def train(self, epochs, batch=8192, lr=1e-3, seed=0) -> np.ndarray:
        loss = np.zeros(epochs, dtype=np.float32)
        self._call("autan_mlp_train", int(epochs), int(batch), float(lr), int(seed),
                   N.ptr(loss, C.c_float))  # fmt: skip
        return loss

    def gradient(self, x, y) -> tuple[float, np.ndarray]:
        x, y = _f32(x), _f32(y)
        g = np.zeros(self.parameter_count, dtype=np.float32)
        loss = C.c_float()
        self._call("autan_mlp_gradient", N.ptr(x, C.c_float), N.ptr(y, C.c_float), x.shape[0],
                   C.byref(loss), N.ptr(g, C.c_float))  # fmt: skip
        return float(loss.value), g

    def predict(self, x) -> np.ndarray:
        x = _f32(x)
        y = np.zeros((x.shape[0], self.outputs), dtype=np.float32)
        self._call("autan_mlp_predict", N.ptr(x, C.c_float), x.shape[0], N.ptr(y, C.c_float), 0)
        return y

    def close(self):
        if getattr(self, "h", None):
            self.lib.autan_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def wall_triangles(mesh, zone: int) -> np.ndarray:
    """The fan triangles (apex: the node mean taken from the first node) of the boundary faces of
    `zone`, as WallSurface builds them (core/src/wall_distance.cpp:111-135): t x 9 (a, b, c)."""
    pts = mesh.points
    fno, fn = mesh.face_node_offsets, mesh.face_nodes
    out = []
    ni = mesh.n_interior_faces
    for f in np.nonzero(mesh.face_zone == zone)[0]:
        if f < ni:
            continue
        nodes = fn[fno[f] : fno[f + 1]]
        p = pts[:, nodes].T
        origin = p[0]
        s = np.zeros(3)
        for q in p:
            s = s + (q - origin)
        m = origin + (1.0 / len(nodes)) * s
        for i in range(len(nodes)):
            out.append(np.concatenate([m, p[i], p[(i + 1) % len(nodes)]]))
    return np.array(out).reshape(-1, 9)


def wall_distance(triangles: list, points: list) -> list:
    """Per case k, the exact distance of each of points[k] (3 x n_k) to triangles[k] (t_k x 9), on
    the GPU (autan_wall_distance)."""
    lib = _bind()
    tri = np.ascontiguousarray(np.concatenate([t.reshape(-1, 9) for t in triangles]), dtype=np.float64)
    toff = np.concatenate([[0], np.cumsum([t.reshape(-1, 9).shape[0] for t in triangles])]).astype(np.int64)
    pts = np.ascontiguousarray(np.concatenate(points, axis=1), dtype=np.float64)
    poff = np.concatenate([[0], np.cumsum([p.shape[1] for p in points])]).astype(np.int64)
    d = np.zeros(pts.shape[1])
    err = N.errbuf()
    N.check(lib.autan_wall_distance(N.ptr(tri, C.c_double), N.ptr(toff, C.c_int64),
                                    N.ptr(pts, C.c_double), N.ptr(poff, C.c_int64), len(points),
                                    pts.shape[1], N.ptr(d, C.c_double), err, len(err)), err)  # fmt: skip
    return [d[poff[k] : poff[k + 1]] for k in range(len(points))]
