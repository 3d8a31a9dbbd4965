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
    fn("autan_mlp_set_engine", C.c_int, vp, i32, C.c_char_p, sz)
    fn("autan_mlp_set_stall_test", C.c_int, vp, i32, C.c_char_p, sz)
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

    def set_engine(self, engine: int) -> None:
        """0: mma.sync kernels; 1: tcgen05 (tensor memory) kernels, a launch per layer; 2: the
        fused tcgen05 kernel (the default at width 128)."""
        self._call("autan_mlp_set_engine", int(engine))

    def set_stall_test(self, polls: int) -> None:
        """Test hook: the fused kernel's first wait runs out after `polls` polls (0: off)."""
        self._call("autan_mlp_set_stall_test", int(polls))

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


# ------------------------------------------------------------------ the experiment


def freestream_states(batch) -> np.ndarray:
    """Each cell's case freestream, conserved (5 x n_cells)."""
    from autan_b200.cases import GAMMA, conserved

    cols = []
    for p in batch.params:
        t = np.radians(p["angle"])
        w = [1.0, p["mach"] * np.cos(t), p["mach"] * np.sin(t), 0.0, 1.0 / GAMMA]
        free = conserved(*(np.array(v) for v in w), GAMMA)
        cols.append(np.repeat(free[:, None], p["cells"], axis=1))
    return np.concatenate(cols, axis=1)


def features(batch) -> np.ndarray:
    """The MLP inputs of every cell (n_cells x 7): centroid x, y, z, distance to the case's bump
    wall (exact, on the GPU), the case's Mach number, flow angle (degrees) and bump height."""
    off = batch.cell_offsets
    xc = batch.mesh["cell_centroid"]
    pts = [xc[:, off[k] : off[k + 1]] for k in range(len(batch.params))]
    dist = wall_distance([p["wall"] for p in batch.params], pts)
    cols = []
    for k, p in enumerate(batch.params):
        n = p["cells"]
        cols.append(np.column_stack([pts[k].T, dist[k], np.full(n, p["mach"]), np.full(n, p["angle"]),
                                     np.full(n, p["bump"])]))  # fmt: skip
    return np.concatenate(cols).astype(np.float32)


def floors(batch, unit=None) -> np.ndarray:
    """Each case's round-off floors (cases x 5): unit (default the fp32 round-off unit of the
    plateau rule, ROUND_OFF_FLOOR) times its residual scales."""
    from autan_b200.euler import ROUND_OFF_FLOOR

    u = ROUND_OFF_FLOOR if unit is None else unit
    return np.stack([u * p["phi"] for p in batch.params])


def bump_forces(batch, force) -> np.ndarray:
    """Per case, the exact sum over its bump-wall faces of the boundary pressure force (3 values),
    from autan_euler_device_boundary_pressure's per-face forces (3 x n_boundary)."""
    import math

    ni = batch.mesh["n_interior_faces"]
    zone = batch.mesh["face_zone"][ni:]
    boff = batch.mesh["boundary_offsets"]
    out = np.zeros((len(batch.params), 3))
    from autan_b200 import mesh as M

    for k in range(len(batch.params)):
        sel = np.arange(boff[k], boff[k + 1])
        sel = sel[zone[sel] == M.ZONE_BUMP]
        out[k] = [math.fsum(force[a, sel]) for a in range(3)]
    return out


def march(batch, u0, orders=8.0, max_steps=200000, batch_steps=100, device=0, reference=None,
          floor_unit=None):
    """The batched march of `batch` from u0 (5 x n_cells), drops taken from `reference` (cases x 5)
    or each case's first iteration, the plateau rule on floors(batch, floor_unit): per-case
    iterations, GPU time, the converged states and the bump forces."""
    with batch.open(device) as dev:
        dev.upload(u0)
        # launch choices from the autotuner on this batch (state restored; every choice has the
        # same bits)
        res_tuning, _ = dev.autotune(cfl=batch.cfl, rk=batch.rk, local=True, trial_steps=2)
        res = dev.march_cases(cfl=batch.cfl, local=True, rk=batch.rk, max_steps=max_steps,
                              batch=batch_steps, orders=orders,
                              floors=floors(batch, floor_unit), reference=reference)  # fmt: skip
        u = dev.download()
        _, force = dev.boundary_pressure()
    res["u"] = u
    res["force"] = bump_forces(batch, force)
    res["tuning"] = res_tuning
    return res


def _case_table(batch, cold, warm, rel) -> list[dict]:
    """Per test case: its draws, cells, both marches' iterations and convergence, force difference."""
    return [dict(case=p["case"], mach=p["mach"], angle=p["angle"], bump=p["bump"], cells=p["cells"],
                 cold_iterations=int(cold["iterations"][k]), warm_iterations=int(warm["iterations"][k]),
                 cold_converged=bool(cold["converged"][k]), warm_converged=bool(warm["converged"][k]),
                 force_rel_diff=float(rel[k]))
            for k, p in enumerate(batch.params)]  # fmt: skip


def _force_difference(cold, warm) -> np.ndarray:
    fc, fw = cold["force"], warm["force"]
    return np.abs(fw - fc).max(axis=1) / np.maximum(np.abs(fc).max(axis=1), 1e-300)


def warm_start(net, batch) -> np.ndarray:
    """The network's starting state of every cell of `batch` (5 x n_cells): freestream + prediction."""
    return freestream_states(batch) + net.predict(features(batch)).T.astype(np.float64)


def save_network(net, path, x_mean, x_std, y_mean, y_std, **extra) -> None:
    """The trained network (FP32 master parameters) and its standardisation, as a .npz."""
    np.savez(path, params=net.parameters(), x_mean=x_mean, x_std=x_std, y_mean=y_mean, y_std=y_std,
             **extra)  # fmt: skip


def load_network(path, seed=11) -> MLP:
    """A network saved by save_network."""
    z = np.load(path)
    net = MLP(seed=seed)
    net.set_scaling(z["x_mean"], z["x_std"], z["y_mean"], z["y_std"])
    net.set_parameters(z["params"])
    return net


def experiment(train_cases=2048, test_cases=64, cells=(2_000, 10_000), epochs=30, batch_rows=8192,
               lr=1e-3, orders=8.0, max_steps=200000, flux="ausm", log=print, save=None,
               load=None, train_seed=1) -> dict:  # fmt: skip
    """The learned warm start end to end: train_cases converged cases (seed train_seed) as
    training data (their batched march's per-case iterations and stop times are reported too),
    the MLP trained on them, then test_cases held-out cases (seed 2) marched from the network's
    prediction and from the freestream. The GPU-time comparison is made on the cases that converge
    from both starts, re-marched as a batch of their own from each start (a batch's GPU time
    follows its cells' iterations: converged cases' cells are skipped); cases that stall above the
    rule's plateau band run to max_steps from either start and are reported apart. save: write the
    trained network (.npz); load: take it from such a file instead of training. Returns the
    timings, iterations, force differences and a per-case table."""
    import time

    from autan_b200 import cases

    out = dict(train_cases=train_cases, test_cases=test_cases, epochs=epochs)
    if load is None:
        t0 = time.perf_counter()
        train = cases.bump_batch(train_cases, seed=train_seed, cells=cells, flux=flux, walls=True)
        log(f"training set: {train_cases} cases, {train.n_cells} cells, set-up {time.perf_counter() - t0:.0f} s")
        sol = march(train, train.u0, orders=orders, max_steps=max_steps)
        log(f"training solutions: {int(sol['converged'].sum())} converged, {sol['steps']} steps, "
            f"{sol['gpu_ms'] / 1e3:.1f} s GPU")  # fmt: skip
        # the training rows: the cells of the cases that converged (a stalled case's last state is
        # not a steady solution)
        keep = np.repeat(sol["converged"].astype(bool), [p["cells"] for p in train.params])
        if not keep.any():
            log("no training case converged: training on every case's last state")
            keep[:] = True
        x = features(train)[keep]
        y = (sol["u"] - freestream_states(train)).T.astype(np.float32)[keep]
        net = MLP(seed=11)
        scaling = (x.mean(0), np.maximum(x.std(0), 1e-6), y.mean(0), np.maximum(y.std(0), 1e-9))
        net.set_scaling(*scaling)
        net.set_data(x, y)
        t1 = time.perf_counter()
        loss = net.train(epochs=epochs, batch=batch_rows, lr=lr, seed=12)
        log(f"training: {epochs} epochs, loss {loss[0]:.3e} -> {loss[-1]:.3e}, {time.perf_counter() - t1:.0f} s")
        if save is not None:
            save_network(net, save, *scaling, loss=loss, train_iterations=sol["iterations"],
                         train_converged=sol["converged"])  # fmt: skip
        out.update(train_cells=train.n_cells, train_converged=int(sol["converged"].sum()),
                   train_rows=int(keep.sum()),
                   loss_first=float(loss[0]), loss_last=float(loss[-1]),
                   training_solution_gpu_s=sol["gpu_ms"] / 1e3, training_steps=int(sol["steps"]),
                   train_iterations_median=float(np.median(sol["iterations"])),
                   train_seed=train_seed, flux=flux, train_tuning=sol["tuning"],
                   train_cases_table=[dict(cells=int(p["cells"]), mach=float(p["mach"]),
                                           iterations=int(sol["iterations"][k]),
                                           converged=bool(sol["converged"][k]),
                                           stop_s=float(sol["stop_ms"][k]) / 1e3)
                                      for k, p in enumerate(train.params)])  # fmt: skip
    else:
        net = load_network(load)
        z = np.load(load)
        if "loss" in z:
            out.update(loss_first=float(z["loss"][0]), loss_last=float(z["loss"][-1]),
                       train_converged=int(z["train_converged"].sum()))  # fmt: skip
    test = cases.bump_batch(test_cases, seed=2, cells=cells, flux=flux, walls=True)
    cold = march(test, freestream_states(test), orders=orders, max_steps=max_steps)
    # the warm start's drops are measured from the freestream start's first residuals, as a run
    # continued from another state keeps its reference (runtime/src/run.cpp:2351-2356)
    warm = march(test, warm_start(net, test), orders=orders, max_steps=max_steps,
                 reference=cold["first"])  # fmt: skip
    rel = _force_difference(cold, warm)
    table = _case_table(test, cold, warm, rel)
    both = np.flatnonzero(cold["converged"] & warm["converged"])
    log(f"test: {len(both)} of {test_cases} cases converge from both starts")
    out.update(test_cells=test.n_cells, cold_converged=int(cold["converged"].sum()),
               warm_converged=int(warm["converged"].sum()), both_converged=int(len(both)),
               all_cold_gpu_s=cold["gpu_ms"] / 1e3, all_warm_gpu_s=warm["gpu_ms"] / 1e3)  # fmt: skip
    if len(both):
        sub = cases.bump_batch(test_cases, seed=2, cells=cells, flux=flux, walls=True,
                               select=[int(k) for k in both])  # fmt: skip
        limit = int(max(cold["iterations"][both].max(), warm["iterations"][both].max())) + 200
        cold_b = march(sub, freestream_states(sub), orders=orders, max_steps=limit)
        warm_b = march(sub, warm_start(net, sub), orders=orders, max_steps=limit,
                       reference=cold_b["first"])  # fmt: skip
        ci, wi = cold["iterations"][both], warm["iterations"][both]
        cw = np.array([p["cells"] for p in sub.params], dtype=np.float64)
        out.update(cold_gpu_s=cold_b["gpu_ms"] / 1e3, warm_gpu_s=warm_b["gpu_ms"] / 1e3,
                   gpu_time_ratio=cold_b["gpu_ms"] / warm_b["gpu_ms"],
                   cold_iterations_median=float(np.median(ci)),
                   warm_iterations_median=float(np.median(wi)),
                   iterations_ratio_median=float(np.median(ci / np.maximum(wi, 1))),
                   cell_iterations_ratio=float((cw * ci).sum() / (cw * np.maximum(wi, 1)).sum()),
                   force_rel_diff_max=float(rel[both].max()),
                   force_rel_diff_median=float(np.median(rel[both])),
                   subset_iterations_match=bool(np.array_equal(cold_b["iterations"], ci)
                                                and np.array_equal(warm_b["iterations"], wi)))  # fmt: skip
    out["cases"] = table
    return out


def fp64_check(load, select, test_cases=32, cells=(20_000, 500_000), orders=11.0,
               max_steps=400000, flux="roe", log=print) -> dict:
    """The force difference between the warm and the freestream start where no FP32 round-off
    plateau stops the march: test cases `select` (the seed-2 draws of `test_cases`, as
    experiment's test set) in FP64, both starts (the saved network `load`) marched to `orders`
    decades with FP64 round-off floors (2^-53 of the residual scales), their bump forces compared.
    Per case: iterations, convergence and the relative force difference."""
    from autan_b200 import cases

    net = load_network(load)
    sub = cases.bump_batch(test_cases, seed=2, cells=cells, flux=flux, walls=True,
                           precision="fp64", select=[int(k) for k in select])  # fmt: skip
    unit = 2.0**-53
    cold = march(sub, freestream_states(sub), orders=orders, max_steps=max_steps, floor_unit=unit)
    warm = march(sub, warm_start(net, sub), orders=orders, max_steps=max_steps,
                 reference=cold["first"], floor_unit=unit)  # fmt: skip
    rel = _force_difference(cold, warm)
    log(f"fp64: {int((cold['converged'] & warm['converged']).sum())} of {len(select)} cases "
        f"reach {orders:g} decades from both starts")  # fmt: skip
    return dict(precision="fp64", orders=orders, cells=int(sub.n_cells),
                cold_gpu_s=cold["gpu_ms"] / 1e3, warm_gpu_s=warm["gpu_ms"] / 1e3,
                cases=[dict(case=int(p["case"]), mach=float(p["mach"]), cells=int(p["cells"]),
                            cold_iterations=int(cold["iterations"][k]),
                            warm_iterations=int(warm["iterations"][k]),
                            cold_converged=bool(cold["converged"][k]),
                            warm_converged=bool(warm["converged"][k]),
                            force_rel_diff=float(rel[k]))
                       for k, p in enumerate(sub.params)])  # fmt: skip
