"""Benchmark of the explicit Euler residual-and-update path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload channel|tets|hex|batch]

Workload (default `channel`): the steady subsonic channel over a Gaussian bump, 480 x 150 x 100
boxes as 8 002 500 hybrid cells (hexahedra, triangular prisms, polyhedral bricks; wall-normal
stretching 1.1), AUSM+-up, second-order LSQ face2 gradients with the Venkatakrishnan limiter (K = 5),
total-pressure inlet at Mach 0.5, static-pressure outlet, slip walls, SSP-RK3 with local time steps
at CFL 1.5, fp32+acc64, from the freestream start. `--workload tets`: the convected isentropic
vortex on 2 073 600 jittered Kuhn tetrahedra (240 x 240 x 6 lattice, nodes moved by U(-0.2, 0.2) h,
seed 0, periodic in x and y, slip in z), HLLC, SSP-RK3 at CFL 0.8. A step is one SSP-RK3 step
(three residual evaluations and updates, the CFL time steps and the exact residual norms).
Synthetic data: the meshes and fields are generated, no dataset is read.

Metric: cell-iterations per second (cells x steps / s), whole job. `value` is device time (CUDA
events on the stepper's stream) with the state resident in HBM; `e2e` is the same metric through
the C ABI with the state in pinned host memory, copied in and out every step. With N > 1 (torchrun)
each rank steps its own copy of the case (independent replicas, weak scaling); the time is the max
over ranks.

`--impl reference` times the reference algorithm on the host cores: the CPU oracle (a C
restatement of the reference's residual and steps) on one thread per core, each thread stepping
its own copy of the workload's CPU sample (cpu_sample: a smaller mesh of the same generator and
scheme, set up by the reference's own mesh, geometry and stencil code from a committed compact
mesh, so that this arm loads nothing of this repository's native library).
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

L2_BYTES = 126 * 2**20


def measured_hbm_peak() -> tuple[float, str]:
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


# The step result a step call reads back: the head of the device's control block (dt bits, the
# invalid-cell marks, step count, dt, fault and special words, the five RMS values).
CONTROL_HEAD = 96

# ------------------------------------------------------------------ algorithmic bytes


def kernel_bytes(case, rk: int, local: bool = False, fused_norms: bool = False) -> dict[str, float]:
    """Algorithmic bytes of one step per kernel kind: every array a kernel touches, read or written
    once, at its stored size (the rule of the reference's physics/bench/euler_bench.cu:321-372,
    applied to this layout); re-reads of neighbours' values are not counted. `local`: the CFL
    steps are per cell (written by the stage-0 gradient launch)."""
    m = case.mesh
    fp32 = case.scheme.precision != "fp64"
    sS = sG = sGV = sC = 4 if fp32 else 8
    n = m.n_owned_cells
    fi = m.n_owned_interior_faces
    nb = m.n_faces - m.n_interior_faces
    nbo = m.n_owned_faces - m.n_interior_faces
    k = int(m.cell_face_offsets[n] - m.cell_face_offsets[0])
    s = int(m.stencil_offsets[n] - m.stencil_offsets[0])
    second = case.scheme.second_order
    stages = 3 if rk == 3 else 4
    inc = 4 * n + 4 * k  # lengths and codes
    boundary = nb * (4 + 5 * sS + 3 * sGV + 1 + 5 * sS + 5 * sS)
    grad = 0.0
    if second:
        grad = (5 * sS * n + 4 * n + 4 * s + 3 * sGV * s + 5 * sS * nb + inc + 6 * sC * fi
                + 3 * sC * nbo + 8 * n + 15 * sG * n + 5 * sS * n)  # fmt: skip
    spectral = (5 * sS * n + inc + 8 * fi + 4 * sGV * fi + 4 * sGV * nbo + 5 * sS * nbo + 8 * n)
    if second:
        # the stage-0 gradient launch also does the spectral radius and the CFL steps: it reads
        # the faces' normals and areas besides the gradient's arrays and, with local steps,
        # writes every cell's step; no separate spectral kernel runs
        fused = 4 * sGV * (fi + nbo) + (8 * n if local else 0)
        spectral = 0.0
    face_common = (5 * sS * n + (20 * sS * n if second else 0) + 8 * n + inc + 8 * fi
                   + 4 * sGV * fi + 6 * sC * fi + nbo * (3 * sGV + 3 * sC + 5 * sS + 1 + sGV))  # fmt: skip
    faces = 0.0
    for st in range(stages):
        b = face_common + 40 * n + 40 * n + 5 * sS * n  # u read, stage/u write, next state write
        if rk == 3 and st > 0:
            b += 40 * n  # stage read
        if rk == 4:
            b += (40 * n if st > 0 else 0) + (40 * n if st < 3 else 0)  # accumulator
        if st == 0 and not fused_norms:
            b += 40 * n  # residual for the norms (face mode 2 sums them in the gather instead)
        faces += b
    return {
        "boundary_states": boundary * stages,
        "gradients": grad * stages + (fused if second else 0.0),
        "spectral": spectral,
        "faces": faces,
        "norms": 0.0 if fused_norms else 40.0 * n,
        "control": 0.0,
    }


# ------------------------------------------------------------------ clocks


class ClockSampler:
    """nvidia-smi samples of the SM clock and throttle reasons while the timed region runs."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")  # fmt: skip

    def __init__(self, gpu_id: str):
        self.gpu_id = gpu_id
        self.proc = None
        self.file = None

    def __enter__(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", self.gpu_id, f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "20"],
                stdout=self.file, stderr=subprocess.DEVNULL,
            )  # fmt: skip
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        if self.file is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.file.flush()
        rows = [r.split(",") for r in Path(self.file.name).read_text().strip().splitlines() if r]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        sm, smax, reasons = [], [], set()
        for r in rows:
            try:
                sm.append(float(r[0]))
                smax.append(float(r[1]))
                for i, nme in enumerate(names):
                    if r[3 + i].strip().lower() == "active":
                        reasons.add(nme)
            except (ValueError, IndexError):
                continue
        os.unlink(self.file.name)
        return {
            "sm_mhz": statistics.median(sm) if sm else None,
            "sm_max_mhz": max(smax) if smax else None,
            "reasons": sorted(reasons),
            "samples": len(sm),
        }


class NvmlClockSampler:
    """The SM clock and the clock-event reasons read through NVML by a host thread about every
    millisecond while the timed region runs (nvidia-smi's sampling period can exceed a short
    region). Reading only: no setting of the GPU is changed."""

    REASONS = {"hw_slowdown": "nvmlClocksEventReasonHwSlowdown",
               "hw_thermal_slowdown": "nvmlClocksEventReasonHwThermalSlowdown",
               "sw_thermal_slowdown": "nvmlClocksEventReasonSwThermalSlowdown",
               "sw_power_cap": "nvmlClocksEventReasonSwPowerCap"}  # fmt: skip

    def __init__(self, uuid: str):
        import pynvml

        self.nvml = pynvml
        pynvml.nvmlInit()
        self.handle = pynvml.nvmlDeviceGetHandleByUUID(uuid)
        self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(self.handle, pynvml.NVML_CLOCK_SM))
        self.samples = []
        self.stop = threading.Event()
        self.thread = None

    def sample(self):
        n = self.nvml
        try:
            self.samples.append((float(n.nvmlDeviceGetClockInfo(self.handle, n.NVML_CLOCK_SM)),
                                 int(n.nvmlDeviceGetCurrentClocksEventReasons(self.handle))))  # fmt: skip
        except Exception:  # a failed read leaves the record short; the bench goes on
            pass

    def run(self):
        while not self.stop.is_set():
            self.sample()
            time.sleep(0.001)

    def __enter__(self):
        self.sample()
        self.thread = threading.Thread(target=self.run, daemon=True)
        self.thread.start()
        return self

    def __exit__(self, *exc):
        self.stop.set()
        self.thread.join()
        self.sample()
        try:
            self.nvml.nvmlShutdown()
        except Exception:
            pass

    def summary(self) -> dict:
        reasons = set()
        for _, bits in self.samples:
            for name, attr in self.REASONS.items():
                if bits & getattr(self.nvml, attr):
                    reasons.add(name)
        sm = [c for c, _ in self.samples]
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.max_mhz,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvml"}  # fmt: skip


def clock_sampler(uuid: str):
    """NVML sampling when it is available, else nvidia-smi."""
    try:
        return NvmlClockSampler(uuid)
    except Exception:
        return ClockSampler(uuid)


def gpu_uuid(device: int) -> str:
    import torch

    try:
        u = str(torch.cuda.get_device_properties(device).uuid)
        return u if u.startswith("GPU-") else "GPU-" + u
    except Exception:
        return str(device)


# ------------------------------------------------------------------ CPU (oracle) throughput


SAMPLES = {"channel": "channel", "tets": "tets", "hex": "hex", "batch": "batch"}
SAMPLE_TEXT = {
    "channel": "a 60x20x10-box hybrid bump channel (13 730 cells) of the 8.0 M-cell workload's "
               "generator and scheme",
    "tets": "a 60x24x6 periodic slab (51 840 cells) of the jittered Kuhn-tetrahedra lattice at its "
            "cell size, HLLC, SSP-RK3",
    "hex": "the 8 192-cell hexahedral vortex (fp64, first-order Roe, classical RK4)",
    "batch": "the first channel of the batch (seed 0) drawn at 20 000 cells, Roe, farfield",
}  # fmt: skip


def vortex_state(centroid, beta: float, centre, gamma: float = 1.4) -> np.ndarray:
    """Shu's isentropic vortex on the freestream rho = p = 1, u = v = 1 (conserved, 5 x cells)."""
    x, y = centroid[0] - centre[0], centroid[1] - centre[1]
    r2 = x * x + y * y
    f = beta / (2.0 * np.pi) * np.exp(0.5 * (1.0 - r2))
    u, v = 1.0 - f * y, 1.0 + f * x
    t = 1.0 - (gamma - 1.0) * beta * beta / (8.0 * gamma * np.pi * np.pi) * np.exp(1.0 - r2)
    rho = t ** (1.0 / (gamma - 1.0))
    p = rho * t
    return np.stack([rho, rho * u, rho * v, np.zeros_like(u), p / (gamma - 1.0) +
                     0.5 * rho * (u * u + v * v)])  # fmt: skip


def cpu_sample(workload: str):
    """The CPU sample of `workload` as the oracle takes it, built without this repository's
    native library: the compact mesh of tests/golden/samples/cpu_sample_<name>.npz assembled, its FP64
    geometry and face2 stencil computed by the reference's own code (oracle/_ref: core/src/mesh.cpp
    assemble, core/src/geometry.cpp compute_geometry, codegen/cpp/geometry.cpp pack_geometry and
    cell_stencil), ghost images given their owner's geometry shifted by their translation, the
    least-squares weights by the oracle (physics/src/euler.cpp:340-416). Returns (mesh dict,
    scheme dict, bc_kind, bc_data, u0, rk, cfl, local, owned cells)."""
    sys.path.insert(0, str(REPO / "tests"))
    import oracle as O
    import ref_setup as R

    z = np.load(REPO / "tests" / "golden" / "samples" / f"cpu_sample_{SAMPLES[workload]}.npz")
    nc, ng = int(z["n_cells"]), int(z["n_ghost"])
    owned = nc - ng
    r = R.reference_setup_arrays(z["points"], z["face_node_offsets"], z["face_nodes"], z["cell0"],
                                 z["cell1"], z["face_zone"], nc, ng)  # fmt: skip
    counts = [int(v) for v in r["counts"]]
    cc, vol = r["cell_centroid"].copy(), r["cell_volume"].copy()
    g = np.asarray(z["ghost_owner"], dtype=np.int64)
    if ng:
        cc[:, owned:] = cc[:, g] + z["ghost_translation"]
        vol[owned:] = vol[g]
    md = dict(zip(("n_cells", "n_owned_cells", "n_faces", "n_interior_faces",
                   "n_owned_interior_faces", "n_owned_faces"), counts))  # fmt: skip
    md.update(owner=r["owner"], neighbour=r["neighbour"], cell_face_offsets=r["cell_face_offsets"],
              cell_faces=r["cell_faces"], ghost_owner=z["ghost_owner"],
              face_normal=r["face_normal"], face_area_magnitude=r["face_area_magnitude"],
              face_centroid=r["face_centroid"],
              face_moment=r["face_moment"] if np.any(r["face_moment"]) else np.zeros(0),
              cell_centroid=cc, cell_volume=vol, stencil_offsets=r["stencil_offsets"],
              stencil=r["stencil"])  # fmt: skip
    kind, data = z["bc_kind"], z["bc_data"]
    md["stencil_lsq_weight"] = O.gradient_weights(md, kind)
    start = json.loads(str(z["start"]))
    if "uniform" in start:
        u0 = np.repeat(np.array(start["uniform"])[:, None], nc, axis=1)
    else:
        u0 = vortex_state(cc, start["vortex"]["beta"], start["vortex"]["centre"])
        if ng:
            u0[:, owned:] = u0[:, g]
    return (md, json.loads(str(z["scheme"])), kind, data, np.ascontiguousarray(u0), int(z["rk"]),
            float(z["cfl"]), bool(z["local"]), owned)  # fmt: skip


def cpu_throughput(steps: int, warmup: int, threads: int, workload: str = "channel",
                   min_seconds: float = 0.0) -> tuple[float, str, int]:  # fmt: skip
    """Cell-iterations per second of the CPU oracle on the host: one thread per core, each stepping
    its own copy of the workload's CPU sample (cpu_sample); the rate of the whole host. `steps`
    steps, then more until at least `min_seconds` have passed."""
    sys.path.insert(0, str(REPO / "tests"))
    import oracle as O

    md, sch, kind, data, u0, rk, cfl, local, cells = cpu_sample(workload)
    oracles = [O.Oracle(md, sch, kind, data) for _ in range(threads)]
    states = [u0.copy() for _ in range(threads)]

    def one_step(i):
        oracles[i].step(states[i], rk=rk, cfl=cfl, local=local)

    def all_threads():
        ts = [threading.Thread(target=one_step, args=(i,)) for i in range(threads)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()

    for _ in range(warmup):
        all_threads()
    t0 = time.perf_counter()
    done = 0
    while done < steps or time.perf_counter() - t0 < min_seconds:
        all_threads()
        done += 1
    elapsed = time.perf_counter() - t0
    rate = cells * threads * done / elapsed
    kind_of_step = "SSP-RK3" if rk == 3 else "RK4"
    sample = (f"{threads} threads x {done} {kind_of_step} steps of {SAMPLE_TEXT[workload]}, each "
              f"thread its own copy; set up by the reference's own mesh assembly, geometry and "
              f"stencil code with the oracle's weights; stepped by the CPU oracle (C, -O2); "
              f"{elapsed:.1f} s")  # fmt: skip
    return rate, sample, threads


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


# ------------------------------------------------------------------ ranks


def reduce_max(x: float, dist=None, device: str = "cpu") -> float:
    """The maximum of x over the ranks of the default process group (x itself without one)."""
    if dist is None:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(x: float, dist=None, device: str = "cpu") -> float:
    """The sum of x over the ranks of the default process group (x itself without one)."""
    if dist is None:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def whole_job_rate(world: int, cells: int, steps: int, seconds: float) -> float:
    """Cell-iterations per second of the whole job: every rank steps its own replica of `cells`
    cells `steps` times, and the job takes the slowest rank's time."""
    return world * cells * steps / seconds


def parse_triple(text: str) -> tuple[int, int, int]:
    a, b, c = (int(v) for v in text.split(","))
    return a, b, c


# ------------------------------------------------------------------ arms


def run_reference(args, rank: int, world: int) -> None:
    if rank != 0:
        return
    threads = args.cpu_threads or host_threads()
    rate, sample, cores = cpu_throughput(args.steps, max(1, min(args.warmup, 1)), threads,
                                         args.workload)  # fmt: skip
    line = {
        "impl": "reference",
        "metric": "cell-iterations/s",
        "value": rate,
        "unit": "cell-iterations/s",
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 (f64 accumulation)",
        "data": "synthetic",
        "config": workload_config(args),
        "cpu_baseline": {"value": rate, "unit": "cell-iterations/s", "cores": cores,
                         "kind": "port", "sample": sample},  # fmt: skip
        "e2e": {"value": rate, "unit": "cell-iterations/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},  # fmt: skip
    }
    print(json.dumps(line), flush=True)


def workload_config(args) -> dict:
    if args.workload == "batch":
        lo, hi = (int(v) for v in args.cells.split(","))
        return {"scaling": "strong: whole cases sharded over the ranks, greedy by cell count",
                "workload": f"{args.cases} batched steady bump channels (seed {args.seed}), cells "
                            f"log-uniform in [{lo}, {hi}], Mach U(0.3, 0.75), flow angle U(-4, 4) "
                            "deg, bump U(0.02, 0.10), farfield inflow/outflow, slip walls, Roe, LSQ "
                            "face2 + Venkatakrishnan K=5, SSP-RK3 with local steps at CFL 1.5, "
                            "fp32+acc64; every stage kernel one launch over all cases",
                "parallelism": f"replicas x{args.gpus}",
                "l2": "working set of every step larger than the 126 MB L2"}  # fmt: skip
    if args.workload == "channel":
        nx, ny, nz = (int(v) for v in args.channel.split(","))
        return {"workload": f"steady subsonic bump channel, {nx}x{ny}x{nz} boxes as hybrid "
                            "hexahedra/prisms/polyhedra (8.0 M cells at the default size), "
                            "AUSM+-up, LSQ face2 + Venkatakrishnan K=5, total-pressure inlet "
                            "M 0.5, static-pressure outlet, slip walls, SSP-RK3 with local "
                            "steps at CFL 1.5, fp32+acc64",
                "parallelism": f"replicas x{args.gpus}",
                "l2": "working set of every step larger than the 126 MB L2"}  # fmt: skip
    if args.workload == "hex":
        return {"workload": "isentropic vortex, 64x64x2 periodic hexahedra (8192 cells), "
                            "first-order Roe, classical RK4, CFL 0.5, fp64",
                "cells": 8192, "l2": "inputs smaller than L2 (launch-bound case)"}  # fmt: skip
    return {
        "workload": "isentropic vortex, 2073600 jittered Kuhn tetrahedra (240x240x6, periodic x/y, "
                    "slip z), LSQ face2 + Venkatakrishnan K=5, HLLC, SSP-RK3, CFL 0.8, fp32+acc64",
        "cells": 2073600,
        "parallelism": f"replicas x{args.gpus}",
        "l2": "working set of every step (about 2 GB) larger than the 126 MB L2",
    }


def fp64_error(case, dev, steps: int, local_rank: int) -> dict:
    """The fp32+acc64 state against the FP64 one after `steps` steps of the workload from its
    start: both run on the device (the fp64 device path equals the CPU FP64 oracle bit for bit on
    the parity meshes, and is used here because the oracle would take hours at full size). The
    largest difference of each conserved component, relative to that component's largest
    magnitude, and the largest of the five."""
    import dataclasses

    from autan_b200.euler import EulerDevice

    dev.upload(case.u0)
    dev.step(cfl=case.cfl, rk=case.rk, local=case.local, n_steps=steps, graph=True)
    u32 = dev.download()
    s64 = dataclasses.replace(case.scheme, precision="fp64")
    with EulerDevice(case.mesh, s64, case.bc_kind, case.bc_data, device=local_rank) as d64:
        d64.upload(case.u0)
        d64.step(cfl=case.cfl, rk=case.rk, local=case.local, n_steps=steps, graph=True)
        u64 = d64.download()
    n = case.mesh.n_owned_cells
    d, ref = np.abs(u32[:, :n] - u64[:, :n]), np.abs(u64[:, :n])
    mom = max(ref[1:4].max(), 1e-300)
    scale = [max(ref[0].max(), 1e-300), mom, mom, mom, max(ref[4].max(), 1e-300)]
    per = [float(d[k].max() / scale[k]) for k in range(5)]
    return {"steps": steps, "max_rel": max(per), "per_component_rel": per,
            "against": "the fp64 device path from the same start (bit-identical to the CPU FP64 "
                       "oracle at full size on the parity tests); the largest difference of "
                       "density and energy relative to their largest magnitude, of the momenta "
                       "relative to the largest momentum magnitude"}  # fmt: skip


def run_converge(args, case, dev, tuned) -> None:
    """A steady march to `--converge` decades (autan_euler_device_march), fp32+acc64 with the
    round-off plateau floors of the case's freestream (runtime/src/run.cpp:1874-1897)."""
    from autan_b200.euler import ROUND_OFF_FLOOR, residual_scales

    floors = None
    if case.scheme.precision != "fp64":
        u0 = case.u0[:, 0]
        rho = float(u0[0])
        speed = float(np.linalg.norm(u0[1:4]) / rho)
        p = float((case.scheme.gamma - 1.0) * (u0[4] - 0.5 * rho * speed * speed))
        floors = ROUND_OFF_FLOOR * residual_scales(case.mesh, rho, p, speed, case.scheme.gamma)
    res = dev.march(cfl=case.cfl, local=case.local, rk=case.rk, max_steps=args.max_steps,
                    batch=200, orders=args.converge, floors=floors)  # fmt: skip
    n = case.mesh.n_owned_cells
    print(json.dumps({
        "metric": f"GPU time to a {args.converge:g}-decade residual drop",
        "value": res["gpu_ms"] / 1e3, "unit": "s", "higher_is_better": False,
        "converged": res["converged"], "iterations": res["iterations"], "steps": res["steps"],
        "plateau_mask": res["plateau_mask"], "first_rms": list(res["first"]),
        "last_rms": list(res["last"]), "cells": n,
        "cell_iterations_per_s": n * res["steps"] / (res["gpu_ms"] / 1e3),
        "config": dict(workload_config(args), tuning=tuned, start="freestream"),
    }), flush=True)  # fmt: skip
    dev.close()


def run_warmstart(args) -> None:
    """The learned warm start end to end (autan_b200.warmstart.experiment): converged training
    cases from the batched solver, the MLP trained on the GPU, held-out cases marched from its
    prediction and from the freestream; one JSON line."""
    import torch

    torch.cuda.set_device(0)
    from autan_b200 import warmstart

    tr, te, lo, hi, ep = (int(v) for v in args.warmstart.split(","))
    res = warmstart.experiment(train_cases=tr, test_cases=te, cells=(lo, hi), epochs=ep,
                               max_steps=args.max_steps, orders=args.converge or 8.0,
                               log=lambda m: print(m, file=sys.stderr, flush=True),
                               save=args.save_network or None, load=args.load_network or None,
                               flux=args.flux, train_seed=args.train_seed)  # fmt: skip
    print(json.dumps({"metric": "GPU time to convergence, freestream start / warm start",
                      "value": res.get("gpu_time_ratio"), "unit": "x", "higher_is_better": True,
                      **res}), flush=True)  # fmt: skip


def run_warmstart_fp64(args) -> None:
    """The warm start's force check in FP64 (autan_b200.warmstart.fp64_check): the selected test
    cases marched from both starts to --converge decades (default 11) with the saved network
    --load-network; one JSON line."""
    import torch

    torch.cuda.set_device(0)
    from autan_b200 import warmstart

    tc, lo, hi = (int(v) for v in args.warmstart_fp64_set.split(","))
    res = warmstart.fp64_check(args.load_network, [int(v) for v in args.warmstart_fp64.split(",")],
                               test_cases=tc, cells=(lo, hi), orders=args.converge or 11.0,
                               max_steps=args.max_steps, flux=args.flux,
                               log=lambda m: print(m, file=sys.stderr, flush=True))  # fmt: skip
    print(json.dumps({"metric": "bump force, warm vs freestream start, FP64 march", **res}), flush=True)


def run_setup_times(args) -> None:
    """The gradient set-up of the workload's mesh (face2 stencil and LSQ weights) on the GPU
    (autan_b200.setup_device) against the host set-up: both results compared bit for bit, the
    host time and the device times; one JSON line."""
    import torch

    torch.cuda.set_device(0)
    from autan_b200 import cases
    from autan_b200.setup_device import DeviceSetup

    if args.workload == "channel":
        case = cases.bump_channel(*(int(v) for v in args.channel.split(",")))
    elif args.workload == "tets":
        case = cases.vortex_tets(*(int(v) for v in args.lattice.split(",")), precision="fp32+acc64")
    else:
        raise SystemExit("--setup-times takes --workload channel or tets")
    m = case.mesh
    kind = np.ascontiguousarray(case.bc_kind, np.uint8)
    t0 = time.perf_counter()
    wh = m.gradient_weights(kind)
    host_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    with DeviceSetup(m) as s:
        off, ent = s.stencil()
        w, retried = s.weights(kind)
        dev = s.times()
    call_s = time.perf_counter() - t0
    print(json.dumps({
        "metric": "gradient set-up (face2 stencil and LSQ weights)", "workload": args.workload,
        "cells": int(m.n_owned_cells), "entries": int(ent.size),
        "stencil_same": bool(np.array_equal(off, m.stencil_offsets) and np.array_equal(ent, m.stencil)),
        "weights_same": bool(np.array_equal(w.view(np.uint64), wh.view(np.uint64))),
        "retried_cells": retried, "host_weights_s": host_s, "device_calls_s": call_s, **dev,
    }), flush=True)  # fmt: skip


def run_mlp_step(args) -> None:
    """The warm-start MLP's training step (7 -> 4 x 128 GELU -> 5, 8192-row minibatches of 65 536
    seeded rows, Adam) and its inference (2^20 rows) per engine: 0 mma.sync a kernel per layer,
    1 tcgen05 a kernel per layer, 2 fused tcgen05. Every train and predict call ends with a stream
    synchronisation, so host time around a call is the device time of its launches plus launch
    overhead; one JSON line."""
    import torch

    torch.cuda.set_device(0)
    from autan_b200.warmstart import MLP

    r = np.random.default_rng(0)
    x = r.normal(size=(65536, 7)).astype(np.float32)
    y = r.normal(size=(65536, 5)).astype(np.float32)
    xp = r.normal(size=(1 << 20, 7)).astype(np.float32)
    flops_step = 0.0
    dims = [(7, 128)] + [(128, 128)] * 3 + [(128, 5)]
    for i, o in dims:  # forward, input gradient (not for the first layer), weight gradient
        flops_step += 2.0 * 8192 * i * o * (3 if i != 7 else 2)
    out = {}
    for engine in (0, 1, 2):
        net = MLP(seed=1)
        net.set_engine(engine)
        net.set_scaling(x.mean(0), x.std(0), y.mean(0), y.std(0))
        net.set_data(x, y)
        net.train(epochs=1, batch=8192, lr=1e-3, seed=2)  # warm-up
        t0 = time.perf_counter()
        net.train(epochs=args.steps, batch=8192, lr=1e-3, seed=3)
        step_ms = (time.perf_counter() - t0) * 1e3 / (8 * args.steps)
        net.predict(xp[:8192])
        t0 = time.perf_counter()
        net.predict(xp)
        pred_ms = (time.perf_counter() - t0) * 1e3
        out[str(engine)] = {"train_step_ms": step_ms, "train_tflops": flops_step / step_ms / 1e9,
                            "predict_1M_rows_ms": pred_ms}  # fmt: skip
        net.close()
    print(json.dumps({"metric": "warm-start MLP training step (8192 rows) and inference (2^20 rows)",
                      "unit": "ms", "engines": out,
                      "note": "host time around synchronising calls; engine 2 is the default"}),
          flush=True)  # fmt: skip


def run_converge_batch(args, batch, dev, tuned) -> None:
    """The batched march to `--converge` decades, each case with its own plateau floors."""
    from autan_b200.euler import ROUND_OFF_FLOOR

    floors = np.stack([ROUND_OFF_FLOOR * p["phi"] for p in batch.params])
    res = dev.march_cases(cfl=batch.cfl, local=True, rk=batch.rk, max_steps=args.max_steps,
                          batch=100, orders=args.converge, floors=floors)  # fmt: skip
    cells = np.array([p["cells"] for p in batch.params])
    it = res["iterations"]
    print(json.dumps({
        "metric": f"GPU time to a {args.converge:g}-decade residual drop of every case",
        "value": res["gpu_ms"] / 1e3, "unit": "s", "higher_is_better": False,
        "cases": len(cells), "cells": int(cells.sum()), "converged": int(res["converged"].sum()),
        "steps": res["steps"], "iterations_min": int(it.min()), "iterations_median": float(np.median(it)),
        "iterations_max": int(it.max()),
        "stop_s": {"min": float(res["stop_ms"].min()) / 1e3,
                   "median": float(np.median(res["stop_ms"])) / 1e3,
                   "max": float(res["stop_ms"].max()) / 1e3,
                   "per_case": [round(float(v) / 1e3, 3) for v in res["stop_ms"]]},
        "iterations_per_case": [int(v) for v in it],
        "cell_iterations": int((cells * it).sum()),
        "cell_iterations_per_s": float((cells * it).sum() / (res["gpu_ms"] / 1e3)),
        "config": dict(workload_config(args), tuning=tuned, start="freestream"),
    }), flush=True)  # fmt: skip
    dev.close()


def run_ours(args, rank: int, world: int, local_rank: int) -> None:
    import torch

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from autan_b200 import cases
    from autan_b200.euler import EulerDevice

    batch = None
    if args.workload == "batch":
        import types

        lo, hi = (int(v) for v in args.cells.split(","))
        # whole cases to ranks, greedy by cell count (no exchange between ranks)
        mine = cases.shard_cases(cases.batch_parameters(args.cases, args.seed, (lo, hi)), world)[rank]
        batch = cases.bump_batch(args.cases, seed=args.seed, cells=(lo, hi), select=mine)
        case = types.SimpleNamespace(mesh=types.SimpleNamespace(**batch.mesh), scheme=batch.scheme,
                                     bc_kind=batch.bc_kind, bc_data=batch.bc_data, u0=batch.u0,
                                     cfl=batch.cfl, rk=batch.rk, local=True)  # fmt: skip
    elif args.workload == "hex":
        case = cases.vortex_hex()
    elif args.workload == "channel":
        case = cases.bump_channel(*(int(v) for v in args.channel.split(",")))
    else:
        nx, ny, nz = (int(v) for v in args.lattice.split(","))
        case = cases.vortex_tets(nx, ny, nz, precision="fp32+acc64")
    n = case.mesh.n_owned_cells
    if batch is not None:
        dev = batch.open(local_rank)
    else:
        dev = EulerDevice(case.mesh, case.scheme, case.bc_kind, case.bc_data, device=local_rank)
    dev.upload(case.u0)
    stream = torch.cuda.ExternalStream(dev.stream)
    if args.tuning:
        dev.set_tuning(**dict(zip(dev.TUNING_KEYS, (int(v) for v in args.tuning.split(",")))))
        tuned = dev.tuning()
    else:
        # The autotuner picks the launch choices on this case (the state is restored after it).
        tuned, _ = dev.autotune(cfl=case.cfl, rk=case.rk, local=case.local, trial_steps=2)
    if args.converge > 0:
        if batch is not None:
            run_converge_batch(args, batch, dev, tuned)
        else:
            run_converge(args, case, dev, tuned)
        return
    # Warm-up (and graph capture).
    dev.step(cfl=case.cfl, rk=case.rk, local=case.local, n_steps=args.warmup, graph=True)
    if args.profile:
        # Eager launches for a profiler: the warm-up above, then `steps` steps kernel by kernel.
        t0 = time.perf_counter()
        r = dev.step(cfl=case.cfl, rk=case.rk, local=case.local, n_steps=args.steps, graph=False)
        print(json.dumps({"profile": True, "cells": n, "steps": args.steps,
                          "wall_s": time.perf_counter() - t0, "rms": list(r.residuals)}))  # fmt: skip
        dev.close()
        return

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x: float) -> float:
        return reduce_max(x, dist, "cuda")

    # -- device-timed steps, state resident in HBM
    launches0 = dev.counters()["launches"]
    barrier()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with clock_sampler(gpu_uuid(local_rank)) as clocks:
        start.record(stream)
        r = dev.step(cfl=case.cfl, rk=case.rk, local=case.local, n_steps=args.steps, graph=True)
        end.record(stream)
        end.synchronize()
    barrier()
    launches = dev.counters()["launches"] - launches0
    ms = max_over_ranks(start.elapsed_time(end))
    # replicas: every rank steps the same cells; a sharded batch: the ranks' cells add up
    sharded = batch is not None
    total = reduce_sum(float(n), dist, "cuda") if sharded else float(world * n)
    value = total * args.steps / (ms * 1e-3)
    if r.invalid_cell is not None:
        raise RuntimeError(f"invalid state at cell {r.invalid_cell}")

    # -- end to end through the C ABI: pinned host state in and out every step
    u_host = torch.empty((5, case.mesh.n_cells), dtype=torch.float64, pin_memory=True).numpy()
    dev.download(out=u_host)
    e2e_steps = max(3, min(args.steps, 10))
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        dev.upload(u_host)
        dev.step(cfl=case.cfl, rk=case.rk, local=case.local, n_steps=1, graph=True)
        dev.download(out=u_host)
    t1 = time.perf_counter()
    e2e_s = max_over_ranks(t1 - t0)
    e2e = total * e2e_steps / e2e_s
    # -- the reference's own device loop (EulerPhysics::device_step, euler_physics.cpp:1538-1570):
    # one DeviceStepper::step call per step, the state kept on the device (the host copy is
    # refreshed only by sync()), each call's result (RMS, dt, invalid cell) read back
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        dev.step(cfl=case.cfl, rk=case.rk, local=case.local, n_steps=1, graph=True)
    t1 = time.perf_counter()
    march_rate = total * e2e_steps / max_over_ranks(t1 - t0)

    # -- per-kernel times (CUDA events around every launch on the stepper's stream)
    kt = dev.kernel_times(cfl=case.cfl, rk=case.rk, local=case.local, n_steps=3)
    alg = kernel_bytes(case, case.rk, case.local, fused_norms=tuned["face_mode"] == 2 and batch is None)
    dominant = max((k for k in kt if kt[k][1] > 0), key=lambda k: kt[k][0])
    per_step_launches = kt[dominant][1] / 3
    avg_ms = kt[dominant][0] / kt[dominant][1]
    bytes_per_launch = alg[dominant] / per_step_launches
    achieved = bytes_per_launch / (avg_ms * 1e-3) / 1e9
    peak, peak_kind = measured_hbm_peak()
    step_ms = ms / args.steps
    step_bytes = sum(alg.values())
    family = {"tets": "tets", "channel": "channel", "batch": "channel"}.get(args.workload, args.workload)
    traffic = committed_traffic(dominant, n, family)
    error = None
    if world == 1 and args.error_steps > 0 and args.workload in ("tets", "channel"):
        error = fp64_error(case, dev, args.error_steps, local_rank)
    line = None
    if rank == 0:
        line = {
            "metric": "cell-iterations/s",
            "value": value,
            "unit": "cell-iterations/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": step_ms,
            "higher_is_better": True,
            "scaling": "strong" if sharded else "weak",
            "vs_baseline": None,
            "dtype": "f32 (f64 accumulation)" if case.scheme.precision != "fp64" else "f64",
            "data": "synthetic",
            "config": dict(workload_config(args), tuning=tuned),
            "e2e_device_loop": {"value": march_rate, "unit": "cell-iterations/s",
                                "h2d_bytes_per_step": 0, "d2h_bytes_per_step": CONTROL_HEAD,
                                "note": "one step call per step through the C ABI, the state on "
                                        "the device, the step result (RMS, dt, invalid cell) read "
                                        "back, as the reference's device_step loop"},
            "e2e": {"value": e2e, "unit": "cell-iterations/s",
                    "h2d_bytes_per_step": 40 * n, "d2h_bytes_per_step": 40 * n + CONTROL_HEAD},  # fmt: skip
            "gpu_launches": int(launches),
            "roofline": {
                "bound": "hbm",
                "kernel": dominant,
                "achieved": achieved,
                "peak": peak,
                "unit": "GB/s",
                "frac": achieved / peak,
                "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind,
                "traffic": traffic,
                "algorithmic_bytes_per_launch": bytes_per_launch,
                "avg_launch_ms": avg_ms,
            },
            "step_roofline": {"algorithmic_bytes": step_bytes,
                              "achieved_gbs": step_bytes / (step_ms * 1e-3) / 1e9,
                              "frac": step_bytes / (step_ms * 1e-3) / 1e9 / peak},  # fmt: skip
            "kernels_ms_per_step": {k: v[0] / 3 for k, v in kt.items()},
            "clocks": clocks.summary(),
            "residual_rms": list(map(float, r.residuals)),
        }
        if error is not None:
            line["error_vs_fp64"] = error
    dev.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        if world == 1 and not args.no_cpu:
            rate, sample, cores = cpu_throughput(2, 1, args.cpu_threads or host_threads(),
                                                 args.workload, min_seconds=10.0)  # fmt: skip
            line["cpu_baseline"] = {"value": rate, "unit": "cell-iterations/s", "cores": cores,
                                    "kind": "port", "sample": sample}  # fmt: skip
        print(json.dumps(line), flush=True)


def run_partitioned(args, rank: int, world: int, local_rank: int) -> None:
    """One mesh over the ranks (strong scaling): each rank steps its partition (consecutive runs
    of the mesh's cell order, equal face cost), the ghosts' primitive and reconstruction records
    exchanged every RK stage and the norms' exact-sum words and the CFL step's minimum reduced,
    through NCCL (TorchRanks) under torchrun; one rank steps the whole mesh through the same path
    (ThreadRanks of one, no ghosts). Device time of the timed steps, max over ranks; the value is
    the whole mesh's cells times the steps over that time."""
    import torch

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from autan_b200 import cases
    from autan_b200 import partition as PT

    if args.workload == "channel":
        case = cases.bump_channel(*(int(v) for v in args.channel.split(",")))
    elif args.workload == "tets":
        case = cases.vortex_tets(*(int(v) for v in args.lattice.split(",")), precision="fp32+acc64")
    else:
        raise SystemExit("--partitioned takes --workload channel or tets")
    weights = case.mesh.gradient_weights(case.bc_kind)
    parts = PT.partition_cells(case.mesh, world)
    part = PT.extract_partition(case.mesh, weights, parts, rank)
    if dist is not None:
        ranks = PT.TorchRanks()
        ranks.set_send_lists(part, device=torch.device("cuda", local_rank))
    else:
        ranks = PT.ThreadRanks(1)
        PT.set_send_lists(part, [np.zeros(0, dtype=np.int64)])
    mb = PT.PartitionedEuler(part, case.scheme, ranks, case.bc_kind, case.bc_data,
                             device=local_rank)  # fmt: skip
    mb.upload(case.u0)
    if args.tuning:
        mb.dev.set_tuning(**dict(zip(mb.dev.TUNING_KEYS, (int(v) for v in args.tuning.split(",")))))
        tuned = mb.dev.tuning()
    else:
        tuned, _ = mb.autotune(cfl=case.cfl, rk=case.rk, local=case.local, trial_steps=2)
        mb.upload(case.u0)
    stream = torch.cuda.ExternalStream(mb.dev.stream)
    mb.step(cfl=case.cfl, rk=case.rk, local=case.local, n_steps=args.warmup)

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    launches0 = mb.dev.counters()["launches"]
    barrier()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with clock_sampler(gpu_uuid(local_rank)) as clocks:
        start.record(stream)
        r = mb.step(cfl=case.cfl, rk=case.rk, local=case.local, n_steps=args.steps)
        end.record(stream)
        end.synchronize()
    barrier()
    launches = mb.dev.counters()["launches"] - launches0
    ms = reduce_max(start.elapsed_time(end), dist, "cuda")
    n_global = case.mesh.n_owned_cells
    value = n_global * args.steps / (ms * 1e-3)
    if r.invalid_cell is not None:
        raise RuntimeError(f"invalid state at cell {r.invalid_cell}")
    # end to end: the rank's local state in from pinned host memory and out every step
    nl = part.mesh["n_cells"]
    u_host = torch.empty((5, nl), dtype=torch.float64, pin_memory=True).numpy()
    mb.dev.download(out=u_host)
    e2e_steps = max(3, min(args.steps, 10))
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        mb.dev.upload(u_host)
        mb.step(cfl=case.cfl, rk=case.rk, local=case.local, n_steps=1)
        mb.dev.download(out=u_host)
    e2e_s = reduce_max(time.perf_counter() - t0, dist, "cuda")
    ghosts = reduce_sum(float(part.n_external), dist, "cuda")
    word = 4 if case.scheme.precision == "fp32+acc64" else 8
    stages = 3 if case.rk == 3 else 4
    line = {
        "metric": "cell-iterations/s",
        "value": value,
        "unit": "cell-iterations/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms / args.steps,
        "higher_is_better": True,
        "scaling": "strong",
        "vs_baseline": None,
        "dtype": "f32 (f64 accumulation)" if word == 4 else "f64",
        "data": "synthetic",
        "config": dict(workload_config(args), parallelism=f"partitioned x{world}",
                       partition="consecutive runs of the cell order, equal face cost",
                       external_ghosts_all_ranks=int(ghosts),
                       exchange_bytes_per_step_all_ranks=int(ghosts) * stages * 32 * word,
                       tuning_rank0=tuned),  # fmt: skip
        "e2e": {"value": n_global * e2e_steps / e2e_s, "unit": "cell-iterations/s",
                "h2d_bytes_per_step": 40 * part.n_owned, "d2h_bytes_per_step": 40 * part.n_owned,
                "note": "per rank, its local state through the C ABI every step"},  # fmt: skip
        "gpu_launches": int(launches),
        "clocks": clocks.summary(),
        "residual_rms": list(map(float, r.residuals)),
    }
    mb.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per launch of the dominant kernel
# kind, averaged over a step's launches, from one ncu capture per mesh family on a smaller case
# of that family (its summary is under profiles/): (kernel kind, mesh family) -> (bytes per
# launch, cells of the capture, the captured kernel and case). The bytes per cell do not depend
# on the lattice size (same stencil, record sizes and cell ordering), so a workload's traffic is
# the entry scaled to its cells. Where the capture holds stages 0 and 1, the step's average is
# (stage 0 + 2 x stage 1) / 3 (stages 1 and 2 do the same work).
TRAFFIC = {
    ("gradients", "tets"): (452191659, 1016064, "k_gradients_occ7, 1 016 064-cell tets lattice"),
    ("gradients", "channel"): (626937259, 994600, "k_gradients_occ7 (rows streamed), 994 600-cell bump channel"),
}


def committed_traffic(kernel: str, n_cells: int, mesh: str):
    """DRAM bytes per launch of `kernel` on `n_cells` cells of mesh family `mesh` ("tets": the
    vortex lattices; "channel": the hybrid bump channels, single or batched) from TRAFFIC, else
    None."""
    entry = TRAFFIC.get((kernel, mesh))
    if entry is None:
        return None
    return float(entry[0]) * n_cells / float(entry[1])


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["tets", "hex", "channel", "batch"], default="channel")
    ap.add_argument("--cases", type=int, default=256, help="batch: number of channel cases")
    ap.add_argument("--cells", default="20000,500000", help="batch: cell range LO,HI (log-uniform)")
    ap.add_argument("--seed", type=int, default=0, help="batch: seed of the case parameters")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--cpu-threads", type=int, default=0,
                    help="threads of the CPU baseline (0: every core this process may use)")
    ap.add_argument("--lattice", default="240,240,6", help="tetrahedral lattice NX,NY,NZ")
    ap.add_argument("--channel", default="480,150,100", help="bump channel boxes NX,NY,NZ")
    ap.add_argument("--tuning", default="", help="launch choices instead of the autotuner: "
                    "grad_chunk,grad_block,face_mode,face_block,gather_block,grad_mode[,"
                    "grad_widen,grad_narrow,grad_minb,grad_depth]")
    ap.add_argument("--converge", type=float, default=0.0,
                    help="instead of the throughput line: march the workload from its start to "
                         "this many decades of residual drop (round-off plateau rule in "
                         "fp32+acc64) and print iterations and GPU time")
    ap.add_argument("--max-steps", type=int, default=100000, help="step cap of --converge")
    ap.add_argument("--warmstart-fp64", default="",
                    help="instead of the throughput line: test cases K1,K2,... of the warm-start "
                         "test set marched in FP64 from both starts (--load-network)")
    ap.add_argument("--warmstart-fp64-set", default="32,20000,500000",
                    help="the warm-start test set the cases are drawn from: CASES,LO,HI")
    ap.add_argument("--setup-times", action="store_true",
                    help="instead of the throughput line: the workload mesh's gradient set-up on "
                         "the GPU against the host's, compared bit for bit and timed")
    ap.add_argument("--mlp-step", action="store_true",
                    help="instead of the throughput line: time the warm-start MLP's training step "
                         "and inference per engine (--steps epochs of 8 steps)")
    ap.add_argument("--warmstart", default="",
                    help="run the learned warm start instead: TRAIN,TEST,LO,HI,EPOCHS (training "
                         "cases, held-out cases, cell range, epochs), e.g. 2048,64,2000,10000,30")
    ap.add_argument("--flux", default="ausm", choices=["ausm", "roe", "hllc"],
                    help="with --warmstart: the flux of the training and held-out cases")
    ap.add_argument("--train-seed", type=int, default=1,
                    help="with --warmstart: the seed of the training cases' draws")
    ap.add_argument("--save-network", default="",
                    help="with --warmstart: write the trained network to this .npz")
    ap.add_argument("--load-network", default="",
                    help="with --warmstart: take the network from this .npz instead of training")
    ap.add_argument("--error-steps", type=int, default=100,
                    help="steps of the fp32+acc64 against fp64 comparison (0: skip)")
    ap.add_argument("--partitioned", action="store_true",
                    help="one mesh partitioned over the ranks (strong scaling; ghost exchange "
                         "through NCCL under torchrun), channel or tets")  # fmt: skip
    ap.add_argument("--profile", action="store_true",
                    help="warm-up, then --steps eager steps only (for ncu)")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("at least 3 warm-up steps")
    if args.mlp_step:
        run_mlp_step(args)
        return
    if args.setup_times:
        run_setup_times(args)
        return
    if args.warmstart_fp64:
        run_warmstart_fp64(args)
        return
    if args.warmstart:
        run_warmstart(args)
        return
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
    elif args.partitioned:
        run_partitioned(args, rank, world, local_rank)
    else:
        run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
