"""The CUDA path against the CPU oracle and the reference-evaluated golden vectors, through the C
ABI (include/autan_euler_device.h). Tolerances: bit-identical wherever the arithmetic is the same
operation sequence (every body but the exp/log of farfield and inlet states); 1e-12 relative in
fp64 otherwise; fp32+acc64 against the fp64 oracle within the bound stated per test."""

from pathlib import Path

import numpy as np
import pytest

import oracle as O
from autan_b200 import cases
from autan_b200.euler import EulerDevice, Scheme

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = sorted(p.stem for p in GOLDEN.glob("*.npz") if p.stem != "bodies")
EXP_LOG = {"chan_ausm2_f64", "chan_roe2_f64"}  # farfield and inlet faces: CUDA exp/log


def bits_equal(a, b):
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    return np.array_equal(a, b) and np.array_equal(np.signbit(a), np.signbit(b))


def rel_err(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def device_of(mesh, scheme, bc_kind, bc, source=None):
    dev = EulerDevice(mesh, Scheme.from_dict(scheme) if isinstance(scheme, dict) else scheme,
                      bc_kind=bc_kind, bc_data=bc, weights=mesh["stencil_lsq_weight"])
    if source is not None:
        dev.set_source(source)
    return dev


@pytest.mark.parametrize("case", CASES)
def test_golden_residual(case):
    mesh, scheme, z = O.load_case(GOLDEN / f"{case}.npz")
    no = mesh["n_owned_cells"]
    with device_of(mesh, scheme, z["bc_kind"], z["bc"], z["source"]) as dev:
        res = dev.residual(z["u"])
        grad, phi = dev.gradients()
    if scheme["second_order"]:
        if case in EXP_LOG:
            # farfield/inlet boundary states enter the limiter's bounds (and kept-face fits)
            assert rel_err(grad, z["grad"][:, :no]) <= 1e-12
            assert rel_err(phi, z["phi"][:, :no]) <= 1e-12
        else:
            assert bits_equal(grad, z["grad"][:, :no])
            assert bits_equal(phi, z["phi"][:, :no])
    if case in EXP_LOG:
        assert rel_err(res[:, :no], z["res"][:, :no]) <= 1e-12
    else:
        assert bits_equal(res[:, :no], z["res"][:, :no]), rel_err(res[:, :no], z["res"][:, :no])


STEP_CASES = [c for c in CASES if "step3_u" in np.load(GOLDEN / f"{c}.npz").files]


@pytest.mark.parametrize("case", STEP_CASES)
def test_golden_steps(case):
    """One SSP-RK3 and one classical RK4 step of every golden case whose boundary states need no
    exp/log (the fp32+acc64 channels with warped faces included), bit for bit."""
    mesh, scheme, z = O.load_case(GOLDEN / f"{case}.npz")
    no = mesh["n_owned_cells"]
    for rk in (3, 4):
        with device_of(mesh, scheme, z["bc_kind"], z["bc"], z["source"]) as dev:
            dev.upload(z["u"])
            r = dev.step(cfl=0.5, rk=rk, n_steps=1)
            u = dev.download()
        assert r.invalid_cell is None
        assert r.time_step == float(z[f"step{rk}_dt"])
        assert bits_equal(r.residuals, z[f"step{rk}_norms"])
        assert bits_equal(u[:, :no], z[f"step{rk}_u"][:, :no])


def run_device(case, steps, graph=True, local=False):
    with EulerDevice(case.mesh, case.scheme, case.bc_kind, case.bc_data) as dev:
        dev.upload(case.u0)
        r = dev.step(cfl=case.cfl, rk=case.rk, n_steps=steps, graph=graph, local=local)
        rms, dts = dev.history(steps)
        return dev.download(), r, rms, dts


def run_oracle(case, steps, local=False, precision=None):
    scheme = case.scheme.as_dict()
    if precision is not None:
        scheme["precision"] = precision
    o = O.Oracle(cases.oracle_mesh_dict(case), scheme, case.bc_kind, case.bc_data)
    u = case.u0.copy()
    norms, dts = [], []
    bad = -1
    for _ in range(steps):
        n, dt, bad = o.step(u, rk=case.rk, cfl=case.cfl, local=local)
        norms.append(n)
        dts.append(dt)
    return u, np.array(norms), np.array(dts), bad


def test_vortex_hex_rk4_200_steps():
    """The 8192-cell periodic vortex, first-order Roe, RK4, CFL 0.5, 200 steps, FP64: the final
    state within 1e-12 relative of the oracle (and, by construction, bit for bit)."""
    case = cases.vortex_hex()
    u_d, r, rms_d, dt_d = run_device(case, case.steps)
    u_o, rms_o, dt_o, bad = run_oracle(case, case.steps)
    no = case.mesh.n_owned_cells
    assert r.invalid_cell is None and bad == -1
    assert rel_err(u_d[:, :no], u_o[:, :no]) <= 1e-12
    assert bits_equal(u_d[:, :no], u_o[:, :no])
    assert bits_equal(rms_d, rms_o)
    assert bits_equal(dt_d, dt_o)


@pytest.mark.parametrize("precision", ["fp64", "fp32+acc64"])
def test_vortex_tets_same_precision(precision):
    """The jittered-tetrahedra vortex (HLLC, LSQ face2 + Venkatakrishnan, SSP-RK3, CFL 0.8) on a
    24 x 24 x 6 lattice (20 736 cells), 10 steps: the device equals the oracle of the same precision
    bit for bit (fp64 bound 1e-12 relative)."""
    case = cases.vortex_tets(24, 24, 6, steps=10, precision=precision)
    u_d, r, rms_d, dt_d = run_device(case, case.steps)
    u_o, rms_o, dt_o, bad = run_oracle(case, case.steps)
    no = case.mesh.n_owned_cells
    assert rel_err(u_d[:, :no], u_o[:, :no]) <= 1e-12
    assert bits_equal(u_d[:, :no], u_o[:, :no])
    assert bits_equal(rms_d, rms_o)
    assert bits_equal(dt_d, dt_o)


def test_vortex_tets_fp32_against_fp64_oracle():
    """fp32+acc64 against the FP64 oracle: after 10 steps the conserved state differs by at most
    2e-6 of its largest magnitude (FP32 resolution of the gauge state, 6e-8, times the growth over
    the steps)."""
    case = cases.vortex_tets(24, 24, 6, steps=10, precision="fp32+acc64")
    u_d, *_ = run_device(case, case.steps)
    u_o, *_ = run_oracle(case, case.steps, precision=0)
    no = case.mesh.n_owned_cells
    err = rel_err(u_d[:, :no], u_o[:, :no])
    print(f"fp32+acc64 vs fp64 oracle: {err:.3e}")
    assert err <= 2e-6


def test_graph_equals_eager_and_repeats():
    """A captured step replays the eager launches bit for bit; two runs give the same bits."""
    case = cases.vortex_tets(16, 16, 6, steps=4, precision="fp32+acc64")
    a, *_ = run_device(case, case.steps, graph=True)
    b, *_ = run_device(case, case.steps, graph=False)
    c, *_ = run_device(case, case.steps, graph=True)
    assert bits_equal(a, b)
    assert bits_equal(a, c)


def test_local_time_steps():
    case = cases.vortex_tets(16, 16, 6, steps=3, precision="fp64")
    u_d, *_ = run_device(case, case.steps, local=True)
    u_o, *_ = run_oracle(case, case.steps, local=True)
    no = case.mesh.n_owned_cells
    assert bits_equal(u_d[:, :no], u_o[:, :no])


def test_freestream_preserved_full_size():
    """Size-independent property at the benchmark's full size (2 073 600 tetrahedra): a uniform
    freestream is a steady state of the residual to round-off (acceptance gate freestream
    preservation, docs/validation/acceptance.md:27): every |R| <= 64 eps (|F| A) per cell."""
    case = cases.vortex_tets(precision="fp64")
    u = np.repeat(np.array(cases.freestream_reference())[:, None], case.mesh.n_cells, axis=1)
    with EulerDevice(case.mesh, case.scheme, case.bc_kind, case.bc_data) as dev:
        res = dev.residual(u)
    no = case.mesh.n_owned_cells
    area = case.mesh.face_area_magnitude
    scale = 3.5 * 2.0 * area.max() * 6
    assert np.abs(res[:, :no]).max() <= 64 * np.finfo(np.float64).eps * scale


def test_conservation_full_size():
    """Size-independent property at full size: over 3 SSP-RK3 steps of the fp32+acc64 benchmark
    case, total mass, x/y momentum and energy (sum of V u over the periodic box with slip walls)
    change by at most 1e-12 relative (the FP64 update and the face-order gather conserve to
    round-off)."""
    case = cases.vortex_tets(precision="fp32+acc64")
    vol = case.mesh.cell_volume[: case.mesh.n_owned_cells]
    no = case.mesh.n_owned_cells
    with EulerDevice(case.mesh, case.scheme, case.bc_kind, case.bc_data) as dev:
        dev.upload(case.u0)
        before = (case.u0[:, :no] * vol).sum(axis=1)
        r = dev.step(cfl=case.cfl, rk=3, n_steps=3)
        after = (dev.download()[:, :no] * vol).sum(axis=1)
    assert r.invalid_cell is None
    for k in (0, 1, 2, 4):
        assert abs(after[k] - before[k]) <= 1e-12 * abs(before[k]), (k, after[k] - before[k])


@pytest.mark.parametrize("precision", ["fp64", "fp32+acc64"])
def test_tuning_variants_are_bit_identical(precision):
    """Every launch choice of the autotuner's space (gradient chunking and blocks, gather-recompute
    or store-gather faces, the stage-0 norms in the gather or in their own pass) gives the same
    bits, states and residual norms, and equals the oracle."""
    case = cases.vortex_tets(16, 16, 6, steps=3, precision=precision)
    u_o, rms_o, *_ = run_oracle(case, case.steps)
    no = case.mesh.n_owned_cells
    for gmode, chunk in ((0, 1), (0, 2), (0, 4), (1, 2), (1, 4), (1, 8), (2, 1), (3, 2), (3, 4),
                         (3, 8)):
        for mode in (0, 1, 2):
            for block in (64, 128) if gmode or chunk == 2 else (64, 256):
                with EulerDevice(case.mesh, case.scheme, case.bc_kind, case.bc_data) as dev:
                    dev.set_tuning(grad_chunk=chunk, grad_block=block, face_mode=mode,
                                   face_block=block, gather_block=256 if block == 64 else 128,
                                   grad_mode=gmode)
                    dev.upload(case.u0)
                    dev.step(cfl=case.cfl, rk=3, n_steps=case.steps)
                    rms, _ = dev.history(case.steps)
                    u = dev.download()
                assert bits_equal(u[:, :no], u_o[:, :no]), (gmode, chunk, mode, block)
                assert bits_equal(rms, rms_o), (gmode, chunk, mode, block)
    if precision == "fp64":
        return
    # mode 4: the products widened on the integer pipe (none, x and y, all), 5-word gathers,
    # two entries in flight bounded for 7 or 6 blocks per SM or four for 5;
    # mode 5: the per-warp TMA row ring of 4 or 8 slots with 2 or 3 gathers in flight
    variants = [dict(grad_mode=4, grad_chunk=ch, grad_widen=w, grad_narrow=g, grad_minb=mb)
                for ch, mb in ((2, 7), (2, 6), (4, 5)) for w in (0, 1, 2) for g in (0, 1)]
    variants += [dict(grad_mode=5, grad_chunk=ch, grad_depth=r, grad_narrow=g)
                 for r in (4, 8) for ch in (2, 3) for g in (0, 1)]
    for i, v in enumerate(variants):
        with EulerDevice(case.mesh, case.scheme, case.bc_kind, case.bc_data) as dev:
            dev.set_tuning(grad_block=128, face_mode=1 + i % 2, **v)
            dev.upload(case.u0)
            dev.step(cfl=case.cfl, rk=3, n_steps=case.steps)
            rms, _ = dev.history(case.steps)
            u = dev.download()
        assert bits_equal(u[:, :no], u_o[:, :no]), v
        assert bits_equal(rms, rms_o), v


@pytest.mark.parametrize("precision", ["fp64", "fp32+acc64"])
def test_gradient_stagings_agree_on_the_channel(precision):
    """The hybrid bump channel (hexahedra, prisms and polyhedral bricks: about 23 stencil entries
    per cell, boundary faces in the stencils, local steps): every gradient staging and depth gives
    the bits of the per-thread loads."""
    case = cases.bump_channel(24, 10, 4, steps=3, precision=precision)
    out = {}
    norms = {}
    for gmode, chunk, block in ((0, 1, 128), (1, 4, 128), (2, 1, 64), (3, 2, 64), (3, 4, 128),
                                (3, 8, 128)):  # fmt: skip
        with EulerDevice(case.mesh, case.scheme, case.bc_kind, case.bc_data) as dev:
            dev.set_tuning(grad_chunk=chunk, grad_block=block, face_mode=1 + gmode % 2,
                           face_block=128, gather_block=128, grad_mode=gmode)  # fmt: skip
            dev.upload(case.u0)
            dev.step(cfl=case.cfl, local=True, rk=3, n_steps=case.steps)
            norms[(gmode, chunk, block)] = dev.history(case.steps)[0]
            out[(gmode, chunk, block)] = dev.download()
    if precision != "fp64":
        variants = [dict(grad_mode=4, grad_chunk=ch, grad_widen=w, grad_narrow=g, grad_minb=mb)
                    for ch, mb, w, g in ((2, 7, 0, 1), (2, 7, 1, 0), (2, 6, 2, 1), (4, 5, 0, 0),
                                         (4, 5, 1, 1))]
        variants += [dict(grad_mode=5, grad_chunk=ch, grad_depth=r, grad_narrow=g)
                     for r, ch, g in ((4, 2, 0), (8, 3, 1), (4, 3, 1), (8, 2, 0))]
        for v in variants:
            with EulerDevice(case.mesh, case.scheme, case.bc_kind, case.bc_data) as dev:
                dev.set_tuning(grad_block=128, face_mode=1, face_block=128, gather_block=128, **v)
                dev.upload(case.u0)
                dev.step(cfl=case.cfl, local=True, rk=3, n_steps=case.steps)
                out[tuple(sorted(v.items()))] = dev.download()
    first = out[(0, 1, 128)]
    for k, u in out.items():
        assert bits_equal(u, first), k
    for k, r in norms.items():
        assert bits_equal(r, norms[(0, 1, 128)]), k


def test_autotune_leaves_the_solution_unchanged():
    case = cases.vortex_tets(20, 20, 6, steps=3, precision="fp32+acc64")
    a, *_ = run_device(case, case.steps)
    with EulerDevice(case.mesh, case.scheme, case.bc_kind, case.bc_data) as dev:
        dev.upload(case.u0)
        tuned, ms = dev.autotune(cfl=case.cfl, rk=3, trial_steps=1)
        assert ms > 0 and dev.tuning() == tuned
        dev.step(cfl=case.cfl, rk=3, n_steps=case.steps)
        b = dev.download()
    assert bits_equal(a, b)


@pytest.mark.parametrize("case", CASES)
def test_golden_face_parts(case):
    """Euler<P>::face_parts: the residual's face part and every owned face's flux."""
    mesh, scheme, z = O.load_case(GOLDEN / f"{case}.npz")
    o = O.Oracle(mesh, scheme, z["bc_kind"], z["bc"], z["source"])
    rf0, ff0 = o.face_parts(z["u"])
    with device_of(mesh, scheme, z["bc_kind"], z["bc"], z["source"]) as dev:
        rf, ff = dev.face_parts(z["u"])
    n = mesh["n_owned_cells"]
    if case in EXP_LOG:
        assert rel_err(rf[:, :n], rf0[:, :n]) <= 1e-12 and rel_err(ff, ff0) <= 1e-12
    else:
        assert bits_equal(rf[:, :n], rf0[:, :n]) and bits_equal(ff, ff0)


@pytest.mark.parametrize("case", CASES)
def test_golden_boundary_pressure(case):
    """Euler<P>::boundary_pressure after a residual of the same state."""
    mesh, scheme, z = O.load_case(GOLDEN / f"{case}.npz")
    o = O.Oracle(mesh, scheme, z["bc_kind"], z["bc"], z["source"])
    o.residual(z["u"])
    p0, f0 = o.boundary_pressure()
    with device_of(mesh, scheme, z["bc_kind"], z["bc"], z["source"]) as dev:
        p, f = dev.boundary_pressure(z["u"])
    if case in EXP_LOG:
        assert rel_err(p, p0) <= 1e-12 and rel_err(f, f0) <= 1e-12
    else:
        assert bits_equal(p, p0) and bits_equal(f, f0)


@pytest.mark.parametrize("case", CASES)
def test_golden_conservation_sums(case):
    """check_conservation's exact sums of the device state, against the oracle's face parts."""
    mesh, scheme, z = O.load_case(GOLDEN / f"{case}.npz")
    o = O.Oracle(mesh, scheme, z["bc_kind"], z["bc"], z["source"])
    want = O.conservation_sums(mesh, *o.face_parts(z["u"]))
    with device_of(mesh, scheme, z["bc_kind"], z["bc"], z["source"]) as dev:
        dev.upload(z["u"])
        sums, d = dev.conservation()
    off = mesh["cell_face_offsets"]
    assert d == int(np.diff(off[: mesh["n_owned_cells"] + 1]).max())
    if case in EXP_LOG:
        # E is a cancellation: compare it on the scale of D; the other rows relatively
        assert np.all(np.abs(sums[0] - want[0]) <= 1e-12 * want[1])
        assert np.allclose(sums[1:], want[1:], rtol=1e-12, atol=0.0)
    else:
        assert bits_equal(sums, want)


def test_conservation_jittered_box_within_gate_bound():
    """A non-periodic jittered tetrahedral box (38 400 cells, slip walls), second order, HLLC,
    fp32+acc64: the device's E_k / D_k within tau = max(64 2^-52, 2 gamma_(d+2)), and its exact
    sums equal to the oracle's."""
    from autan_b200 import mesh as M

    n = (40, 40, 4)
    ext = (1.0, 1.0, 0.1)
    disp = M.vortex_jitter(n, ext, 0.2, 0)
    mesh = M.lattice("tetra", n, (0, 0, 0), ext, (False, False, False), displacement=disp,
                     rcm="morton")  # fmt: skip
    case = cases.vortex_tets(24, 24, 6)  # the scheme of the tetrahedral workload
    kind = np.full(mesh.n_boundary_faces, M.BC_SLIP, dtype=np.uint8)
    rng = np.random.default_rng(3)
    x = mesh.cell_centroid
    rho = 1.0 + 0.1 * np.sin(6 * x[0]) * np.cos(5 * x[1])
    u = np.stack([rho, rho * (0.3 + 0.05 * x[1]), rho * 0.1 * x[0], 0.01 * rng.standard_normal(mesh.n_cells),
                  2.5 + 0.1 * np.cos(4 * x[0])])  # fmt: skip
    with EulerDevice(mesh, case.scheme, bc_kind=kind) as dev:
        dev.upload(u)
        sums, d = dev.conservation()
    md = cases.oracle_mesh_dict(cases.Case("box", mesh, case.scheme, kind, np.zeros((5, mesh.n_boundary_faces)),
                                           u, 3, 0.8, 1))  # fmt: skip
    o = O.Oracle(md, case.scheme.as_dict(), kind, np.zeros((5, mesh.n_boundary_faces)), None)
    want = O.conservation_sums(md, *o.face_parts(u))
    assert bits_equal(sums, want)
    m = d + 2
    tau = max(64 * 2.0**-52, 2 * m * 2.0**-53 / (1 - m * 2.0**-53))
    E, D = sums[0], sums[1]
    assert np.all(D > 0)
    assert np.all(np.abs(E) / D <= tau), np.abs(E) / D


@pytest.mark.parametrize("precision", ["fp64", "fp32+acc64"])
def test_bump_channel_local_steps(precision):
    """The hybrid bump channel (hexahedra, prisms, polyhedral bricks; AUSM+-up, total-pressure
    inlet, static-pressure outlet, slip walls), 5 SSP-RK3 steps with local time steps at CFL 1.5,
    against the oracle in the same precision: the inlet state's pow/exp/log are CUDA's on the device
    and the C library's in the oracle, so the bound is 1e-12 relative in FP64 and 1e-5 in
    fp32+acc64 (a last-place difference of the float inlet state carried through 5 steps)."""
    case = cases.bump_channel(24, 12, 4, precision=precision, steps=5)
    u_d, r, rms_d, _ = run_device(case, case.steps, local=True)
    u_o, rms_o, _, bad = run_oracle(case, case.steps, local=True)
    assert bad == -1 and r.invalid_cell is None
    bound = 1e-12 if precision == "fp64" else 1e-5
    assert rel_err(u_d, u_o) <= bound
    assert rel_err(rms_d, rms_o) <= 1e3 * bound


def test_bump_channel_conservation_gate():
    """D2 gate 7 on the hybrid channel after 20 local steps (fp32+acc64): the device's E_k / D_k
    within tau = max(64 2^-52, 2 gamma_(d+2)) for every equation."""
    case = cases.bump_channel(30, 15, 4, steps=20)
    with EulerDevice(case.mesh, case.scheme, case.bc_kind, case.bc_data) as dev:
        dev.upload(case.u0)
        dev.step(cfl=case.cfl, rk=case.rk, n_steps=case.steps, local=True)
        sums, d = dev.conservation()
    m = d + 2
    tau = max(64 * 2.0**-52, 2 * m * 2.0**-53 / (1 - m * 2.0**-53))
    E, D = sums[0], sums[1]
    assert np.all(np.isfinite(sums)) and np.all(D > 0)
    assert np.all(np.abs(E) / D <= tau), np.abs(E) / D


def test_march_to_convergence_matches_the_oracle():
    """A steady march (autan_euler_device_march, batches of 7 graph-launched steps) of a small
    channel (state inlet, pressure outlet, slip walls; no exp/log on the path), fp64, local steps at
    CFL 1.5, to a 2-decade drop: the same converged iteration and the same residual bits as the
    oracle's steps fed to the rule's restatement."""
    from autan_b200 import mesh as M

    case = cases.bump_channel(12, 6, 2, precision="fp64")
    kind, data = case.bc_kind.copy(), case.bc_data.copy()
    inlet = kind == M.BC_INLET
    kind[inlet] = M.BC_STATE
    data[:, inlet] = np.array([1.0, 0.5, 0.0, 0.0, 1.0 / 1.4])[:, None]
    with EulerDevice(case.mesh, case.scheme, kind, data) as dev:
        dev.upload(case.u0)
        res = dev.march(cfl=1.5, local=True, rk=3, max_steps=2000, batch=7, orders=2.0)
    assert res["converged"] and res["invalid_cell"] is None
    assert 0 <= res["steps"] - res["iterations"] < 7
    md = cases.oracle_mesh_dict(cases.Case("march", case.mesh, case.scheme, kind, data, case.u0,
                                           3, 1.5, 1, True))  # fmt: skip
    o = O.Oracle(md, case.scheme.as_dict(), kind, data)
    u = case.u0.copy()
    norms = [o.step(u, rk=3, cfl=1.5, local=True)[0] for _ in range(res["steps"])]
    it, mask = O.convergence_iteration(np.array(norms), 2.0)
    assert (it, mask) == (res["iterations"], res["plateau_mask"])
    assert bits_equal(res["first"], norms[0]) and bits_equal(res["last"], norms[it - 1])


@pytest.mark.parametrize("which", ["channel", "tets", "hex"])
def test_checkpoint_and_resume_are_bit_identical(which):
    """A checkpoint is the FP64 state downloaded from the device (DeviceStepper::download, what the
    reference's checkpoint.cgns holds, runtime/src/run.cpp:2391-2480); resuming uploads it into a
    new stepper. Two steps, a checkpoint, two more steps on a fresh handle give the bits of four
    uninterrupted steps: the step carries no state beyond the conserved state."""
    if which == "channel":
        case = cases.bump_channel(24, 12, 4, steps=4)
    elif which == "tets":
        case = cases.vortex_tets(12, 12, 3, steps=4, extent=(10.0, 10.0, 2.5))
    else:
        case = cases.vortex_hex(16, 16, 2, steps=4)

    def run(u, n):
        with EulerDevice(case.mesh, case.scheme, case.bc_kind, case.bc_data) as dev:
            dev.upload(u)
            dev.step(cfl=case.cfl, rk=case.rk, local=case.local, n_steps=n)
            return dev.download()

    straight = run(case.u0, 4)
    resumed = run(run(case.u0, 2), 2)
    no = case.mesh.n_owned_cells
    assert bits_equal(resumed[:, :no], straight[:, :no])
