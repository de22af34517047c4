"""The CUDA path against the oracle (and through it the reference's goldens), on a B200.

* one Newton step from perturbed states, every quantity, against `oracle.dd.newton_step` and its
  current (the per-step check of jaxdd tests/test_solver.py:1595-1617's approach);
* every golden case through both drop-in solvers, against SimSS at the reference's tolerances and
  against the oracle's own curve and converged flags;
* a batch of drawn devices (the benchmark's distributions) against the oracle's `solve_batch`:
  J within 1e-6 of each device's current scale, the converged flags equal.
"""

import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from conftest import GOLDEN  # noqa: E402
from jaxdd_b200 import _lib  # noqa: E402
from jaxdd_b200.batch import _gpu, descriptor, prepare, solve_batch  # noqa: E402
from jaxdd_b200.device import build_device  # noqa: E402
from jaxdd_b200.simss_input import read_setup, simss_voltages  # noqa: E402
from jaxdd_b200.solver import solve_jv  # noqa: E402
from oracle import dd  # noqa: E402
from test_oracle import GOLDENS  # noqa: E402

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA GPU")]

STEP_CASES = ["thin_l1_light", "steady_1e17_thin_light", "iface_charged_light",
              "two_regions_light", "diff_iface_light", "region_etl_light"]


def _dev(case):
    return build_device(read_setup(GOLDEN / "inputs" / case / "simulation_setup.txt"),
                        grid="simss")


def _kernel_step(batch, y, logs, vint, share, bern):
    """dd_newton_step on lane-ordered arrays (device order in, device order out)."""
    g = _gpu(batch)
    B, Bp, npmax = batch["n"], batch["Bp"], batch["np_max"]
    K = 2 if batch["ka"] + batch["kc"] <= 2 else 4
    lanes = batch["lane_of"]
    yl = np.zeros((npmax + 2, 3, Bp))
    ll = np.zeros((K, Bp))
    vl = np.zeros(Bp)
    for k in range(B):
        NP = y.shape[1]
        yl[1:NP + 1, :, lanes[k]] = y[k]
        ll[:logs.shape[1], lanes[k]] = logs[k]
        vl[lanes[k]] = vint[k]
    ty = torch.from_numpy(yl).cuda()
    tl = torch.from_numpy(ll).cuda()
    tv = torch.from_numpy(vl).cuda()
    size = torch.zeros(Bp, dtype=torch.float64, device="cuda")
    J = torch.zeros(Bp, dtype=torch.float64, device="cuda")
    desc = descriptor(batch, g, ty)
    ws = g.workspace(desc)
    opts = _lib.DdOpts(1e-10, 60, 60, 0, _lib.DD_BERNOULLI[bern], 0, 0, 0)
    _lib.check(_lib.lib().dd_newton_step(
        ctypes.byref(desc), ty.data_ptr(), tl.data_ptr(), tv.data_ptr(), float(share),
        ctypes.byref(opts), size.data_ptr(), J.data_ptr(), ws.data_ptr(), ws.numel(),
        torch.cuda.current_stream().cuda_stream), "dd_newton_step")
    torch.cuda.synchronize()
    yo, lo, so, Jo = ty.cpu().numpy(), tl.cpu().numpy(), size.cpu().numpy(), J.cpu().numpy()
    NP = y.shape[1]
    return (np.stack([yo[1:NP + 1, :, lanes[k]] for k in range(B)]),
            np.stack([lo[:logs.shape[1], lanes[k]] for k in range(B)]),
            so[lanes], Jo[lanes])


@pytest.mark.parametrize("bern", ["exact", "simss"])
def test_one_newton_step_matches_the_oracle(bern):
    devs = [_dev(c) for c in STEP_CASES]
    d = dd.prepare(devs)
    batch = prepare(devs)
    rng = np.random.default_rng(7)
    Vint = np.array([0.3, 0.6, 0.9, 0.1, 1.0, 0.5])
    y = dd.initial(d, Vint)[:, 1:-1]
    y = dd.poisson_solve(y, d, d["s"], d["ion"], Vint, 6)
    y = y + rng.normal(scale=[0.002, 0.05, 0.05], size=y.shape)
    bnd = dd.bounds(d, Vint)
    logs = dd.ion_logs(dd.full_of(bnd, y)[..., 0], d["ion"], d["Vt"]) + rng.normal(scale=0.01, size=(len(devs), 4))
    new, logs_new, size = dd.newton_step(y, logs, bnd, d, d["s"], d["ion"], dd.BERNOULLI[bern])
    J = dd.current(d, dd.full_of(bnd, new), dd.BERNOULLI[bern])
    gy, gl, gs, gJ = _kernel_step(batch, y, logs, Vint, 1.0, bern)
    _assert_same_step(d, y, new, gy)
    assert np.allclose(gl, logs_new, rtol=0, atol=1e-9)
    assert np.allclose(gs, size, rtol=1e-8)
    assert np.all(np.abs(gJ - J) <= 1e-9 * (np.abs(J) + batch["J_scale"]))


def _assert_same_step(d, y, new, gy, tol=1e-8):
    """Steps equal to `tol` of each device's largest, the potential everywhere, a density where
    it is above `n_floor`. Below the floor its logarithm's step is undetermined at round-off
    (jaxdd solver.py:74-88: such a density moves no current and does not count for
    convergence): both solvers clip it, to a sign decided by rounding."""
    step_o, step_g = new - y, gy - y
    above = y[..., 1:] >= np.log(d["s"]["n_floor"])[..., None]
    mask = np.concatenate([np.ones_like(above[..., :1]), above], -1)
    scale = np.max(np.abs(step_o) * mask, axis=(1, 2))[:, None, None] + 1e-300
    assert np.max(np.abs(step_g - step_o) * mask / scale) < tol


def test_a_step_near_the_solution_matches_the_oracle():
    """Twelve Newton steps into a solve, where the steps are small and more of the linear solve's
    digits show."""
    devs = [_dev(c) for c in STEP_CASES]
    d = dd.prepare(devs)
    batch = prepare(devs)
    Vint = np.array([0.3, 0.6, 0.9, 0.1, 1.0, 0.5])
    y = dd.initial(d, Vint)[:, 1:-1]
    y = dd.poisson_solve(y, d, d["s"], d["ion"], Vint, 60)
    bnd = dd.bounds(d, Vint)
    logs = dd.ion_logs(dd.full_of(bnd, y)[..., 0], d["ion"], d["Vt"])
    for _ in range(12):
        y, logs, size = dd.newton_step(y, logs, bnd, d, d["s"], d["ion"], dd.bern_exact)
    new, logs_new, size = dd.newton_step(y, logs, bnd, d, d["s"], d["ion"], dd.bern_exact)
    J = dd.current(d, dd.full_of(bnd, new), dd.bern_exact)
    gy, gl, gs, gJ = _kernel_step(batch, y, logs, Vint, 1.0, "exact")
    _assert_same_step(d, y, new, gy, tol=1e-6)
    assert np.allclose(gl, logs_new, rtol=0, atol=1e-12)
    assert np.all(np.abs(gs - size) <= 1e-6 * size + 1e-14)
    assert np.all(np.abs(gJ - J) <= 1e-10 * batch["J_scale"])


def test_frozen_ions_in_one_step_and_scaled_ions():
    """A step with the ions scaled (an ion-density stage, share 1/16)."""
    devs = [_dev(c) for c in ("steady_1e17_thin_light", "two_regions_light")]
    d = dd.prepare(devs)
    batch = prepare(devs)
    share = 1 / 16
    s_k, ion_k = dd._scaled(d["s"], d["ion"], share)
    dk = dd._with(d, s_k, ion_k)
    Vint = np.array([0.2, 0.7])
    y = dd.initial(d, Vint)[:, 1:-1]
    y = dd.poisson_solve(y, dk, s_k, ion_k, Vint, 8)
    bnd = dd.bounds(d, Vint)
    logs = dd.ion_logs(dd.full_of(bnd, y)[..., 0], ion_k, d["Vt"])
    new, logs_new, size = dd.newton_step(y, logs, bnd, dk, s_k, ion_k, dd.bern_exact)
    gy, gl, gs, gJ = _kernel_step(batch, y, logs, Vint, share, "exact")
    _assert_same_step(dk, y, new, gy)
    assert np.allclose(gl, logs_new, rtol=0, atol=1e-9)


@pytest.mark.parametrize("case", list(GOLDENS))
def test_goldens_through_the_gpu(case):
    setup = read_setup(GOLDEN / "inputs" / case / "simulation_setup.txt")
    ref = np.genfromtxt(GOLDEN / "inputs" / case / "JV.dat", names=True)
    V = simss_voltages(setup) if case == "logv_light" else ref["Vint"]
    dev = build_device(setup, grid="simss")
    scale = np.max(np.abs(ref["Jext"]))
    tol_jv, tol_batch = GOLDENS[case]
    # solve_batch, against SimSS and the oracle
    J, ok, its = solve_batch(prepare([dev]), V, bernoulli_name="simss")
    Jo, oko, itso = dd.solve_batch(dd.prepare([dev]), V, bernoulli_name="simss")
    assert np.array_equal(ok, oko)
    js = float(dd.prepare([dev])["J_scale"][0])
    assert np.max(np.abs(J - Jo)) < 1e-6 * js
    assert np.max(np.abs(J[0] - ref["Jext"])) < max(tol_batch or 0, tol_jv or 0, 2e-5) * scale
    # solve_jv
    if tol_jv is not None:
        r = solve_jv(dev, V, bernoulli_name="simss")
        Jj, okj, _ = dd.solve_jv(dev, V, bernoulli_name="simss")
        assert r.converged.all() and np.array_equal(r.converged, okj)
        assert np.max(np.abs(r.J - ref["Jext"])) < tol_jv * scale
        assert np.max(np.abs(r.J - Jj)) < 1e-6 * js


def test_drawn_devices_match_the_oracle():
    """Twelve devices of the benchmark's distributions (NP 400, half frozen after a 1.0 V
    pre-bias, half with free ions, interface and bulk traps drawn): J within 1e-6 of each
    device's current scale, converged flags equal."""
    from jaxdd_b200.workloads import V_SCAN, drawn_devices
    devs = drawn_devices(12)
    J, ok, its = solve_batch(prepare(devs), V_SCAN)
    od = dd.prepare(devs)
    Jo, oko, _ = dd.solve_batch(od, V_SCAN)
    assert np.array_equal(ok, oko)
    err = np.max(np.abs(J - Jo), axis=1) / od["J_scale"]
    assert np.all(err < 1e-6), err



def test_pin_cell_at_its_full_size_through_both_solvers():
    """The p-i-n cell at its stated size (HTL 20 nm / absorber 400 nm / ETL 30 nm, NP 300, 61
    voltages from -0.2 to 1.3 V) through `solve_jv` and `solve_batch` on the GPU, against the
    oracle's `solve_jv` and `solve_batch` (jaxdd solver.py:2041-2060, batch.py:1136-1162): J within
    1e-6 of the current scale at every voltage, converged flags equal, every point converged."""
    from jaxdd_b200.workloads import V_SCAN, pin_stack
    dev = pin_stack(NP=300)
    assert len(dev.x) == 302
    js = float(dd.prepare([dev])["J_scale"][0])
    r = solve_jv(dev, V_SCAN)
    Jo, oko, _ = dd.solve_jv(dev, V_SCAN)
    assert r.converged.all() and np.array_equal(r.converged, oko)
    assert np.max(np.abs(r.J - Jo)) < 1e-6 * js, np.max(np.abs(r.J - Jo)) / js
    J, ok, _ = solve_batch(prepare([dev]), V_SCAN)
    Jb, okb, _ = dd.solve_batch(dd.prepare([dev]), V_SCAN)
    assert ok.all() and np.array_equal(ok, okb)
    assert np.max(np.abs(J - Jb)) < 1e-6 * js, np.max(np.abs(J - Jb)) / js
    # the two solvers reach the same roots: each curve within the other's tolerance
    assert np.max(np.abs(J[0] - r.J)) < 1e-6 * js


def test_voltage_lists_in_any_order_with_repeats_and_alone():
    """The voltages as a caller may give them (jaxdd batch.py:1043-1045 returns every result in
    the caller's order): unsorted with a voltage repeated, and a single voltage, through
    `solve_batch` and `solve_jv`, for the p-i-n cell and a frozen and a free-ion drawn device,
    against the oracle: J within 1e-6 of the current scale, converged flags equal; a repeated
    voltage's results agree to the same bar wherever it sits in the list."""
    from jaxdd_b200.workloads import drawn_devices, pin_stack
    devs = [pin_stack(NP=120)] + drawn_devices(2, NP=120)
    od = dd.prepare(devs)
    scale = od["J_scale"][:, None]
    V = [0.5, 0.5, -0.1, 1.0, 0.5, 0.2]
    J, ok, its = solve_batch(prepare(devs), V)
    Jo, oko, _ = dd.solve_batch(od, V)
    assert J.shape == ok.shape == its.shape == (3, 6)
    assert np.array_equal(ok, oko) and ok.all()
    assert np.all(np.abs(J - Jo) < 1e-6 * scale)
    assert np.all(np.abs(J[:, [1, 4]] - J[:, [0]]) < 1e-6 * scale)
    J1, ok1, _ = solve_batch(prepare(devs), [0.3])
    Jo1, oko1, _ = dd.solve_batch(od, [0.3])
    assert J1.shape == (3, 1) and np.array_equal(ok1, oko1) and ok1.all()
    assert np.all(np.abs(J1 - Jo1) < 1e-6 * scale)
    for k, d in enumerate(devs):
        for volts in (V, [0.3]):
            r = solve_jv(d, volts)
            Jj, okj, _ = dd.solve_jv(d, volts)
            assert np.array_equal(r.converged, okj) and r.converged.all()
            assert np.max(np.abs(r.J - Jj)) < 1e-6 * scale[k, 0]
            assert np.array_equal(r.V, np.asarray(volts, dtype=float))
