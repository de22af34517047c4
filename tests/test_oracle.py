"""The oracle pinned against the reference's golden J-V curves (SimSS 5.36 runs committed in the
reference's tests/data) at the reference's own tolerances, and its invariants.

Tolerances and solvers follow the reference's tests (jaxdd tests/test_solver.py): 194-204
(thin_l1_light 1e-5), 254-273 (held 1e-9, both solvers), 275-299 (regions 1e-6 / 2e-5), 302-321
(two regions 2e-6), 878-888 (ions 2e-5), 890-906 (interface traps), 1318-1345 (resistances),
1348-1358 (uniform generation), 408-420 (logarithmic scan), 1556-1575 (dark, batch, invariants),
277-290 of the differential current (1e-9 single, 1e-8 batch). Beside the curves: the hand-written
Jacobian against differences of the residual, the bordered solve against a dense one, two passes
against one, Newton's end at a step that is not a number, the ions' numbers, the Bernoulli
functions, and `solve_state` against `solve_states`."""

import numpy as np
import pytest

from conftest import GOLDEN
from jaxdd_b200.device import build_device
from jaxdd_b200.simss_input import read_setup, simss_voltages
from oracle import dd

#: case -> (tolerance of solve_jv, tolerance of solve_batch or None)
GOLDENS = {
    "thin_l1_light": (1e-5, None),
    "frozen_1e17_x1_thin_light": (2e-5, None),
    "steady_1e17_thin_light": (2e-5, None),
    "held_thin_light": (1e-9, 1e-9),
    "iface_charged_light": (1e-5, 1e-5),
    "iface_ions_light": (2e-5, None),
    "pin_iface_light": (1e-5, None),
    "region_etl_light": (1e-6, 1e-6),
    "region_htl_frozen_light": (2e-5, 2e-5),
    "two_regions_light": (2e-6, 2e-6),
    "frozen_thick_htl_dark": (None, 2e-5),
    "diff_iface_light": (1e-9, 1e-8),
    "none_light": (1e-5, None),
    "resist_light": (1e-5, 1e-5),
    "logv_light": (1e-5, None),
}


def _case(case):
    setup = read_setup(GOLDEN / "inputs" / case / "simulation_setup.txt")
    ref = np.genfromtxt(GOLDEN / "inputs" / case / "JV.dat", names=True)
    V = simss_voltages(setup) if case == "logv_light" else ref["Vint"]
    return build_device(setup, grid="simss"), V, ref


@pytest.mark.parametrize("case", list(GOLDENS))
def test_oracle_reproduces_simss(case):
    dev, V, ref = _case(case)
    scale = np.max(np.abs(ref["Jext"]))
    tol_jv, tol_batch = GOLDENS[case]
    if tol_jv is not None:
        J, ok, _ = dd.solve_jv(dev, V, bernoulli_name="simss")
        assert ok.all()
        assert np.max(np.abs(J - ref["Jext"])) < tol_jv * scale
    if tol_batch is not None:
        J, ok, _ = dd.solve_batch(dd.prepare([dev]), V, bernoulli_name="simss")
        assert ok.all()
        assert np.max(np.abs(J[0] - ref["Jext"])) < tol_batch * scale
        if case == "resist_light":  # V_ext = V_int + J·R_series against SimSS's
            assert np.max(np.abs(V + J[0] * dev.R_series - ref["Vext"])) < 1e-4
        if case == "frozen_thick_htl_dark":  # dark: monotone, zero at 0 V
            b = dd.prepare([dev])
            js = float(b["J_scale"][0])
            assert np.all(np.diff(J[0]) > -dd.CURRENT_TOL * js)
            assert abs(J[0][np.argmin(np.abs(V))]) < dd.CURRENT_TOL * js


def test_batch_equals_single_and_mixed_batches():
    """A batch of different devices (one with four ion slots, one with two, one without ions)
    gives each device the curve it has alone (tests/test_solver.py:1479-1533)."""
    names = ["two_regions_light", "pin_iface_light", "thin_l1_light"]
    devs = [_case(c)[0] for c in names]
    V = np.round(np.arange(-0.1, 1.25 + 1e-9, 0.05), 6)
    J, ok, _ = dd.solve_batch(dd.prepare(devs), V)
    assert ok.all()
    for k, dev in enumerate(devs):
        Js, oks, _ = dd.solve_batch(dd.prepare([dev]), V)
        scale = float(dd.prepare([dev])["J_scale"][0])
        assert np.max(np.abs(J[k] - Js[0])) < 1e-9 * scale


@pytest.mark.parametrize("x", [-30.0, -1.0, -1e-3, 1e-3, 0.3, 2.0, 30.0])
def test_bernoulli_identity(x):
    """B(−x) = B(x) + x (tests/test_solver.py:56-59), and B' by central differences."""
    for bern in (dd.bern_exact,):
        assert float(bern(-x)[0]) == pytest.approx(float(bern(x)[0]) + x, rel=1e-12, abs=1e-14)
        h = 1e-6 * max(1.0, abs(x))
        fd = (bern(x + h)[0] - bern(x - h)[0]) / (2 * h)
        assert float(bern(x)[1]) == pytest.approx(float(fd), rel=1e-6, abs=1e-9)


def test_block_sweep_equals_a_dense_solve():
    """The block Thomas sweep against a dense solve (tests/test_solver.py:1753-1773)."""
    rng = np.random.default_rng(0)
    nb, NP, m = 3, 12, 3
    A = rng.normal(size=(nb, NP, 3, 3))
    C = rng.normal(size=(nb, NP, 3, 3))
    Bb = rng.normal(size=(nb, NP, 3, 3)) + 8 * np.eye(3)
    A[:, 0] = 0
    C[:, -1] = 0
    d = rng.normal(size=(nb, NP, 3, m))
    x = dd.block_thomas(A, Bb, C, d)
    for b in range(nb):
        M = np.zeros((3 * NP, 3 * NP))
        for i in range(NP):
            M[3 * i:3 * i + 3, 3 * i:3 * i + 3] = Bb[b, i]
            if i:
                M[3 * i:3 * i + 3, 3 * i - 3:3 * i] = A[b, i]
            if i < NP - 1:
                M[3 * i:3 * i + 3, 3 * i + 3:3 * i + 6] = C[b, i]
        ref = np.linalg.solve(M, d[b].reshape(3 * NP, m))
        assert np.allclose(x[b].reshape(3 * NP, m), ref, rtol=1e-10, atol=1e-12)


def test_short_circuit_current_never_exceeds_the_generation():
    """|J_sc| ≤ the generation's current (tests/test_solver.py:207-215)."""
    dev, _, _ = _case("thin_l1_light")
    J, ok, _ = dd.solve_jv(dev, np.array([0.0]))
    from jaxdd_b200.constants import Q
    generated = Q * np.sum(dev.h[:-1] * dev.G[:-1]) / np.sum(dev.h[:-1]) * dev.L
    assert ok.all() and -J[0] <= generated * (1 + 1e-9)


def test_states_restatement_is_consistent_with_the_curves():
    """`solve_states` (batch.py:1165-1191) restated: its J and flags are `solve_batch`'s, the
    contacts' states are their boundary values, the splitting is V_T ln(n p / n_i^2), and the
    radiative measures are finite with PLQY below one (radiative recombination is a part of the
    generation at most)."""
    from jaxdd_b200.workloads import drawn_devices
    devs = drawn_devices(2, NP=60)
    b = dd.prepare(devs)
    V = [0.9, 0.0, 0.5]
    st = dd.solve_states(b, V)
    J, ok, _ = dd.solve_batch(b, V)
    assert np.array_equal(st["J"], J) and np.array_equal(st["converged"], ok)
    assert st["V"].shape == (2, 3, 62) and st["implied_voc"].shape == (2, 3)
    bnd = dd.bounds(b, np.full(2, 0.5))
    assert np.allclose(st["V"][:, 2, 0], bnd[:, 0, 0]) and np.allclose(st["V"][:, 2, -1], bnd[:, 1, 0])
    ni2 = b["rec"]["ni2"][:, None, :]
    assert np.allclose(st["qfls"], b["Vt"][:, None, None] * np.log(st["n"] * st["p"] / ni2))
    assert np.all(np.isfinite(st["implied_voc"])) and np.all((st["plqy"] > 0) & (st["plqy"] < 1))
    # the ions at the boundary points are their neighbours'
    assert np.array_equal(st["anion"][..., 0], st["anion"][..., 1])


def test_state_restatement_is_each_devices_batch_state():
    """`solve_state` (solver.py:2063-2093) restated: as the reference checks it against
    `solve_states` (tests/test_free_surface.py:290-310), each device's implied V_oc to 1e-8 V,
    its PLQY to 1e-7 and its densities to 1e-7 where Newton weighs them (above its floor), for
    the SimSS cell of `none_light` and that of `resist_light` (a shunt of 0.3 Ohm m^2), the
    p-i-n cell and a frozen and a free-ion drawn device, at 0 and 0.8 V; its current is
    `solve_jv`'s at the same voltage less the shunt's (to the bit without a shunt, to 1e-12 of
    it with one), which pins it on SimSS's curve through `test_oracle_reproduces_simss`; and a
    generation factor scales the generation as `solve_jv`'s does."""
    from jaxdd_b200.workloads import drawn_devices, pin_stack
    cell = build_device(read_setup(GOLDEN / "inputs" / "none_light" / "simulation_setup.txt"))
    shunted = build_device(read_setup(GOLDEN / "inputs" / "resist_light" / "simulation_setup.txt"))
    assert shunted.R_shunt > 0
    devs = [cell, shunted, pin_stack(NP=120)] + drawn_devices(2, NP=120)
    for d in devs:
        for V in (0.0, 0.8):
            s = dd.solve_state(d, V)
            b = dd.solve_states(dd.prepare([d]), V)
            assert s["converged"] and b["converged"][0, 0]
            assert s["V"].shape == s["n"].shape == s["anion"].shape == (len(d.x),)
            assert abs(b["implied_voc"][0, 0] - s["implied_voc"]) < 1e-8
            assert abs(b["plqy"][0, 0] / s["plqy"] - 1) < 1e-7
            floor = 1e-12 * np.max(d.N_c)
            for key in ("n", "p"):
                w = s[key] > floor
                np.testing.assert_allclose(b[key][0, 0][w], s[key][w], rtol=1e-7)
            J, ok, _ = dd.solve_jv(d, [V])
            shunt = V / d.R_shunt if d.R_shunt > 0 else 0.0
            assert ok[0] and abs(s["J"] - (J[0] - shunt)) <= 1e-12 * abs(shunt)
            assert np.allclose(s["qfls"], d.Vt * np.log(s["n"] * s["p"] / d.ni ** 2))
    half = dd.solve_state(cell, 0.0, g_frac=0.5)
    J, _, _ = dd.solve_jv(cell, [0.0], g_frac=0.5)
    assert half["J"] == J[0]  # at 0 V the shunt carries nothing
    assert half["plqy"] != dd.solve_state(cell, 0.0)["plqy"]


def test_two_passes_give_the_one_pass_result():
    """jaxdd's two passes (`first_max_iter` steps per voltage, then the devices that missed it
    with `max_iter`) give one pass at `max_iter`'s flags and Newton steps exactly and its curves
    to round-off (tests/test_solver.py:1495-1513), on the reference's three cases, two of them
    twice, one of which needs more than six steps at a voltage; so the GPU kernel, which runs
    the one pass (every lane advancing on its own), returns what the two passes return. Also on
    the benchmark's drawn devices (frozen and free ions)."""
    from jaxdd_b200.workloads import drawn_devices
    cases = ["thin_l1_light", "frozen_1e17_x1_thin_light", "steady_1e17_thin_light"]
    devices = [build_device(read_setup(GOLDEN / "inputs" / c / "simulation_setup.txt"))
               for c in cases]
    V = np.round(np.arange(-0.2, 1.3 + 1e-9, 0.1), 6)
    for devs in (devices + devices[:2], drawn_devices(4, NP=120)):
        b = dd.prepare(devs)
        first = dd.solve_one(b, V, dd.BERNOULLI["exact"], 1e-10, 6, 60)[1]  # the first pass
        one = dd.solve_batch(b, V, first_max_iter=None)
        two = dd.solve_batch(b, V, first_max_iter=6)
        assert one[1].all()
        assert np.array_equal(one[1], two[1]) and np.array_equal(one[2], two[2])
        assert np.max(np.abs(one[0] - two[0])) <= 1e-12 * np.max(np.abs(one[0]))
        if devs[0] is devices[0]:
            assert 0 < (~first.all(axis=1)).sum() < len(devs)  # a second pass ran


def test_newton_ends_at_a_step_that_is_not_a_number():
    """A Newton loop whose iterate is lost ends there, unconverged, after that one step, not at
    `max_iter` (tests/test_solver.py:2115-2131): no later step is a number either, and the lane
    would otherwise pay every one of them. The same loop from the intact start converges."""
    dev, _, _ = _case("steady_1e17_thin_light")
    d = dd.prepare([dev])
    full = dd.initial(d, np.zeros(1))
    y = full[:, 1:-1].copy()
    logs = dd.ion_logs(full[..., 0], d["ion"], d["Vt"])
    _, _, _, ok, it = dd.newton_loop(y, logs, d, 0.0, dd.BERNOULLI["exact"], 1e-10, 50)
    assert ok[0] and 1 < it[0] < 50
    y[0, 7, 1] = np.nan
    _, _, _, ok, it = dd.newton_loop(y, logs, d, 0.0, dd.BERNOULLI["exact"], 1e-10, 50)
    assert not ok[0] and it[0] == 1


def test_free_ions_keep_their_number():
    """The steady state moves the ions, never creates them (tests/test_solver.py:1462-1476):
    at any potential the normalisations `ion_logs` gives make each region's trapezoidal number
    its total (the constraints zero to 1e-12), on the steady-ions case and a two-region one."""
    rng = np.random.default_rng(0)
    for case in ("steady_1e17_thin_light", "two_regions_light"):
        dev, _, _ = _case(case)
        d = dd.prepare([dev])
        V = rng.normal(0.0, 0.3, (1, len(dev.x)))
        logs = dd.ion_logs(V, d["ion"], d["Vt"])
        g, _, _ = dd.ion_constraints(V, logs, d["ion"], d["Vt"])
        assert np.any(dd._masks(d["ion"])[1] > 0)
        assert np.allclose(g, 0.0, atol=1e-12)


def _fd_column(f, x, idx, h=1e-6):
    """Central difference of `f` along one entry `idx` of `x`."""
    xp, xm = x.copy(), x.copy()
    xp[idx] += h
    xm[idx] -= h
    fp, fm = f(xp), f(xm)
    return [(a - b) / (2 * h) for a, b in zip(fp, fm)], fp


@pytest.mark.parametrize("case", ["iface_charged_light", "two_regions_light", "pin_iface_light",
                                  "steady_1e17_thin_light"])
def test_the_blocks_are_the_residuals_derivatives(case):
    """The hand-written Jacobian (the reference takes it by autodiff: tests/test_solver.py's
    `the_jacobian_by_edges_is_autodiff_of_the_rows` and `the_interface_traps_jacobian_is_
    autodiff`) against central differences of the residual at a state off the solution: the
    blocks A, B, C of every row next to a perturbed point, nothing elsewhere; the slots' columns
    U; the constraints' W and D. To 1e-7 of each row's largest entry, beside the difference's
    own rounding (the residual's size over the step)."""
    dev, _, _ = _case(case)
    d = dd.prepare([dev])
    bnd = dd.bounds(d, np.array([0.4]))
    rng = np.random.default_rng(1)
    y = dd.initial(d, np.array([0.4]))[:, 1:-1].copy()
    y[..., 0] += rng.normal(0, 0.02, y.shape[1])
    y[..., 1:] += rng.normal(0, 0.2, (y.shape[1], 2))
    logs = dd.ion_logs(dd.full_of(bnd, y)[..., 0], d["ion"], d["Vt"])
    bern = dd.BERNOULLI["exact"]
    F0, g0, (A, Bb, C, U, W, D) = dd.system(y, logs, bnd, d, d["s"], d["ion"], bern)
    NP, h, eps = y.shape[1], 1e-6, np.finfo(float).eps
    scale = np.maximum(np.maximum(np.abs(A[0]).max(2), np.abs(Bb[0]).max(2)), np.abs(C[0]).max(2))

    def bar(F):  # each row's allowance: 1e-7 of its scale plus the difference's rounding
        return 1e-7 * scale + 100 * eps * np.maximum(np.abs(F[0]), np.abs(F0[0])) / h

    def by_state(yy):
        F, g, _ = dd.system(yy, logs, bnd, d, d["s"], d["ion"], bern)
        return F, g

    interfaces = [i for i in dev.i1[:-1]]
    nodes = sorted({0, 1, NP // 2, NP - 1} | {j for i in interfaces for j in (i - 2, i - 1, i)
                                              if 0 <= j < NP})
    for j in nodes:
        for c in range(3):
            (dF, dg), (Fp, _) = _fd_column(by_state, y, (0, j, c), h)
            an = np.zeros_like(dF[0])
            an[j] = Bb[0, j, :, c]
            if j > 0:
                an[j - 1] = C[0, j - 1, :, c]
            if j < NP - 1:
                an[j + 1] = A[0, j + 1, :, c]
            assert np.all(np.abs(dF[0] - an) <= bar(Fp)), (j, c)
            if c == 0:
                assert np.allclose(dg[0], W[0, :, j], rtol=0, atol=1e-7 * np.max(np.abs(W)) + 1e-30)
            else:
                assert np.all(dg == 0)
    held = dd._held(d["ion"])[0]
    for k in range(logs.shape[1]):
        (dF, dg), (Fp, _) = _fd_column(
            lambda ll: dd.system(y, ll, bnd, d, d["s"], d["ion"], bern)[:2], logs, (0, k), h)
        assert np.all(np.abs(dF[0] - U[0, :, :, k]) <= bar(Fp)), k
        if not held[k]:
            assert np.allclose(dg[0], D[0, :, k], rtol=0, atol=1e-7)


def test_the_bordered_system_is_solved():
    """The bordered solve (batch.py:595-603: the block sweep on 1 + K right-hand sides, then
    the K x K Schur complement) against a dense solve of the whole system [[T, U], [W, D]]
    (tests/test_solver.py's `the_bordered_system_and_its_transpose_are_solved`), for the
    steady form (W on the potential only) and the time step's (W on every unknown), K = 2
    and 4."""
    from oracle import transient
    rng = np.random.default_rng(3)
    for m, K, solve in ((3, 2, dd.bordered_solve), (3, 4, dd.bordered_solve),
                        (5, 2, transient.bordered_solve), (5, 4, transient.bordered_solve)):
        nb, NP = 2, 9
        A = rng.normal(size=(nb, NP, m, m))
        C = rng.normal(size=(nb, NP, m, m))
        Bb = rng.normal(size=(nb, NP, m, m)) + 8 * m * np.eye(m)
        A[:, 0] = 0
        C[:, -1] = 0
        U = rng.normal(size=(nb, NP, m, K))
        W = rng.normal(size=(nb, K, NP)) if m == 3 else rng.normal(size=(nb, K, NP, m))
        D = rng.normal(size=(nb, K, K)) + 4 * NP * np.eye(K)
        r, rg = rng.normal(size=(nb, NP, m)), rng.normal(size=(nb, K))
        x, z = solve(A, Bb, C, U, W, D, r, rg)
        for b in range(nb):
            n = m * NP
            M = np.zeros((n + K, n + K))
            for i in range(NP):
                M[m * i:m * i + m, m * i:m * i + m] = Bb[b, i]
                if i:
                    M[m * i:m * i + m, m * i - m:m * i] = A[b, i]
                if i < NP - 1:
                    M[m * i:m * i + m, m * i + m:m * i + 2 * m] = C[b, i]
            M[:n, n:] = U[b].reshape(n, K)
            if m == 3:
                M[n:, 0:n:3] = W[b]
            else:
                M[n:, :n] = W[b].reshape(K, n)
            M[n:, n:] = D[b]
            ref = np.linalg.solve(M, np.concatenate([r[b].reshape(n), rg[b]]))
            assert np.allclose(np.concatenate([x[b].reshape(n), z[b]]), ref, rtol=1e-10,
                               atol=1e-12)


def test_bernoulli_is_finite_at_zero_and_simss_is_within_its_own_error():
    """B(0) = 1 and B'(0) = -1/2, neither seeing 0/0 (tests/test_solver.py:50-53); SIMsalabim's
    Bernoulli function is the exact one to 1e-3 over [-5, 5] (tests/test_solver.py:62-64)."""
    B, dB = dd.bern_exact(np.array([0.0]))
    assert B[0] == 1.0 and dB[0] == pytest.approx(-0.5)
    x = np.linspace(-5.0, 5.0, 2001)
    assert np.max(np.abs(dd.bern_simss(x)[0] / dd.bern_exact(x)[0] - 1)) < 1e-3
