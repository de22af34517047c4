"""`solve_impedance` on the GPU (`dd_admittance`, and `dd_admittance_ions` with mobile ions)
against the oracle's restatement of jaxdd's `_admittance` (with bulk and interface traps following
at their own rates, the ions as unknowns of their own), and the reference's known answers on the
GPU's own results: the steady slope at a very low frequency (against the GPU's `solve_states`
differenced, the ions moving with the voltage), the geometric capacitance far above every
relaxation."""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from jaxdd_b200 import prepare, solve_states  # noqa: E402
from jaxdd_b200.device import build_device  # noqa: E402
from jaxdd_b200.impedance import solve_impedance  # noqa: E402
from jaxdd_b200.simss_input import setup_from_texts  # noqa: E402
from jaxdd_b200.workloads import drawn_texts, pin_texts  # noqa: E402
from oracle import impedance as imp  # noqa: E402

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA GPU")]

F = np.array([1.0, 1e3, 1e5, 1e6, 1e9])


def _devices(NP=100):
    """The p-i-n cell, with interface traps, and two of the drawn stacks without their ions."""
    out = [build_device(setup_from_texts(pin_texts(NP)))]
    t = pin_texts(NP)
    for name in ("L1.txt", "L2.txt"):
        t[name] = t[name].replace("N_t_int = 0", "N_t_int = 1e15")
    out.append(build_device(setup_from_texts(t)))
    for k in (1, 3):
        t = drawn_texts(k, np.random.default_rng([20261203, k]), NP)
        for key in ("N_anion", "N_cation", "mu_anion", "mu_cation"):
            t["L2.txt"] = "\n".join(f"{key} = 0" if line.split("=")[0].strip() == key else line
                                    for line in t["L2.txt"].splitlines()) + "\n"
        t["L2.txt"] = t["L2.txt"].replace("ionsMayEnter = 1", "ionsMayEnter = 0")
        out.append(build_device(setup_from_texts(t)))
    return out


def test_admittance_matches_the_oracle():
    devs = _devices()
    r = solve_impedance(prepare(devs), F, voltage=0.7)
    Yo, Zo, Jo, oko = imp.solve_impedance(devs, F, voltage=0.7)
    assert np.array_equal(r.converged, oko) and r.converged.all()
    rel = np.abs(r.Y - Yo) / np.abs(Yo)
    assert np.max(rel) < 1e-6, rel
    np.testing.assert_allclose(r.Z, Zo, rtol=1e-6)


def test_the_limits_on_the_gpu():
    devs = _devices()[:2]
    V0, dV = 0.6, 1e-5
    r = solve_impedance(prepare(devs), [1e-7, 1e14], voltage=V0, tol=1e-12, max_iter=200)
    st = solve_states(prepare(devs), [V0 - dV, V0 + dV], tol=1e-12, max_iter=200)
    slope = (st["J"][:, 1] - st["J"][:, 0]) / (2 * dV)
    np.testing.assert_allclose(r.Y[:, 0].real, slope, rtol=1e-6)
    for k, d in enumerate(devs):
        x, eps = np.asarray(d.x), np.asarray(d.eps)
        geometric = 1.0 / np.sum(np.diff(x) * 0.5 * (1 / eps[:-1] + 1 / eps[1:]))
        assert r.capacitance[k, 1] == pytest.approx(geometric, rel=1e-4)


def test_with_mobile_ions_matches_the_oracle():
    """`dd_admittance_ions`: the drawn mobile-ion stacks with free mobile ions (5×5 blocks, each
    region's number kept), and in the same batch the p-i-n cell without ions (its ions' rows
    identities), against the oracle (`admittance_ions`, and `admittance` for the cell)."""
    from jaxdd_b200.workloads import transient_devices
    devs = transient_devices(3, NP=100) + [build_device(setup_from_texts(pin_texts(100)))]
    r = solve_impedance(prepare(devs), F, voltage=0.8)
    Yo, Zo, Jo, oko = imp.solve_impedance(devs, F, voltage=0.8)
    assert np.array_equal(r.converged, oko) and r.converged.all()
    rel = np.abs(r.Y - Yo) / np.abs(Yo)
    assert np.max(rel) < 1e-6, rel


def test_with_mobile_ions_the_low_frequency_limit_is_the_steady_slope():
    from jaxdd_b200.workloads import transient_devices
    devs = transient_devices(2, NP=100)
    V0, dV = 0.8, 1e-5
    r = solve_impedance(prepare(devs), [1e-7], voltage=V0, tol=1e-12, max_iter=200)
    st = solve_states(prepare(devs), [V0 - dV, V0 + dV], tol=1e-12, max_iter=200)
    slope = (st["J"][:, 1] - st["J"][:, 0]) / (2 * dV)
    np.testing.assert_allclose(r.Y[:, 0].real, slope, rtol=1e-5)
    assert np.all(np.abs(r.Y[:, 0].imag) < 1e-4 * np.abs(slope))


def test_what_impedance_refuses():
    from jaxdd_b200.workloads import drawn_devices
    with pytest.raises(NotImplementedError, match="frozen"):
        solve_impedance(prepare(drawn_devices(2, NP=50)), [1e3])


def _fast_ion_stack(NP=60, differential=False):
    """One of the drawn mobile-ion stacks with its ions at 1e-9 m²/Vs: they follow at 1 kHz."""
    from jaxdd_b200.workloads import SEED_ION_STACKS
    k = 1
    texts = drawn_texts(k, np.random.default_rng([SEED_ION_STACKS, k]), NP)
    texts["L2.txt"] = "\n".join(
        f"{line.split('=')[0].strip()} = 1e-9"
        if line.split("=")[0].strip() in ("mu_anion", "mu_cation") else line
        for line in texts["L2.txt"].splitlines()) + "\n"
    return build_device(setup_from_texts(_differential(texts) if differential else texts))


def _differential(texts):
    """The same device with SIMsalabim's differential current (`currDiffInt = 1`)."""
    setup = texts["simulation_setup.txt"]
    assert "currDiffInt = 2" in setup
    return dict(texts, **{"simulation_setup.txt": setup.replace("currDiffInt = 2",
                                                                "currDiffInt = 1")})


@pytest.mark.parametrize("bernoulli_name", ["exact", "simss"])
def test_the_differential_current_matches_the_oracle(bernoulli_name):
    """`currDiffInt = 1` (each interval's Scharfetter–Gummel flux in the current, jaxdd
    batch.py:366-369, 471-479) in both kernels: the p-i-n cell with and without interface traps
    and two drawn stacks without ions (`dd_admittance`), then two mobile-ion stacks with the
    differential current beside one with the integral form (`dd_admittance_ions`), against the
    oracle to 1e-6."""
    from jaxdd_b200.workloads import SEED_ION_STACKS
    plain = []
    for interface in (False, True):
        t = pin_texts(100)
        if interface:
            for name in ("L1.txt", "L2.txt"):
                t[name] = t[name].replace("N_t_int = 0", "N_t_int = 1e15")
        plain.append(build_device(setup_from_texts(_differential(t))))
    ions = [build_device(setup_from_texts(_differential(drawn_texts(
        k, np.random.default_rng([SEED_ION_STACKS, k]), 100)))) for k in (1, 3)]
    ions.append(build_device(setup_from_texts(drawn_texts(
        5, np.random.default_rng([SEED_ION_STACKS, 5]), 100))))
    assert [d.curr_diff for d in ions] == [True, True, False]
    for devs, V0 in ((plain, 0.7), (ions, 0.8)):
        r = solve_impedance(prepare(devs), F, voltage=V0, bernoulli_name=bernoulli_name)
        Yo, Zo, Jo, oko = imp.solve_impedance(devs, F, voltage=V0,
                                              bernoulli_name=bernoulli_name)
        assert np.array_equal(r.converged, oko) and r.converged.all()
        rel = np.abs(r.Y - Yo) / np.abs(Yo)
        assert np.max(rel) < 1e-6, rel


def _gpu_sine_response(dev, V0, f, amp, per_period=40, periods=20, fitted=4):
    """The GPU transient's admittance at `f` from a sine of `amp` on `V0` (jaxdd
    tests/test_impedance.py:47-63's protocol)."""
    from jaxdd_b200.simss_input import TVG
    from jaxdd_b200.transient import solve_transient
    dt = 1.0 / (f * per_period)
    k = np.arange(1, per_period * periods + 1)
    t = np.concatenate([[0.0], k * dt])
    V = np.concatenate([[V0], V0 + amp * np.sin(2 * np.pi * f * k * dt)])
    r = solve_transient(prepare([dev]), TVG.steps(t, V, float(dev.G_frac), 0), tol=1e-12,
                        max_iter=60)
    assert r.converged.all()
    m = k > per_period * (periods - fitted)
    ph = 2 * np.pi * f * k[m] * dt
    X = np.stack([np.ones(m.sum()), np.sin(ph), np.cos(ph)], -1)
    c = np.linalg.lstsq(X, r.J[0, 1:][m], rcond=None)[0]
    return (c[1] + 1j * c[2]) / amp, dt


@pytest.mark.parametrize("case", ["ions", "interface", "ions-differential",
                                  "interface-differential"])
def test_the_dt_form_is_the_gpu_transients_response(case):
    """The two GPU paths against each other: `solve_impedance(..., dt=)` (`dd_admittance_ions`,
    `dd_admittance`) is the GPU transient's (`dd_transient`) response to a small sine at steps of
    dt, with mobile ions following at 1 kHz, and with interface traps at 10 kHz (1e-6 and 1e-7,
    the reference's bars), and the oracle's dt form."""
    differential = case.endswith("-differential")
    if case.startswith("ions"):
        dev, V0, f, amp, bar = _fast_ion_stack(differential=differential), 0.8, 1e3, 1e-4, 1e-6
    else:
        t = pin_texts(60)
        for name in ("L1.txt", "L2.txt"):
            t[name] = t[name].replace("N_t_int = 0", "N_t_int = 1e15")
        if differential:
            t = _differential(t)
        dev, V0, f, amp, bar = build_device(setup_from_texts(t)), 0.6, 1e4, 1e-5, 1e-7
    assert dev.curr_diff == differential
    Yt, dt = _gpu_sine_response(dev, V0, f, amp, periods=20 if case.startswith("ions") else 12)
    r = solve_impedance(prepare([dev]), [f], voltage=V0, tol=1e-12, max_iter=200, dt=dt)
    assert abs(r.Y[0, 0] / Yt - 1) < bar
    Yo = imp.solve_impedance([dev], [f], voltage=V0, tol=1e-12, max_iter=200, dt=dt)[0][0, 0]
    assert abs(r.Y[0, 0] / Yo - 1) < 1e-6


@pytest.mark.parametrize("differential", [False, True])
def test_two_ion_regions_of_each_species_match_the_oracle(differential):
    """`dd_admittance_ions` with four slots (two regions of each species, each its own column of
    the border and its own current), beside two one-region mobile-ion stacks and the p-i-n cell
    without ions in the same launch, with the integral and the differential current, against the
    oracle to 1e-6 (the differential current to 1e-5: each interval's current is the difference
    of two fluxes far larger than it, whose rounding both tangents carry; measured 1.1e-6)."""
    from jaxdd_b200.workloads import SEED_ION_STACKS
    from tests.test_impedance_oracle import two_region_texts
    texts = [two_region_texts(100), two_region_texts(100, "1e-9")]
    texts += [drawn_texts(k, np.random.default_rng([SEED_ION_STACKS, k]), 100) for k in (1, 3)]
    texts.append(pin_texts(100))
    devs = [build_device(setup_from_texts(_differential(t) if differential else t))
            for t in texts]
    b = prepare(devs)
    assert b["ka"] == 2 and b["kc"] == 2
    r = solve_impedance(b, F, voltage=0.8)
    Yo, Zo, Jo, oko = imp.solve_impedance(devs, F, voltage=0.8)
    assert np.array_equal(r.converged, oko) and r.converged.all()
    rel = np.abs(r.Y - Yo) / np.abs(Yo)
    assert np.max(rel) < (1e-5 if differential else 1e-6), rel


@pytest.mark.parametrize("bernoulli_name", ["exact", "simss"])
@pytest.mark.parametrize("differential", [False, True])
def test_ion_regions_at_a_contact_match_the_oracle(bernoulli_name, differential):
    """Ion regions that reach a contact: a region of two layers at the left contact (two slots)
    and two regions of each species at both contacts (four), in one launch each, the contact's
    ions from its neighbour's in each region's number (its derivatives in the neighbour's
    potential and, through the contact's, in V_int) and in the current (the step's and the
    steady state's forms, jaxdd's density of 1 before the step there), with the integral and the
    differential current and both Bernoulli functions, against the oracle to 1e-6; at 1 Hz to
    1e-5, where a region at a contact makes the admittance sensitive to the steady state itself
    (the oracle's own moves 8e-7 between steady states at tol 1e-10 and 1e-13; measured 4e-6),
    and to 1e-5 with the differential current, each interval's current the difference of two
    far larger fluxes (measured 4.5e-6 at 1 kHz)."""
    from tests.test_impedance_oracle import contact_texts
    for case in ("zimt_region_slow_light", "two_regions_light"):
        texts = contact_texts(case, 200)
        devs = [build_device(setup_from_texts(_differential(texts) if differential else texts),
                             grid="simss")]
        assert devs[0].anion_mask[0]
        r = solve_impedance(prepare(devs), F, voltage=0.5, bernoulli_name=bernoulli_name)
        Yo, Zo, Jo, oko = imp.solve_impedance(devs, F, voltage=0.5,
                                              bernoulli_name=bernoulli_name)
        assert np.array_equal(r.converged, oko) and r.converged.all()
        rel = np.abs(r.Y - Yo) / np.abs(Yo)
        bar = 1e-5 if differential else 1e-6
        assert np.max(rel[:, 0]) < 1e-5 and np.max(rel[:, 1:]) < bar, (case, rel)
