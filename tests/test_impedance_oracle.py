"""The impedance oracle (`oracle/impedance.py`) against the reference's own known answers
(jaxdd tests/test_impedance.py): at a very low frequency the admittance is the steady J-V
curve's slope, far above every relaxation the capacitance is the layers' geometric one,
1/∫dx/ε; `Z = 1/(Y + G_shunt) + R_series`. On workload 1's p-i-n cell, with and without
interface traps; with mobile ions as unknowns of their own (the drawn mobile-ion stacks): at 1e-7 Hz
the steady slope with the ions moving (the reference's bar, 1e-5), far above every relaxation the
capacitance of the same stack without ions (the ions frozen there), ions frozen at a pre-bias
refused as the reference refuses them."""

import numpy as np
import pytest

from jaxdd_b200.device import build_device
from jaxdd_b200.simss_input import setup_from_texts
from jaxdd_b200.workloads import SEED_ION_STACKS, drawn_texts, pin_texts, transient_devices
from oracle import dd
from oracle import impedance as imp


def _cell(NP=60, interface=False):
    texts = pin_texts(NP)
    if interface:
        for name in ("L1.txt", "L2.txt"):
            texts[name] = texts[name].replace("N_t_int = 0", "N_t_int = 1e15")
    return build_device(setup_from_texts(texts))


@pytest.mark.parametrize("interface", [False, True])
def test_low_frequency_is_the_steady_slope(interface):
    dev = _cell(interface=interface)
    V0, dV = 0.6, 1e-5
    Y, _, _, ok = imp.solve_impedance([dev], [1e-7], voltage=V0, tol=1e-12, max_iter=200)
    st = dd.solve_states(dd.prepare([dev]), [V0 - dV, V0 + dV], tol=1e-12, max_iter=200)
    slope = (st["J"][0, 1] - st["J"][0, 0]) / (2 * dV)
    assert ok.all()
    assert Y[0, 0].real == pytest.approx(slope, rel=1e-6)
    assert abs(Y[0, 0].imag) < 1e-4 * abs(slope)


def test_high_frequency_is_the_geometric_capacitance():
    dev = _cell()
    x, eps = np.asarray(dev.x), np.asarray(dev.eps)
    geometric = 1.0 / np.sum(np.diff(x) * 0.5 * (1 / eps[:-1] + 1 / eps[1:]))
    f = np.array([1e6, 1e14])
    Y, _, _, _ = imp.solve_impedance([dev], f, voltage=0.6)
    C = Y.imag / (2 * np.pi * f)
    assert C[0, 1] == pytest.approx(geometric, rel=1e-4)
    assert C[0, 0] > C[0, 1]


def test_the_series_resistance_and_the_shunt():
    texts = pin_texts(60)
    texts["simulation_setup.txt"] = (texts["simulation_setup.txt"]
                                     .replace("R_shunt = -1", "R_shunt = 0.1")
                                     .replace("R_series = 0", "R_series = 1e-4"))
    dev = build_device(setup_from_texts(texts))
    Y, Z, _, _ = imp.solve_impedance([dev], [1e3, 1e6], voltage=0.3)
    np.testing.assert_allclose(Z, 1.0 / (Y + 10.0) + 1e-4, rtol=1e-12)


def _without_ions(texts):
    lines = []
    for line in texts["L2.txt"].splitlines():
        key = line.split("=")[0].strip()
        if key in ("N_anion", "N_cation", "mu_anion", "mu_cation", "ionsMayEnter"):
            line = f"{key} = 0"
        lines.append(line)
    return dict(texts, **{"L2.txt": "\n".join(lines) + "\n"})


@pytest.mark.parametrize("k", [0, 1])
def test_with_ions_low_frequency_is_the_steady_slope(k):
    dev = transient_devices(1, NP=150, start=k)[0]
    assert dev.anion_total > 0 and not dev.pre_cond
    V0, dV = 0.8, 1e-5
    Y, _, _, ok = imp.solve_impedance([dev], [1e-7], voltage=V0, tol=1e-12, max_iter=200)
    st = dd.solve_states(dd.prepare([dev]), [V0 - dV, V0 + dV], tol=1e-12, max_iter=200)
    slope = (st["J"][0, 1] - st["J"][0, 0]) / (2 * dV)
    assert ok.all()
    assert Y[0, 0].real == pytest.approx(slope, rel=1e-5)
    assert abs(Y[0, 0].imag) < 1e-4 * abs(slope)


def test_with_ions_high_frequency_is_the_stack_without_them():
    k = 3
    texts = drawn_texts(k, np.random.default_rng([SEED_ION_STACKS, k]), 150)
    f = np.array([1e6, 1e16])
    C = []
    for t in (texts, _without_ions(texts)):
        Y, _, _, _ = imp.solve_impedance([build_device(setup_from_texts(t))], f, voltage=0.8)
        C.append(Y.imag / (2 * np.pi * f))
    assert C[0][0, 1] == pytest.approx(C[1][0, 1], rel=1e-9)
    # the ions change the steady state (its band bending), so at 1 MHz the two differ
    assert C[0][0, 0] != pytest.approx(C[1][0, 0], rel=1e-3)


def test_with_ions_frozen_at_a_pre_bias_refused():
    k = 0  # an even device of the drawn workload: pre-biased, its ions frozen
    dev = build_device(setup_from_texts(drawn_texts(k, np.random.default_rng([SEED_ION_STACKS, k]),
                                                    60)))
    assert dev.pre_cond and dev.fix_ions
    with pytest.raises(NotImplementedError, match="frozen"):
        imp.solve_impedance([dev], [1e3], voltage=0.5)


def contact_texts(case, NP=None, mu=None):
    """The input texts of a golden case (tests/golden/inputs), with `NP` points and the ions'
    mobility `mu` (m²/Vs) where given."""
    import re
    from tests.test_transient_oracle import INPUTS
    texts = {f.name: f.read_text() for f in (INPUTS / case).iterdir() if f.suffix == ".txt"}
    for name in texts:
        if name.startswith("L") and mu is not None:
            texts[name] = re.sub(r"^(mu_anion|mu_cation)\s*=\s*[0-9.eE+-]+",
                                 lambda m: f"{m.group(1)} = {mu}", texts[name], flags=re.M)
    if NP is not None:
        texts["simulation_setup.txt"] = re.sub(r"^NP\s*=\s*\d+", f"NP = {NP}",
                                               texts["simulation_setup.txt"], flags=re.M)
    return texts


@pytest.mark.parametrize("case", ["zimt_region_slow_light", "two_regions_light"])
def test_ion_regions_that_reach_a_contact(case):
    """Ion regions that reach a contact (a region of two layers at the left contact; two regions
    of each species, one at each contact): the contact's ions from its neighbour's
    (`_ion_full`: at the step's dti = 1 in each region's number, whose derivative in V_int
    through the contact's potential joins the border's right-hand side, Boltzmann's in the
    current at dti = 0). At 1e-7 Hz the steady slope (1e-5, the reference's bar with ions;
    measured 9e-10). Far above every relaxation the capacitance is not the geometric one: the
    contact's ions follow the potential at once (their neighbour's density through the potential
    step), so keeping each region's number moves its inner ions (6e-4 and 3e-4 below it here)."""
    dev = build_device(setup_from_texts(contact_texts(case)), grid="simss")
    assert dev.anion_mask[0] and dev.cation_mask[0]
    V0, dV = 0.5, 1e-5
    Y, _, _, ok = imp.solve_impedance([dev], [1e-7, 1e14], voltage=V0, tol=1e-12, max_iter=200)
    st = dd.solve_states(dd.prepare([dev]), [V0 - dV, V0 + dV], tol=1e-12, max_iter=200)
    slope = (st["J"][0, 1] - st["J"][0, 0]) / (2 * dV)
    assert ok.all()
    assert Y[0, 0].real == pytest.approx(slope, rel=1e-5)
    x, eps = np.asarray(dev.x), np.asarray(dev.eps)
    geometric = 1.0 / np.sum(np.diff(x) * 0.5 * (1 / eps[:-1] + 1 / eps[1:]))
    assert 1e-4 < 1 - Y[0, 1].imag / (2 * np.pi * 1e14) / geometric < 1e-3


def test_ion_regions_at_both_contacts_against_the_transient():
    """With `dt`, two regions of each species reaching both contacts, the ions at 1e-9 m²/Vs,
    against the oracle transient's response to a 10 µV sine at 100 kHz. jaxdd's `_admittance`
    takes the contact's ions before the step as a density of 1 (`_full`'s masked contact), so its
    linearised current keeps a term of the contact's density that the transient, whose contact
    before a step is the last step's, has not: 6.5e-6 between the two (the bar 1e-5); with the
    contact's own density before the step they agree to 4.5e-9. This build follows jaxdd."""
    dev = build_device(setup_from_texts(contact_texts("two_regions_light", 60, "1e-9")),
                       grid="simss")
    assert dev.anion_mask[0] and dev.anion_mask[-1]
    Yt, dt = _sine_response(dev, 0.5, 1e5, amp=1e-5)
    Yd = imp.solve_impedance([dev], [1e5], voltage=0.5, tol=1e-12, max_iter=200, dt=dt)[0][0, 0]
    assert 1e-6 < abs(Yd / Yt - 1) < 1e-5


def _sine_response(dev, V0, f, amp=1e-4, per_period=40, periods=20, fitted=4):
    """The oracle transient's admittance at `f`: `J = J₀ + amp·(Re Y·sin + Im Y·cos)` fitted over
    the last periods of a sine of `amp` on `V0` at constant steps (jaxdd
    tests/test_impedance.py:47-63's protocol)."""
    from oracle import transient
    dt = 1.0 / (f * per_period)
    k = np.arange(1, per_period * periods + 1)
    t = np.concatenate([[0.0], k * dt])
    V = np.concatenate([[V0], V0 + amp * np.sin(2 * np.pi * f * k * dt)])
    o = transient.solve_transient(dd.prepare([dev]), t, V, np.full(len(t), float(dev.G_frac)),
                                  tol=1e-12, max_iter=60)
    assert o["converged"].all()
    m = k > per_period * (periods - fitted)
    ph = 2 * np.pi * f * k[m] * dt
    X = np.stack([np.ones(m.sum()), np.sin(ph), np.cos(ph)], -1)
    c = np.linalg.lstsq(X, o["J"][0, 1:][m], rcond=None)[0]
    return (c[1] + 1j * c[2]) / amp, dt


def test_with_ions_the_dt_form_is_the_transients_response():
    """With `dt` the admittance is what the transient (itself pinned on ZimT) sees through implicit
    Euler at steps of `dt`: its response to a 0.1 mV sine (40 steps a period, 20 periods) on a
    mobile-ion stack whose ions (μ 1e-9 m²/Vs) follow at 1 kHz, the traps' occupations' dynamics
    included: to 1e-6 (measured 1.3e-8; the reference's bar with ions). The continuous response
    differs from it by implicit Euler's error (4 % here)."""
    k = 1
    texts = drawn_texts(k, np.random.default_rng([SEED_ION_STACKS, k]), 60)
    texts["L2.txt"] = "\n".join(
        f"{line.split('=')[0].strip()} = 1e-9"
        if line.split("=")[0].strip() in ("mu_anion", "mu_cation") else line
        for line in texts["L2.txt"].splitlines()) + "\n"
    dev = build_device(setup_from_texts(texts))
    Yt, dt = _sine_response(dev, 0.8, 1e3)
    Yd = imp.solve_impedance([dev], [1e3], voltage=0.8, tol=1e-12, max_iter=200, dt=dt)[0][0, 0]
    Yc = imp.solve_impedance([dev], [1e3], voltage=0.8, tol=1e-12, max_iter=200)[0][0, 0]
    assert abs(Yd / Yt - 1) < 1e-6
    assert abs(Yc / Yt - 1) > 1e-2


def test_with_interface_traps_the_dt_form_is_the_transients_response():
    """Interface traps are each edge's occupation in time: with `dt` the admittance is the
    transient's response to a 10 µV sine on the p-i-n cell with interface traps (1e-7, the
    reference's bar; measured 6e-9 at 10 kHz), 8 % off the continuous response."""
    dev = _cell(NP=60, interface=True)
    Yt, dt = _sine_response(dev, 0.6, 1e4, amp=1e-5, periods=12)
    Yd = imp.solve_impedance([dev], [1e4], voltage=0.6, tol=1e-12, max_iter=200, dt=dt)[0][0, 0]
    Yc = imp.solve_impedance([dev], [1e4], voltage=0.6, tol=1e-12, max_iter=200)[0][0, 0]
    assert abs(Yd / Yt - 1) < 1e-7
    assert abs(Yc / Yt - 1) > 1e-2


def _differential(texts):
    """The same device with SIMsalabim's differential current (`currDiffInt = 1`)."""
    setup = texts["simulation_setup.txt"]
    assert "currDiffInt = 2" in setup
    return dict(texts, **{"simulation_setup.txt": setup.replace("currDiffInt = 2",
                                                                "currDiffInt = 1")})


def test_the_differential_current_low_frequency_is_the_steady_slope():
    """With `currDiffInt = 1` every interval carries its Scharfetter–Gummel flux (jaxdd
    batch.py:366-369); its tangent (complex step through the flux, the Bernoulli function
    continued to complex arguments) gives the steady slope at 1e-7 Hz. dV 1e-4: the differential
    current cancels large fluxes, so a smaller difference is round-off (4e-6 at dV 1e-6)."""
    dev = build_device(setup_from_texts(_differential(pin_texts(60))))
    assert dev.curr_diff
    V0, dV = 0.6, 1e-4
    for name in ("exact", "simss"):
        Y, _, _, ok = imp.solve_impedance([dev], [1e-7], voltage=V0, tol=1e-12, max_iter=200,
                                          bernoulli_name=name)
        st = dd.solve_states(dd.prepare([dev]), [V0 - dV, V0 + dV], tol=1e-13, max_iter=200,
                             bernoulli_name=name)
        slope = (st["J"][0, 1] - st["J"][0, 0]) / (2 * dV)
        assert ok.all()
        assert Y[0, 0].real == pytest.approx(slope, rel=1e-6)


@pytest.mark.parametrize("case", ["ions", "interface"])
def test_the_differential_current_dt_form_is_the_transients_response(case):
    """The differential current's admittance with `dt` against the oracle transient's response to
    a small sine (its current the same fluxes, from its own solve): with mobile ions following at
    1 kHz (their own fluxes too, jaxdd batch.py:471-479) to 1e-6, with interface traps to 1e-7
    (measured 1.4e-8 and 6e-9)."""
    if case == "ions":
        k = 1
        texts = drawn_texts(k, np.random.default_rng([SEED_ION_STACKS, k]), 60)
        texts["L2.txt"] = "\n".join(
            f"{line.split('=')[0].strip()} = 1e-9"
            if line.split("=")[0].strip() in ("mu_anion", "mu_cation") else line
            for line in texts["L2.txt"].splitlines()) + "\n"
        V0, f, amp, periods, bar = 0.8, 1e3, 1e-4, 20, 1e-6
    else:
        texts = pin_texts(60)
        for name in ("L1.txt", "L2.txt"):
            texts[name] = texts[name].replace("N_t_int = 0", "N_t_int = 1e15")
        V0, f, amp, periods, bar = 0.6, 1e4, 1e-5, 12, 1e-7
    dev = build_device(setup_from_texts(_differential(texts)))
    Yt, dt = _sine_response(dev, V0, f, amp=amp, periods=periods)
    Yd = imp.solve_impedance([dev], [f], voltage=V0, tol=1e-12, max_iter=200, dt=dt)[0][0, 0]
    assert abs(Yd / Yt - 1) < bar


def two_region_texts(NP=100, mu="1e-12"):
    """A five-layer stack with two ion regions of each species inside it: HTL 20 nm / absorber
    200 nm (anions and cations 1e23 m^-3) / spacer 20 nm without ions / absorber 250 nm (anions
    3e22, cations 5e22 m^-3) / ETL 30 nm, the ions' mobility `mu` (m²/Vs)."""
    from jaxdd_b200.workloads import _layer, _setup
    setup = _setup(NP).replace("l3 = L3.txt\n", "l3 = L3.txt\nl4 = L4.txt\nl5 = L5.txt\n")
    absorber = dict(eps_r="24", E_c="4.0", E_v="5.6", mu_n="1e-4", mu_p="1e-4",
                    N_t_bulk="1e20", E_t_bulk="4.8", k_direct="1e-17", G_ehp="2.5e27",
                    layerGen="1", mu_anion=mu, mu_cation=mu, ionsMayEnter="1")
    return {"simulation_setup.txt": setup,
            "L1.txt": _layer(L="20e-9", eps_r="3.5", E_c="2.6", E_v="5.6", mu_n="1e-6",
                             mu_p="1e-6", N_A="1e22"),
            "L2.txt": _layer(L="200e-9", N_anion="1e23", N_cation="1e23", **absorber),
            "L3.txt": _layer(L="20e-9", eps_r="24", E_c="4.0", E_v="5.6", mu_n="1e-4",
                             mu_p="1e-4"),
            "L4.txt": _layer(L="250e-9", N_anion="3e22", N_cation="5e22", **absorber),
            "L5.txt": _layer(L="30e-9", eps_r="10", E_c="4.0", E_v="7.2", mu_n="1e-5",
                             mu_p="1e-5", N_D="1e22")}


def test_two_ion_regions_of_each_species():
    """Several ion regions of a species (jaxdd's `_admittance` with a slot per region, its
    border keeping each region's number): at 1e-7 Hz the steady slope with the ions moving
    (1e-5, the reference's bar with ions; measured 1.5e-9), far above every relaxation the
    geometric capacitance, and with `dt` the oracle transient's response to a 0.1 mV sine at
    1 kHz, the ions at 1e-9 m²/Vs (1e-6; measured 3.5e-9)."""
    dev = build_device(setup_from_texts(two_region_texts()))
    b = dd.prepare([dev])
    assert b["ion"]["a_slots"].shape[1] == 2 and b["ion"]["c_slots"].shape[1] == 2
    assert not (dev.anion_mask[0] or dev.anion_mask[-1])
    V0, dV = 0.8, 1e-5
    Y, _, _, ok = imp.solve_impedance([dev], [1e-7, 1e14], voltage=V0, tol=1e-12, max_iter=200)
    st = dd.solve_states(b, [V0 - dV, V0 + dV], tol=1e-12, max_iter=200)
    slope = (st["J"][0, 1] - st["J"][0, 0]) / (2 * dV)
    assert ok.all()
    assert Y[0, 0].real == pytest.approx(slope, rel=1e-5)
    x, eps = np.asarray(dev.x), np.asarray(dev.eps)
    geometric = 1.0 / np.sum(np.diff(x) * 0.5 * (1 / eps[:-1] + 1 / eps[1:]))
    assert Y[0, 1].imag / (2 * np.pi * 1e14) == pytest.approx(geometric, rel=1e-4)
    dev = build_device(setup_from_texts(two_region_texts(60, "1e-9")))
    Yt, dt = _sine_response(dev, 0.8, 1e3)
    Yd = imp.solve_impedance([dev], [1e3], voltage=0.8, tol=1e-12, max_iter=200, dt=dt)[0][0, 0]
    assert abs(Yd / Yt - 1) < 1e-6
