"""The transient on the GPU (`dd_transient` through `jaxdd_b200.solve_transient`) against the
oracle (`oracle.transient`) on the same devices and steps, and against ZimT 5.36's own `Jext`
(the reference's tests/data) at the reference's tolerances: electrons and holes, the bulk traps
in time, mobile ions over 2 x 50 ms and 2 x 5 s, ion regions that reach a contact, the internal
voltage an unknown (the open circuit's photovoltage, a series resistance); a state carried
across a split (`profiles`, `initial`); the transient workload (drawn devices with mobile
ions, a step to 0.9 V, log-spaced steps) on fewer steps; ZimT's failure modes; at the transient workload's
2000 steps the properties that hold at any size (every step converged and kept, each region's
ions kept to their total, the current finite); and the integrated current's forward-mode
gradient in the ion density and mobility against differences of whole transients."""

import numpy as np
import pytest

from jaxdd_b200.batch import prepare
from jaxdd_b200.device import build_device
from jaxdd_b200.simss_input import TVG
from jaxdd_b200.transient import solve_transient
from jaxdd_b200.workloads import drawn_device, transient_steps
from oracle import dd, transient
from tests.test_transient_oracle import ZIMT, zimt_case, zimt_transient

pytestmark = pytest.mark.gpu


def _number(dens, mask, d):
    """A region's ions per area, trapezoidal over its intervals (`_ion_number`)."""
    pair = mask[1:] & mask[:-1]
    return np.sum(0.5 * (dens[1:] + dens[:-1]) * pair * d.h[:-1] * d.L)


@pytest.mark.parametrize("case", sorted(ZIMT))
def test_zimt_transients_match_the_oracle_and_zimt(case):
    setup, tvg, ref = zimt_case(case)
    dev = build_device(setup, grid="simss")
    r = solve_transient(prepare([dev]), tvg, bernoulli_name="simss", zimt_current=True)
    o = zimt_transient(dd.prepare([dev]), tvg)
    assert r.converged.all() and r.accepted.all() and r.stop[0] == 0
    scale = np.max(np.abs(ref["Jext"]))
    # the GPU against the oracle: the same algorithm, to Newton's tolerance
    assert np.max(np.abs(r.J_ext[0] - o["J_ext"][0])) < 1e-10 * scale
    # against ZimT, as the reference's own tests (test_solver.py:544-581)
    assert np.max(np.abs(r.J_ext[0] - ref["Jext"])) < ZIMT[case] * scale
    assert np.mean(r.iterations[0] == o["iterations"][0]) > 0.95


def test_zimt_transients_in_one_batch_each_with_its_own_steps():
    """jaxdd test_solver.py:719-737 on the GPU: ZimT's transients of 241 steps as one batch, each
    device with its own steps (the integral current beside the differential one, bulk traps,
    charged interface traps, mobile ions): each within its bar of ZimT's `Jext`."""
    cases = sorted(c for c in ZIMT if c != "zimt_steady_light")
    runs = [zimt_case(c) for c in cases]
    batch = prepare([build_device(setup, grid="simss") for setup, _, _ in runs])
    r = solve_transient(batch, [tvg for _, tvg, _ in runs], bernoulli_name="simss",
                        zimt_current=True)
    assert r.converged.all() and r.accepted.all()
    for k, (case, (_, _, ref)) in enumerate(zip(cases, runs)):
        scale = np.max(np.abs(ref["Jext"]))
        assert np.max(np.abs(r.J_ext[k] - ref["Jext"])) < ZIMT[case] * scale, case


def test_two_ion_regions_per_species_reaching_the_contacts():
    """Anions and cations in both transport layers, every region reaching a contact (its density
    there from its neighbour's), through a sweep to 0.9 V and back: the GPU against the oracle
    with every region's ion current and with ZimT's last region's (1e-9 of the scale; measured
    1.2e-10), and in the latter against ZimT's `Jext` to 1e-8 (`zimt_ion_currents`,
    test_solver.py:618-637); the final state's ions each region's total."""
    setup, tvg, ref = zimt_case("zimt_regions2_light")
    dev = build_device(setup, grid="simss")
    scale = np.max(np.abs(ref["Jext"]))
    for last in (False, True):
        r = solve_transient(prepare([dev]), tvg, bernoulli_name="simss", zimt_current=True,
                            zimt_ion_currents=last)
        o = transient.solve_transient(dd.prepare([dev]), tvg.t, tvg.Vext, tvg.G_frac, tvg.track,
                                      tvg.failure_mode, bernoulli_name="simss",
                                      zimt_current=True, zimt_ion_currents=last)
        assert r.converged.all() and o["converged"].all()
        assert np.max(np.abs(r.J_ext[0] - o["J_ext"][0])) < 1e-9 * scale, last
        if last:
            assert np.max(np.abs(r.J_ext[0] - ref["Jext"])) < 1e-8 * scale
    ion = dd.prepare([dev])["ion"]
    for name, slots, totals in (("anion", ion["a_slots"][0], ion["a_totals"][0]),
                                ("cation", ion["c_slots"][0], ion["c_totals"][0])):
        dens = getattr(r.final, name)[0]
        for mask, total in zip(slots, totals):
            m = mask > 0
            assert m[0] or m[-1]
            assert abs(_number(np.where(m, dens, 0.0), m, dev) / total - 1) < 1e-9, name


def test_the_photovoltage_at_the_open_circuit():
    """The internal voltage an unknown of each step (`vint`, the open circuit): ZimT 5.36's
    photovoltage through a light pulse of 1 µs and 1 ms after to 1e-10 V, the current 0 to
    1e-10 of the photocurrent (test_solver.py:740-752), the oracle's voltage to 1e-12 V."""
    from tests.test_transient_oracle import zimt_vint
    setup, tvg, ref = zimt_case("zimt_tpv_light")
    dev = build_device(setup, grid="simss")
    r = solve_transient(prepare([dev]), tvg, bernoulli_name="simss", zimt_current=True)
    o = zimt_vint(dd.prepare([dev]), tvg)
    assert r.converged.all() and r.accepted.all()
    assert np.max(np.abs(r.V_int[0] - ref["Vint"])) < 1e-10
    assert np.max(np.abs(r.V_int[0] - o["V_int"][0])) < 1e-12
    assert np.max(np.abs(r.J_ext)) < 1e-10 * np.max(ref["JphotoL2"])
    np.testing.assert_array_equal(r.V_ext, r.V_int)


def test_a_series_resistance_beside_given_voltages_and_ions_in_a_batch():
    """jaxdd test_solver.py:770-780 and 862-875 on the GPU: the series resistance's sweep (Vint
    the unknown whose Vint + Jext R_series is Vext) beside a device with the voltage given (its
    row Vint = Vext) and one with mobile ions (5x5 blocks with the voltage's border), each
    device its own steps: ZimT's Jext to 1e-9 (1e-7 with the ions) of its scale, Vint to 1e-9 V;
    the oracle's to 1e-10 of the scale."""
    from tests.test_transient_oracle import zimt_vint
    names = ("zimt_rseries_sweep_light", "zimt_photo_light", "zimt_ions_fast_light")
    cases = [zimt_case(c) for c in names]
    devs = [build_device(setup, grid="simss") for setup, _, _ in cases]
    r = solve_transient(prepare(devs), [tvg for _, tvg, _ in cases], bernoulli_name="simss",
                        zimt_current=True)
    assert r.converged.all()
    for k, ((_, tvg, ref), tol) in enumerate(zip(cases, (1e-9, 1e-9, 1e-7))):
        scale = np.max(np.abs(ref["Jext"]))
        assert np.max(np.abs(r.J_ext[k] - ref["Jext"])) < tol * scale, names[k]
        assert np.max(np.abs(r.V_ext[k] - tvg.Vext)) < 1e-9, names[k]
    assert np.max(np.abs(r.V_int[0] - cases[0][2]["Vint"])) < 1e-9
    assert np.max(np.abs(r.V_int[1:] - np.stack([t.Vext for _, t, _ in cases[1:]]))) < 1e-12
    o = zimt_vint(dd.prepare(devs[:1]), cases[0][1])
    scale = np.max(np.abs(o["J_ext"][0]))
    assert np.max(np.abs(r.J_ext[0] - o["J_ext"][0])) < 1e-10 * scale


@pytest.mark.parametrize("case", ["zimt_track_tpv_light", "zimt_track_tpv3_light"])
def test_the_automatic_stop(case):
    """ZimT's automatic stop (Track 2 and 3, five equal states in a row) on the photovoltage
    after a pulse: stopped where the oracle stops and as ZimT 5.36 within one step, the kept
    steps' Vint to 1e-10 V of ZimT's (test_solver.py:782-799)."""
    from jaxdd_b200.transient import STOP_STATIC
    from tests.test_transient_oracle import zimt_track
    setup, tvg, ref = zimt_case(case)
    dev = build_device(setup, grid="simss")
    r = solve_transient(prepare([dev]), tvg, bernoulli_name="simss", zimt_current=True)
    o = zimt_track(dd.prepare([dev]), tvg)
    rows = int(r.accepted[0].sum())
    assert r.stop[0] == STOP_STATIC and abs(rows - len(ref)) <= 1 and rows < len(tvg.t)
    np.testing.assert_array_equal(r.accepted, o["accepted"])
    assert r.accepted[0, :rows].all() and r.converged[0, :rows].all()
    rows = min(rows, len(ref))
    assert np.max(np.abs(r.V_int[0, :rows] - ref["Vint"][:rows])) < 1e-10


@pytest.mark.parametrize("case", ["zimt_photo_light", "zimt_sweep_diff_light",
                                  "zimt_iface_sweep_light", "zimt_ions_slow_light",
                                  "zimt_rseries_sweep_light", "zimt_sweep_spv_light"])
def test_zimts_columns(case):
    """ZimT's tJFile columns (`TransientResult.columns`, `tj_columns`) on the GPU against ZimT
    5.36's own at the reference's tolerances (test_solver.py:517-541) and against the oracle's
    (`transient.columns`): the currents to 1e-9 of the scale, the voltages to 1e-9 V; errJ
    (the rms of each interval's current about the mean, which the densities below the floor
    move: 2.7e-6 of the scale seen after the light switches) and the QFLS at the reference's
    bars against ZimT."""
    from jaxdd_b200.transient import tj_columns
    from tests.test_transient_oracle import COLUMN_CASES, check_columns, tj_named
    setup, tvg, ref = zimt_case(case)
    dev = build_device(setup, grid="simss")
    r = solve_transient(prepare([dev]), tvg, bernoulli_name="simss", zimt_current=True)
    assert r.converged.all()
    nl = len(dev.i0)
    qfls, steady = COLUMN_CASES[case]
    check_columns(r.columns, 0, nl, ref, qfls, steady)
    o = transient.solve_transient(dd.prepare([dev]), tvg.t, tvg.Vext, tvg.G_frac, tvg.track,
                                  tvg.failure_mode, bernoulli_name="simss", zimt_current=True,
                                  oc=tvg.oc, layers=[(dev.i0, dev.i1)])
    mine, theirs = tj_named(r.columns, 0, nl, True), tj_named(o["columns"], 0, nl, True)
    scale = max(np.max(np.abs(ref["Jext"])), np.max(ref["JphotoL2"]))
    rows = np.ones(len(ref), bool) if steady else ref["t"] > 0
    for name, v in mine.items():
        err = np.abs(v - theirs[name])
        if name.startswith("QFLS"):
            assert np.max(err[rows]) < qfls, name
        elif name == "errJ":
            assert np.max(err) < 1e-5 * scale, name
        else:
            assert np.max(err) < (1e-9 if name.startswith("V") else 1e-9 * scale), name
    named = tj_columns(r, 0, spv="VL1" in ref.dtype.names)
    assert set(named) | {"t", "G_frac"} == set(ref.dtype.names)


def test_the_automatic_stop_by_convvar():
    """ZimT's automatic stop comparing states by their densities or currents (convVar 1-4) on
    the photo transient with Track 3 on every step, tolDens 1e-4 and tolCurr 1e-9 A/m² (errJ
    decides): stopped where the oracle stops, within one step (errJ's last digits, moved by the
    densities below the floor, decide a comparison at its threshold)."""
    from tests.test_transient_oracle import loose_tvg, zimt_track_loose
    for cv in (1, 2, 3, 4):
        setup, tvg = loose_tvg(cv)
        r = solve_transient(prepare([build_device(setup, grid="simss")]), tvg,
                            bernoulli_name="simss", zimt_current=True, columns=False)
        o = zimt_track_loose(cv)
        assert r.stop[0] == o["stop"][0] == 1, cv
        assert abs(int(r.accepted[0].sum()) - int(o["accepted"][0].sum())) <= 1, cv


def test_ion_stacks_transient_matches_the_oracle():
    devs = [drawn_device(k) for k in (1, 3, 5)]
    tvg = transient_steps(40)
    r = solve_transient(prepare(devs), tvg)
    o = transient.solve_transient(dd.prepare(devs), tvg.t, tvg.Vext, tvg.G_frac, tvg.track,
                                  tvg.failure_mode)
    assert r.converged.all() and o["converged"].all()
    np.testing.assert_array_equal(r.accepted, o["accepted"])
    for k in range(len(devs)):
        scale = np.max(np.abs(o["J_ext"][k]))
        assert np.max(np.abs(r.J_ext[k] - o["J_ext"][k])) < 1e-9 * scale, k
    # the final state: each region's ions their total
    for k, d in enumerate(devs):
        assert abs(_number(r.final.anion[k], d.anion_mask, d) / d.anion_total - 1) < 1e-9
        assert abs(_number(r.final.cation[k], d.cation_mask, d) / d.cation_total - 1) < 1e-9


def test_failure_modes_as_the_oracle():
    """Newton held to 3 iterations so that steps fail: failureMode 0 stops at the first failed
    step, 1 keeps every step, 2 skips the failed ones (and the next step's dt is from the last
    kept one)."""
    setup, tvg, _ = zimt_case("zimt_photo_light")
    dev = build_device(setup, grid="simss")
    S = 30
    for fm in (0, 1, 2):
        steps = TVG.steps(tvg.t[:S], tvg.Vext[:S], tvg.G_frac[:S], 0, failure_mode=fm)
        r = solve_transient(prepare([dev]), steps, max_iter=3, bernoulli_name="simss",
                            zimt_current=True)
        o = transient.solve_transient(dd.prepare([dev]), steps.t, steps.Vext, steps.G_frac,
                                      steps.track, fm, max_iter=3, bernoulli_name="simss",
                                      zimt_current=True)
        assert not o["converged"].all()
        np.testing.assert_array_equal(r.converged, o["converged"])
        np.testing.assert_array_equal(r.accepted, o["accepted"])
        np.testing.assert_array_equal(r.stop, o["stop"])
        kept = o["accepted"][0]
        scale = np.max(np.abs(o["J_ext"][0][kept]))
        assert np.max(np.abs(r.J_ext[0][kept] - o["J_ext"][0][kept])) < 1e-8 * scale


def test_ion_stacks_full_steps_hold_their_invariants():
    devs = [drawn_device(k) for k in range(1, 129, 2)]
    r = solve_transient(prepare(devs), transient_steps(2000))
    assert r.converged.mean() > 0.999 and r.accepted.all()
    assert np.all(np.isfinite(r.J_ext))
    for k, d in enumerate(devs):
        assert abs(_number(r.final.anion[k], d.anion_mask, d) / d.anion_total - 1) < 1e-8


def _scaled_device(k, lnN=0.0, lnmu=0.0, NP=120, R_series=0.0):
    """The mobile-ion stack `k` with its ion density and mobility scaled by e^lnN and e^lnmu
    (and a series resistance, Ohm m², where given)."""
    from jaxdd_b200.simss_input import setup_from_texts
    from jaxdd_b200.workloads import SEED_ION_STACKS, drawn_texts
    idx = 2 * k + 1
    t = drawn_texts(idx, np.random.default_rng([SEED_ION_STACKS, idx]), NP)
    if R_series:
        t["simulation_setup.txt"] = t["simulation_setup.txt"].replace(
            "R_series = 0\n", f"R_series = {R_series!r}\n")
    lines = []
    for line in t["L2.txt"].splitlines():
        key, _, val = (part.strip() for part in line.partition("="))
        if key in ("N_anion", "N_cation"):
            line = f"{key} = {float(val) * float(np.exp(lnN))!r}"
        elif key in ("mu_anion", "mu_cation"):
            line = f"{key} = {float(val) * float(np.exp(lnmu))!r}"
        lines.append(line)
    t["L2.txt"] = "\n".join(lines) + "\n"
    return build_device(setup_from_texts(t))


def _charge(r, t):
    """The integrated current of each device: J over each kept step's dt."""
    out = []
    for k in range(r.J.shape[0]):
        prev, q = 0.0, 0.0
        for s in range(t.shape[1]):
            if r.accepted[k, s]:
                if t[k, s] > 0:
                    q += r.J[k, s] * (t[k, s] - prev)
                prev = t[k, s]
        out.append(q)
    return np.array(out)


def test_charge_gradients_match_differences_of_whole_transients():
    """The forward-mode tangents of `dd_transient` (the integrated current's derivatives in
    ln N_ion and ln mu_ion) against central differences of whole transients of the rebuilt
    devices, Richardson-extrapolated (steps 1e-3 and 2e-3): on the GPU's own transient and, for
    one device, the oracle's."""
    from jaxdd_b200.transient import charge_gradients
    ks = (0, 1, 2)
    tvg = transient_steps(40)
    base = [_scaled_device(k) for k in ks]
    g = charge_gradients(prepare(base), tvg)
    assert g.result.converged.all()
    np.testing.assert_allclose(g.Q, _charge(g.result, g.result.t), rtol=1e-12)

    def fd(which, solve):
        def q(h):
            devs = [_scaled_device(k, **{which: h}) for k in ks]
            return solve(devs)
        d1 = (q(1e-3) - q(-1e-3)) / 2e-3
        d2 = (q(2e-3) - q(-2e-3)) / 4e-3
        return (4 * d1 - d2) / 3

    def gpu(devs):
        r = solve_transient(prepare(devs), tvg)
        return _charge(r, r.t)

    # measured: 1e-9 of each derivative; the differences' own accuracy is near 1e-8
    for which, mine in (("lnN", g.dQ_dlnN_ion), ("lnmu", g.dQ_dlnmu_ion)):
        ref = fd(which, gpu)
        assert np.all(np.abs(mine - ref) < 1e-6 * np.abs(ref) + 1e-9 * np.abs(g.Q)), \
            (which, mine, ref)

    def oracle(devs):
        o = transient.solve_transient(dd.prepare(devs[:1]), tvg.t, tvg.Vext, tvg.G_frac)
        t = np.broadcast_to(tvg.t, o["J"].shape)
        return _charge(type("R", (), {"J": o["J"], "accepted": o["accepted"]})(), t)

    for which, mine in (("lnN", g.dQ_dlnN_ion), ("lnmu", g.dQ_dlnmu_ion)):
        ref = fd(which, oracle)
        assert abs(mine[0] - ref[0]) < 1e-6 * abs(ref[0]) + 1e-9 * abs(g.Q[0]), (which, mine[0],
                                                                                 ref)


def _scaled_contact_device(case, lnN=0.0, lnmu=0.0, NP=100):
    """A golden case whose ion regions reach the contacts, its ions' densities and mobilities
    scaled by e^lnN and e^lnmu, at NP points."""
    import re
    from jaxdd_b200.simss_input import setup_from_texts
    from tests.test_impedance_oracle import contact_texts
    texts = contact_texts(case, NP)
    for name, text in texts.items():
        if not name.startswith("L"):
            continue
        for key, f in (("N_anion", lnN), ("N_cation", lnN), ("mu_anion", lnmu),
                       ("mu_cation", lnmu)):
            text = re.sub(rf"^{key}\s*=\s*([0-9.eE+-]+)",
                          lambda m: f"{key} = {float(m.group(1)) * float(np.exp(f))!r}", text,
                          flags=re.M)
        texts[name] = text
    return build_device(setup_from_texts(texts), grid="simss")


@pytest.mark.parametrize("case", ["zimt_region_slow_light", "two_regions_light"])
def test_charge_gradients_with_ion_regions_at_the_contacts(case):
    """The tangents where ion regions reach the contacts (the contacts' ions from their
    neighbours in each region's number and in the current, along each tangent too): against
    central differences of whole GPU transients of the rebuilt device, Richardson-extrapolated
    (1e-6), and of the oracle's transients (1e-5: the two transients' own round-off apart moves
    the differences; measured 1.6e-6 in ln mu)."""
    from jaxdd_b200.transient import charge_gradients
    tvg = transient_steps(40)
    base = [_scaled_contact_device(case)]
    assert base[0].anion_mask[0]
    g = charge_gradients(prepare(base), tvg)
    assert g.result.converged.all()

    def fd(which, solve):
        def q(h):
            return solve([_scaled_contact_device(case, **{which: h})])
        d1 = (q(1e-3) - q(-1e-3)) / 2e-3
        d2 = (q(2e-3) - q(-2e-3)) / 4e-3
        return (4 * d1 - d2) / 3

    def gpu(devs):
        r = solve_transient(prepare(devs), tvg)
        return _charge(r, r.t)

    def oracle(devs):
        o = transient.solve_transient(dd.prepare(devs), tvg.t, tvg.Vext, tvg.G_frac)
        t = np.broadcast_to(tvg.t, o["J"].shape)
        return _charge(type("R", (), {"J": o["J"], "accepted": o["accepted"]})(), t)

    for which, mine in (("lnN", g.dQ_dlnN_ion), ("lnmu", g.dQ_dlnmu_ion)):
        for solve, bar in ((gpu, 1e-6), (oracle, 1e-5)):
            ref = fd(which, solve)
            assert np.all(np.abs(mine - ref) < bar * np.abs(ref) + 1e-9 * np.abs(g.Q)), \
                (which, solve.__name__, mine, ref)


@pytest.mark.parametrize("circuit", ["series", "open"])
def test_charge_gradients_with_the_internal_voltage_an_unknown(circuit):
    """The tangents with the internal voltage an unknown of every step (its own tangent from the
    tangent system's voltage row, the current's and the next step's through it): a series
    resistance of 1e-4 Ohm m² at 0.9 V, and the open circuit from the steady state at 0 V under
    light, against central differences of whole GPU transients and of the oracle's. At the open
    circuit the current is 0 at every step (the voltage's row), so are the charge and its
    derivatives: there the bar is 1e-9 of the current scale times the transient's length."""
    import dataclasses
    from jaxdd_b200.transient import charge_gradients
    tvg = transient_steps(40)
    rs = 1e-4 if circuit == "series" else 0.0
    if circuit == "open":
        tvg = dataclasses.replace(tvg, oc=tvg.t > 0)
    ks = (0, 1)
    base = [_scaled_device(k, R_series=rs) for k in ks]
    g = charge_gradients(prepare(base), tvg)
    assert g.result.converged.all()
    assert np.ptp(g.result.V_int[0, 1:]) > 1e-3  # the internal voltage moves

    def fd(which, solve):
        def q(h):
            return solve([_scaled_device(k, R_series=rs, **{which: h}) for k in ks])
        d1 = (q(1e-3) - q(-1e-3)) / 2e-3
        d2 = (q(2e-3) - q(-2e-3)) / 4e-3
        return (4 * d1 - d2) / 3

    def gpu(devs):
        r = solve_transient(prepare(devs), tvg)
        return _charge(r, r.t)

    def oracle(devs):
        o = transient.solve_transient(dd.prepare(devs[:1]), tvg.t, tvg.Vext, tvg.G_frac,
                                      oc=tvg.oc)
        t = np.broadcast_to(tvg.t, o["J"].shape)
        return _charge(type("R", (), {"J": o["J"], "accepted": o["accepted"]})(), t)

    floor = np.abs(g.Q) if circuit == "series" else prepare(base)["J_scale"] * tvg.t[-1]
    for which, mine in (("lnN", g.dQ_dlnN_ion), ("lnmu", g.dQ_dlnmu_ion)):
        ref = fd(which, gpu)
        assert np.all(np.abs(mine - ref) < 1e-6 * np.abs(ref) + 1e-9 * floor), (which, mine, ref)
        ref = fd(which, oracle)
        assert abs(mine[0] - ref[0]) < 1e-6 * abs(ref[0]) + 1e-9 * floor[0], (which, mine, ref)


def test_uneven_devices_and_their_own_steps_in_one_launch():
    """Devices of different grid sizes (`prepare(..., ragged=True)`) each with its own step list
    (the steps' per-lane layout) in one launch: each device's result is its transient alone."""
    devs = [drawn_device(k, NP=n) for k, n in ((1, 60), (3, 90), (5, 75))]
    tvgs = [transient_steps(30, V=v) for v in (0.9, 0.7, 1.0)]
    r = solve_transient(prepare(devs, ragged=True), tvgs)
    assert r.converged.all()
    for k, (d, tv) in enumerate(zip(devs, tvgs)):
        alone = solve_transient(prepare([d]), tv)
        np.testing.assert_array_equal(r.iterations[k], alone.iterations[0])
        scale = np.max(np.abs(alone.J[0]))
        assert np.max(np.abs(r.J[k] - alone.J[0])) < 1e-12 * scale
        np.testing.assert_allclose(r.final.V[k], alone.final.V[0], rtol=0, atol=1e-12)


def _part(tvg, part):
    """The steps `part` (a slice) of `tvg`."""
    import dataclasses
    return dataclasses.replace(tvg, **{k: getattr(tvg, k)[part]
                                       for k in ("t", "Vext", "oc", "G_frac", "track", "dti")})


def _split_case(case):
    """A device and its steps: two of ZimT's cases (mobile ions through a sweep and back; bulk
    traps with light on and off), and the p-i-n cell with interface traps through a sweep."""
    if case in ZIMT:
        setup, tvg, _ = zimt_case(case)
        return build_device(setup, grid="simss"), tvg, dict(bernoulli_name="simss",
                                                            zimt_current=True)
    from jaxdd_b200.simss_input import setup_from_texts
    from jaxdd_b200.workloads import pin_texts
    t = pin_texts(60)
    for name in ("L1.txt", "L2.txt"):
        t[name] = t[name].replace("N_t_int = 0", "N_t_int = 1e15")
    times = np.concatenate([[0.0], np.logspace(-9, -4, 50)])
    V = np.concatenate([[0.0], np.linspace(0.0, 0.9, 25), np.linspace(0.9, 0.0, 25)])
    return build_device(setup_from_texts(t)), TVG.steps(times, V), {}


@pytest.fixture(scope="module", params=["zimt_ions_fast_light", "zimt_traps_photo_light",
                                        "interface"])
def unsplit(request):
    dev, tvg, kw = _split_case(request.param)
    batch = prepare([dev])
    return request.param, dev, batch, tvg, kw, solve_transient(batch, tvg, profiles=True, **kw)


def test_a_transient_split_at_a_step_goes_on_as_the_unsplit_one(unsplit):
    """jaxdd tests/test_transient_state.py:41-70 on the GPU: split at its middle step and
    continued from the first half's last state (`final`) or from that step's state in the
    unsplit run's profiles (`state(k)`), a transient gives the unsplit one's currents to 1e-9
    of their scale, its densities and ions to 1e-6 and its potential to 1e-9 V; the last state
    kept is the last step's."""
    case, dev, batch, tvg, kw, full = unsplit
    assert full.converged.all() and full.accepted.all()
    k = len(tvg.t) // 2
    first = solve_transient(batch, _part(tvg, slice(0, k + 1)), **kw)
    rest = _part(tvg, slice(k + 1, None))
    scale = np.max(np.abs(full.J_ext))
    for start in (first.final, full.state(k)):
        r = solve_transient(batch, rest, initial=start, profiles=True, **kw)
        assert r.converged.all(), case
        np.testing.assert_allclose(r.J_ext[0], full.J_ext[0, k + 1:], rtol=0, atol=1e-9 * scale)
        for name in ("n", "p", "anion", "cation"):
            np.testing.assert_allclose(r.profiles[name][0], full.profiles[name][0, k + 1:],
                                       rtol=1e-6, err_msg=f"{case}: {name}")
        np.testing.assert_allclose(r.profiles["V"][0], full.profiles["V"][0, k + 1:], rtol=0,
                                   atol=1e-9)
        np.testing.assert_array_equal(r.t[0], tvg.t[k + 1:])
    last = full.state(-1)
    for name in ("V", "n", "p", "anion", "cation", "f_bulk", "f_interface", "V_int", "dti", "t"):
        np.testing.assert_allclose(getattr(full.final, name), getattr(last, name), rtol=1e-12,
                                   atol=1e-15, err_msg=name)
    # the traps carry their occupations across the split
    if case != "zimt_ions_fast_light":
        occ = "f_interface" if case == "interface" else "f_bulk"
        assert np.any(full.profiles[occ][0] != 0)
        r = solve_transient(batch, rest, initial=full.state(k), profiles=True, **kw)
        np.testing.assert_allclose(r.profiles[occ][0], full.profiles[occ][0, k + 1:],
                                   rtol=1e-6, atol=1e-12)


def test_the_profiles_ions_hold_each_species_total(unsplit):
    """At every step the profiles' ions (0 outside their regions) count each region's total,
    trapezoidal as the solver counts them, to 1e-9."""
    case, dev, _, _, _, full = unsplit
    for name, mask, total in (("anion", dev.anion_mask, dev.anion_total),
                              ("cation", dev.cation_mask, dev.cation_total)):
        dens = full.profiles[name][0]
        if mask is None or not total:
            assert not dens.any(), case
            continue
        m = np.asarray(mask, bool)
        assert np.all(dens[:, ~m] == 0), case
        for step in dens:
            assert abs(_number(step, m, dev) / total - 1) < 1e-9, case


def test_a_step_state_needs_the_profiles():
    setup, tvg, _ = zimt_case("zimt_photo_light")
    r = solve_transient(prepare([build_device(setup, grid="simss")]), _part(tvg, slice(0, 3)),
                        bernoulli_name="simss")
    with pytest.raises(ValueError, match="profiles=True"):
        r.state(1)
