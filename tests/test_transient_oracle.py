"""The transient oracle pinned on ZimT 5.36's own transients (the reference's tests/data, copied
to tests/golden/inputs): `Jext` through 241 steps to the reference's tolerances
(test_solver.py:544-581: 1e-9 of the scale for electrons and holes and for the traps, 1e-7 with
mobile ions), ZimT's Bernoulli function and sums (`zimt_current`): light on and off, a sweep to
1.2 V and back in 2 x 100 ns in the integral and the differential current, the absorber's traps,
charged interface traps through the sweep, mobile ions over 2 x 50 ms and 2 x 5 s, in a region
of two layers that reaches a contact (its density there from its neighbour's, nothing flowing
over the contact's interval), two regions per species with ZimT's last-region ion currents, and
steady states at t = 0 (test_solver.py:454-470, 618-637). Also: the tVG reader's checks,
the traps' step against its closed form and its derivatives, the ions' number kept in every step,
and the refusals of what is out of scope."""

import functools

import numpy as np
import pytest

from jaxdd_b200.device import build_device
from jaxdd_b200.simss_input import TVG, read_setup, read_tvg, setup_from_texts
from oracle import dd, transient

INPUTS = __import__("pathlib").Path(__file__).resolve().parent / "golden" / "inputs"

ZIMT = {"zimt_photo_light": 1e-9, "zimt_traps_photo_light": 1e-9,
        "zimt_ions_fast_light": 1e-7, "zimt_ions_slow_light": 1e-7,
        "zimt_sweep_light": 1e-9, "zimt_sweep_diff_light": 1e-9,
        "zimt_iface_sweep_light": 1e-9, "zimt_steady_light": 1e-9,
        "zimt_region_slow_light": 1e-7, "zimt_region_diff_light": 1e-7}


def zimt_case(case):
    setup = read_setup(INPUTS / case / "simulation_setup.txt")
    return setup, read_tvg(setup), np.genfromtxt(INPUTS / case / "tj.dat", names=True)


def zimt_transient(batch, tvg, steps=None):
    S = len(tvg.t) if steps is None else steps
    return transient.solve_transient(batch, tvg.t[:S], tvg.Vext[:S], tvg.G_frac[:S],
                                     tvg.track[:S], tvg.failure_mode, bernoulli_name="simss",
                                     zimt_current=True)


@functools.lru_cache(maxsize=None)
def zimt_columns_run(case):
    """ZimT's steps of `case` with its tJFile columns (`layers`: the device's layers), run once
    for both the `Jext` and the columns tests: the columns are one more pass over each step's
    solution, which leaves the steps themselves as they are."""
    setup, tvg, ref = zimt_case(case)
    dev = build_device(setup, grid="simss")
    r = transient.solve_transient(dd.prepare([dev]), tvg.t, tvg.Vext, tvg.G_frac, tvg.track,
                                  tvg.failure_mode, bernoulli_name="simss", zimt_current=True,
                                  oc=tvg.oc, layers=[(dev.i0, dev.i1)])
    return tvg, ref, dev, r


@pytest.mark.parametrize("case", sorted(ZIMT))
def test_the_oracle_reproduces_zimt(case):
    setup, tvg, ref = zimt_case(case)
    if case in COLUMN_CASES and not tvg.oc.any():
        r = zimt_columns_run(case)[3]
    else:
        r = zimt_transient(dd.prepare([build_device(setup, grid="simss")]), tvg)
    assert r["converged"].all() and r["accepted"].all() and r["stop"][0] == 0
    scale = np.max(np.abs(ref["Jext"]))
    assert np.max(np.abs(r["J_ext"][0] - ref["Jext"])) < ZIMT[case] * scale


def test_the_ions_keep_their_number_in_every_step():
    """Each region's rescaling is a slot of the bordered system: after every kept step the
    anions' and cations' numbers are their totals (to Newton's tolerance)."""
    setup, tvg, _ = zimt_case("zimt_ions_fast_light")
    b = dd.prepare([build_device(setup, grid="simss")])
    r = zimt_transient(b, tvg, steps=12)
    full = transient.full_of(b, r["y"], np.array([tvg.Vext[11]]))
    g, _, _ = transient.constraints(full, r["logs"], b["ion"])
    masks, totals = dd._masks(b["ion"])
    assert np.any(totals > 0)
    assert np.max(np.abs(g)) < 1e-9


def test_the_traps_step_is_the_closed_form_and_its_derivatives():
    rng = np.random.default_rng(7)
    Cn, Cp = 10 ** rng.uniform(-15, -13, 50), 10 ** rng.uniform(-15, -13, 50)
    nt0, pt0 = 10 ** rng.uniform(10, 16, 50), 10 ** rng.uniform(10, 16, 50)
    n, p = 10 ** rng.uniform(14, 22, 50), 10 ** rng.uniform(14, 22, 50)
    f_old = rng.uniform(0, 1, 50)
    # a steady state: both the steady occupation
    (mean, end, vac), _, _ = transient.trap_step(Cn, Cp, nt0, pt0, n, p, f_old, 0.0)
    a = Cn * (n + nt0) + Cp * (p + pt0)
    np.testing.assert_allclose(mean, (Cn * n + Cp * pt0) / a, rtol=1e-15)
    np.testing.assert_allclose(end, mean, rtol=0)
    np.testing.assert_allclose(vac, (Cn * nt0 + Cp * p) / a, rtol=1e-15)
    # over a step: f(t) = s + (f_old − s)·exp(−a t), its mean over the step
    dti = 10 ** rng.uniform(2, 9, 50)
    (mean, end, vac), d_n, d_p = transient.trap_step(Cn, Cp, nt0, pt0, n, p, f_old, dti)
    s = (Cn * n + Cp * pt0) / a
    np.testing.assert_allclose(end, s + (f_old - s) * np.exp(-a / dti), rtol=1e-12)
    x = a / dti
    # (1 − e^−x)/x as written loses digits at small x (the oracle takes expm1)
    np.testing.assert_allclose(mean, s + (f_old - s) * (1 - np.exp(-x)) / x, rtol=1e-9)
    np.testing.assert_allclose(mean + vac, 1.0, rtol=1e-12)
    # the derivatives are ~1e-8 of values near 1: a central difference at h = 1e-4 (round-off
    # 1e-12/h, truncation h²)
    for k, deriv in ((0, d_n), (1, d_p)):
        for j in range(3):
            h = 1e-4
            up = [n * (1 + h), p] if k == 0 else [n, p * (1 + h)]
            dn = [n * (1 - h), p] if k == 0 else [n, p * (1 - h)]
            fu = transient.trap_step(Cn, Cp, nt0, pt0, *up, f_old, dti)[0][j]
            fd = transient.trap_step(Cn, Cp, nt0, pt0, *dn, f_old, dti)[0][j]
            base = n if k == 0 else p
            fdiff = (fu - fd) / (2 * h * base)
            np.testing.assert_allclose(deriv[j], fdiff, rtol=1e-4,
                                       atol=1e-12 * np.max(abs(fdiff)))


def test_tvg_as_zimt_reads_it():
    _, tvg, ref = zimt_case("zimt_ions_fast_light")
    assert len(tvg.t) == 241 == len(ref) and tvg.t[0] == 0 and tvg.failure_mode == 0
    np.testing.assert_allclose(tvg.t, ref["t"], rtol=1e-9)
    assert tvg.dti[0] == 0 and np.allclose(tvg.dti[1:], 1 / np.diff(tvg.t))
    base = (INPUTS / "zimt_photo_light" / "simulation_setup.txt").read_text()
    files = {f.name: f.read_text() for f in (INPUTS / "zimt_photo_light").glob("*.txt")}

    def tvg_of(text):
        return read_tvg(setup_from_texts(dict(files, **{"simulation_setup.txt": base,
                                                          "tVG.txt": text})))

    assert len(tvg_of("t Vext G_frac Track\n0 0 1 0\n1e-6 0.5 1 1\n\n2 0 0 0\n").t) == 2
    assert tvg_of("t Vext G_frac Track\n0 oc 1 0\n").oc[0]
    for text, match in (("x y\n0 0 1 0\n", "header"),
                        ("t Vext G_frac Track\n1 0 1 0\n", "steady-state"),
                        ("t Vext G_frac Track\n0 0 1 0\n2 0 1 0\n1 0 1 0\n", "Time steps"),
                        ("t Vext G_frac Track\n0 0 1 0\n1 0 1 4\n", "offending"),
                        ("t Vext G_frac Track\n0 0 1 1\n1 0 1 2\n", "Track=1")):
        with pytest.raises(ValueError, match=match):
            tvg_of(text)
    steps = TVG.steps([0, 1e-9, 1e-8], [0, 0.9, 0.9])
    assert steps.dti[0] == 0 and np.isclose(steps.dti[2], 1 / 9e-9)
    with pytest.raises(ValueError):
        TVG.steps([1e-9, 1e-8], 0.9)


def test_two_ion_regions_per_species_as_zimt_counts_their_currents():
    """Anions and cations in both transport layers, each region reaching a contact, through a
    sweep to 0.9 V and back in 2 x 50 ms: with ZimT's last-region ion currents
    (`zimt_ion_currents`) ZimT's `Jext` to 1e-8 of its scale (test_solver.py:618-637); every
    region's current (the default) differs from it by more."""
    setup, tvg, ref = zimt_case("zimt_regions2_light")
    b = dd.prepare([build_device(setup, grid="simss")])
    scale = np.max(np.abs(ref["Jext"]))
    last = transient.solve_transient(b, tvg.t, tvg.Vext, tvg.G_frac, tvg.track, tvg.failure_mode,
                                     bernoulli_name="simss", zimt_current=True,
                                     zimt_ion_currents=True)
    assert last["converged"].all()
    assert np.max(np.abs(last["J_ext"][0] - ref["Jext"])) < 1e-8 * scale
    every = zimt_transient(b, tvg)
    assert np.max(np.abs(every["J_ext"][0] - ref["Jext"])) > 1e-7 * scale


def zimt_vint(batch, tvg):
    """ZimT's steps with the internal voltage an unknown where they are at the open circuit."""
    return transient.solve_transient(batch, tvg.t, tvg.Vext, tvg.G_frac, tvg.track,
                                     tvg.failure_mode, bernoulli_name="simss", zimt_current=True,
                                     oc=tvg.oc)


def test_the_photovoltage_at_the_open_circuit_reproduces_zimt():
    """The open circuit, the internal voltage an unknown of each step's Newton solve: ZimT
    5.36's photovoltage through a light pulse of 1 µs and 1 ms after, 151 steps, to 1e-10 V;
    the current 0 to 1e-10 of the photocurrent (test_solver.py:740-752)."""
    setup, tvg, ref = zimt_case("zimt_tpv_light")
    r = zimt_vint(dd.prepare([build_device(setup, grid="simss")]), tvg)
    assert r["converged"].all() and tvg.oc.all()
    assert np.max(np.abs(r["V_int"][0] - ref["Vint"])) < 1e-10
    assert np.max(np.abs(r["J_ext"])) < 1e-10 * np.max(ref["JphotoL2"])


def test_the_open_circuit_in_the_steady_state_is_simss_voc():
    """The open circuit at `t = 0` (the internal voltage the unknown of the steady state): SimSS
    5.36's V_oc, from its curve at 0.1 mV steps around it (the reference's thin_l1_voc_light, a
    cubic through its points), to 1e-10 V (test_solver.py:750-765)."""
    import dataclasses
    setup, tvg, _ = zimt_case("zimt_tpv_light")
    first = dataclasses.replace(tvg, **{k: getattr(tvg, k)[:1] for k in
                                        ("t", "Vext", "oc", "G_frac", "track", "dti")})
    r = transient.solve_transient(dd.prepare([build_device(setup, grid="simss")]), first.t,
                                  first.Vext, first.G_frac, first.track, first.failure_mode,
                                  bernoulli_name="simss", oc=first.oc)
    jv = np.genfromtxt(INPUTS / "thin_l1_voc_light" / "JV.dat", names=True)
    roots = np.roots(np.polyfit(jv["Vext"] - jv["Vext"].mean(), jv["Jext"], 3))
    roots = roots[np.abs(roots.imag) == 0].real + jv["Vext"].mean()
    voc = roots[(roots > jv["Vext"].min()) & (roots < jv["Vext"].max())]
    assert first.oc[0] and r["converged"].all() and voc.size == 1
    assert abs(r["V_int"][0, 0] - voc[0]) < 1e-10


def test_a_series_resistance_in_time_reproduces_zimt():
    """`R_series` with a shunt, `Vint` the unknown whose `Vint + Jext R_series` is the given
    `Vext`: ZimT 5.36's `Jext` through a sweep to 1.2 V and back in 2 x 100 ns to 1e-9 of its
    scale, `Vint` to 1e-9 V (test_solver.py:770-780)."""
    setup, tvg, ref = zimt_case("zimt_rseries_sweep_light")
    dev = build_device(setup, grid="simss")
    r = zimt_vint(dd.prepare([dev]), tvg)
    assert r["converged"].all()
    assert np.max(np.abs(r["J_ext"][0] - ref["Jext"])) < 1e-9 * np.max(np.abs(ref["Jext"]))
    assert np.max(np.abs(r["V_int"][0] - ref["Vint"])) < 1e-9
    assert np.max(np.abs(r["V_int"][0] + dev.R_series * r["J_ext"][0] - tvg.Vext)) < 1e-9


def zimt_track(batch, tvg):
    """ZimT's steps with the automatic stop's controls (`convVar`, `tolPois`, `tolDens`)."""
    return transient.solve_transient(batch, tvg.t, tvg.Vext, tvg.G_frac, tvg.track,
                                     tvg.failure_mode, bernoulli_name="simss", zimt_current=True,
                                     oc=tvg.oc, conv_var=tvg.conv_var, tol_pois=tvg.tol_pois,
                                     tol_dens=tvg.tol_dens, tol_curr=tvg.tol_curr)


def loose_tvg(cv):
    """ZimT's photo steps with Track 3 on every step, tolPois and tolDens 1e-4, tolCurr 1e-9 and
    convVar `cv`."""
    import dataclasses
    setup, tvg, _ = zimt_case("zimt_photo_light")
    return setup, dataclasses.replace(tvg, track=np.full(len(tvg.t), 3), conv_var=cv,
                                      tol_pois=1e-4, tol_dens=1e-4, tol_curr=1e-9)


def zimt_track_loose(cv):
    setup, tvg = loose_tvg(cv)
    return zimt_track(dd.prepare([build_device(setup, grid="simss")]), tvg)


@pytest.mark.parametrize("case", ["zimt_track_tpv_light", "zimt_track_tpv3_light"])
def test_the_automatic_stop_reproduces_zimt(case):
    """ZimT's automatic stop (five equal states in a row) on the photovoltage after a pulse:
    each step compared with the steady state before the pulse (Track 1 there, 2 after it), and
    each with the one before (Track 3); stopped as ZimT 5.36 within one step (its states
    compare within tolPois 1e-12 V, where ZimT's own error decides the step), Vint of the kept
    steps to 1e-10 V (test_solver.py:782-799)."""
    setup, tvg, ref = zimt_case(case)
    r = zimt_track(dd.prepare([build_device(setup, grid="simss")]), tvg)
    rows = int(r["accepted"][0].sum())
    assert r["stop"][0] == transient.STOP_STATIC and abs(rows - len(ref)) <= 1
    assert rows < len(tvg.t)
    assert r["accepted"][0, :rows].all() and r["converged"][0, :rows].all()
    rows = min(rows, len(ref))
    assert np.max(np.abs(r["V_int"][0, :rows] - ref["Vint"][:rows])) < 1e-10


def test_states_compare_as_zimt_compares_them():
    """`states_equal` as ZimT's `States_Are_Equal` (test_solver.py:802-824): never at another
    G_frac or with the potentials apart by tolPois; then by convVar the densities (1), the
    current within tolCurr or the smaller errJ (2), either (3) or both (4)."""
    base = {"V": np.zeros((1, 4)), "n": np.ones((1, 4)), "p": np.ones((1, 4)),
            "a": np.zeros((1, 4)), "c": np.zeros((1, 4))}
    G, one = np.ones(1), np.ones(1)
    dens_off = dict(base, n=np.ones((1, 4)) * (1 + 1e-5))

    def eq(B, cv, GB=G, JB=1.0, errA=0.0, errB=0.0):
        return bool(transient.states_equal(base, B, G, GB, 1e-6, 1e-6, cv, 1e-3, one,
                                           JB * one, errA * one, errB * one)[0])
    expect = {1: (False, True), 2: (True, False), 3: (True, True), 4: (False, False)}
    for cv, (with_dens_off, with_curr_off) in expect.items():
        assert eq(base, cv)
        assert eq(dens_off, cv) == with_dens_off, cv
        assert eq(base, cv, JB=1.1) == with_curr_off, cv
        assert not eq(base, cv, GB=np.full(1, 0.5))
        assert not eq(dict(base, V=np.full((1, 4), 1e-6)), cv)
    assert eq(dict(base, n=np.ones((1, 4)) * (1 + 1e-7)), 1)
    assert eq(base, 2, JB=1.1, errA=0.3, errB=0.2)  # within both states' errJ


def test_the_automatic_stop_compares_as_convvar_says():
    """ZimT's photo transient with Track 3 on every step, the densities compared loosely
    (tolDens 1e-4) and the currents strictly (tolCurr 1e-9 A/m², so errJ decides): comparing
    currents (convVar 2, or with the densities 4) stops later than comparing densities (1, or
    either 3). The four controls run as one batch of four copies of the device, one convVar
    each, over the first 100 of the 241 steps: every one of them stops inside those (the stops
    are at steps 61 and 70), which the stop flags confirm."""
    setup, tvg = loose_tvg(1)
    cvs = np.array([1, 2, 3, 4])
    S = 100
    r = transient.solve_transient(dd.prepare([build_device(setup, grid="simss")] * 4), tvg.t[:S],
                                  tvg.Vext[:S], tvg.G_frac[:S], tvg.track[:S], tvg.failure_mode,
                                  bernoulli_name="simss", zimt_current=True, oc=tvg.oc[:S],
                                  conv_var=cvs, tol_pois=tvg.tol_pois, tol_dens=tvg.tol_dens,
                                  tol_curr=tvg.tol_curr)
    assert np.all(r["stop"] == transient.STOP_STATIC), r["stop"]
    rows = dict(zip(cvs.tolist(), r["accepted"].sum(axis=1).astype(int).tolist()))
    assert rows[1] == rows[3] < rows[2] == rows[4] < S, rows


LAYER_COLUMNS = ("QFLS", "Jphoto", "Jdir", "JbulkElec", "JbulkHoles")
IFACE_COLUMNS = ("JintElec", "JintHoles")


def tj_named(c, k, nl, spv=False):
    """Device `k`'s columns (`columns` of a transient) as ZimT's tJFile names them."""
    out = {"errJ": c["errJ"][k]}
    for name in LAYER_COLUMNS:
        out.update({f"{name}L{j + 1}": c[name][k][:, j] for j in range(nl)})
    for name in IFACE_COLUMNS:
        out.update({f"{name}L{j + 1}L{j + 2}": c[name][k][:, j] for j in range(nl - 1)})
    for name in ("JminLeft", "JminRight", "JShunt", "Jnion", "Jpion", "JD"):
        out[name] = c[name][k]
    if spv:
        out.update({f"VL{j + 1}": c["VL"][k][:, j] for j in range(nl)})
    return out


def check_columns(c, k, nl, ref, qfls, steady=True):
    """Device `k`'s tJFile columns against ZimT's, as the reference checks them
    (test_solver.py:517-541): every column ZimT writes; the currents and recombination as
    currents to 1e-7 of the scale (the larger of Jext and the photocurrent), errJ to 1e-5,
    voltages to 1e-9 V, the QFLS to `qfls` V, with `steady` False only over the time steps."""
    spv = "VL1" in ref.dtype.names
    named = tj_named(c, k, nl, spv)
    assert set(named) | {"t", "G_frac", "Vext", "Jext", "Vint", "Jint"} == set(ref.dtype.names)
    scale = max(np.max(np.abs(ref["Jext"])), np.max(ref["JphotoL2"]))
    rows = np.ones(len(ref), bool) if steady else ref["t"] > 0
    for name, v in named.items():
        err = np.abs(v - ref[name])
        if name.startswith("QFLS"):
            assert np.max(err[rows]) < qfls, name
        elif name.startswith("V"):
            assert np.max(err) < 1e-9, name
        else:
            assert np.max(err) < (1e-5 if name == "errJ" else 1e-7) * scale, name


#: ZimT's cases whose tJFile columns the oracle reproduces: (QFLS bar in V, the steady rows
#: checked). Under light to 1e-9 V; in the dark after it to 4e-6 V, where ZimT's Gummel
#: overshoots before it settles; not in the steady state at t = 0 of the interface traps' sweep,
#: where ZimT leaves a transport layer's minority carriers unconverged (test_solver.py:719-737).
COLUMN_CASES = {"zimt_photo_light": (4e-6, True), "zimt_sweep_light": (1e-9, True),
                "zimt_sweep_diff_light": (1e-9, True), "zimt_traps_photo_light": (4e-6, True),
                "zimt_iface_sweep_light": (4e-6, False), "zimt_ions_slow_light": (4e-6, True),
                "zimt_tpv_light": (1e-9, True), "zimt_rseries_sweep_light": (1e-9, True),
                "zimt_sweep_spv_light": (1e-9, True)}


@pytest.mark.parametrize("case", sorted(COLUMN_CASES))
def test_the_oracle_reproduces_zimts_columns(case):
    """ZimT's tJFile columns (`columns`, restating transient._columns) against ZimT 5.36's
    own, at the reference's tolerances."""
    tvg, ref, dev, r = zimt_columns_run(case)
    qfls, steady = COLUMN_CASES[case]
    check_columns(r["columns"], 0, len(dev.i0), ref, qfls, steady)


def test_what_the_transient_refuses():
    setup, tvg, _ = zimt_case("zimt_photo_light")
    b = dd.prepare([build_device(setup, grid="simss")])
    setup, tvg, _ = zimt_case("zimt_region_slow_light")
    b = dd.prepare([build_device(setup, grid="simss")])
    b["R_series"] = np.array([1e-4])
    with pytest.raises(NotImplementedError, match="reaches a contact"):
        transient.solve_transient(b, tvg.t[:3], tvg.Vext[:3], tvg.G_frac[:3])


def test_a_given_state_is_checked_before_any_solve():
    """`solve_transient(..., initial=)` refuses, before it touches a GPU, what jaxdd refuses
    (tests/test_transient_state.py:93-114): a first time not after the state's, a state of
    another grid, densities that are not positive."""
    import dataclasses

    from jaxdd_b200.batch import prepare
    from jaxdd_b200.transient import TransientState, solve_transient
    setup, tvg, _ = zimt_case("zimt_photo_light")
    dev = build_device(setup, grid="simss")
    batch = prepare([dev])
    ones = np.ones((1, len(dev.x)))
    good = TransientState(t=np.array([0.0]), V=0 * ones, n=1e10 * ones, p=1e10 * ones,
                          anion=0 * ones, cation=0 * ones, V_int=np.zeros(1), J_ext=np.zeros(1),
                          dti=np.zeros(1), f_bulk=np.zeros((1, len(dev.x) - 2)),
                          f_interface=np.zeros(1))
    later = dataclasses.replace(tvg, **{k: getattr(tvg, k)[1:]
                                        for k in ("t", "Vext", "oc", "G_frac", "track", "dti")})
    with pytest.raises(ValueError, match="starts after it"):
        solve_transient(batch, later, initial=dataclasses.replace(good, t=np.array([1.0])))
    with pytest.raises(ValueError, match=r"initial\.n"):
        solve_transient(batch, later, initial=dataclasses.replace(good, n=np.ones((1, 3))))
    with pytest.raises(ValueError, match="positive"):
        solve_transient(batch, later, initial=dataclasses.replace(good, p=0 * ones))
    with pytest.raises(ValueError, match=r"initial\.V_int"):
        solve_transient(batch, later, initial=dataclasses.replace(good, V_int=np.zeros(2)))
    with pytest.raises(ValueError, match=r"initial\.f_bulk"):
        solve_transient(batch, later, initial=dataclasses.replace(good, f_bulk=np.zeros((1, 4))))


@pytest.mark.parametrize("case", ["zimt_ions_fast_light", "zimt_traps_photo_light",
                                  "zimt_iface_sweep_light", "zimt_region_slow_light",
                                  "zimt_regions2_light"])
def test_the_blocks_of_a_step_are_its_residuals_derivatives(case):
    """The 5x5 Jacobian of a time step (the reference takes it by autodiff:
    tests/test_solver.py's `the_ions_blocks_in_time_are_autodiff`) against central differences
    of the step's residual, off the solution, over a 1 us step with the traps' occupations
    anywhere in (0, 1): the blocks next to every perturbed point (bulk and interface traps, ion
    regions inside the device and at its contacts, whose densities follow their neighbours), the
    slots' columns and the constraints' derivatives. To 1e-7 of each row's largest entry beside
    the difference's own rounding."""
    setup, tvg, _ = zimt_case(case)
    dev = build_device(setup, grid="simss")
    d = dd.prepare([dev])
    bern = dd.BERNOULLI["simss"]
    Vint = np.array([0.5])
    y3, logs, _ = dd.start(d, Vint, bern, 1e-10, 200)
    s, ion, Vt = d["s"], d["ion"], d["Vt"]
    la, lc = dd.point_logs(logs, ion)
    za, zc = la + y3[..., 0] / Vt[:, None], lc - y3[..., 0] / Vt[:, None]
    y = np.concatenate([y3, np.stack([np.where(s["a_mask"] > 0, za, 0.0),
                                      np.where(s["c_mask"] > 0, zc, 0.0)], -1)], -1)
    NP = y.shape[1]
    rng = np.random.default_rng(2)
    before = transient.full_of(d, y, Vint)
    tr = {"dti": np.array([1e6]), "n": np.exp(before[:, 1:-1, 1]),
          "p": np.exp(before[:, 1:-1, 2]), "a": np.exp(before[:, 1:-1, 3]) * s["a_mask"],
          "c": np.exp(before[:, 1:-1, 4]) * s["c_mask"], "fb": rng.uniform(0, 1, (1, NP)),
          "fi": rng.uniform(0, 1, (1, NP + 1))}
    mobile = np.stack([s["a_mask"][0], s["c_mask"][0]], -1) > 0
    y[..., 0] += rng.normal(0, 0.01, NP)
    y[..., 1:3] += rng.normal(0, 0.1, (NP, 2))
    y[..., 3:] += np.where(mobile, rng.normal(0, 0.1, (NP, 2)), 0.0)

    def system(yy, ll):
        full, dV = transient.ion_full(d, transient.full_of(d, yy, Vint), bern, tr["dti"])
        F, A, Bb, C, U = transient.assemble(full, d, tr, ll, bern)
        g, W, D = transient.constraints(full, ll, ion, dV)
        return F, g, (A, Bb, C, U, W, D)

    F0, _, (A, Bb, C, U, W, D) = system(y, logs)
    h, eps = 1e-6, np.finfo(float).eps
    scale = np.maximum(np.maximum(np.abs(A[0]).max(2), np.abs(Bb[0]).max(2)), np.abs(C[0]).max(2))

    def bar(F):
        return 1e-7 * scale + 100 * eps * np.maximum(np.abs(F[0]), np.abs(F0[0])) / h

    nodes = sorted({0, 1, NP // 2, NP - 2, NP - 1}
                   | {j for i in dev.i1[:-1] for j in (i - 2, i - 1, i) if 0 <= j < NP})
    for j in nodes:
        for c in range(5):
            yp, ym = y.copy(), y.copy()
            yp[0, j, c] += h
            ym[0, j, c] -= h
            Fp, gp, _ = system(yp, logs)
            Fm, gm, _ = system(ym, logs)
            an = np.zeros_like(F0[0])
            an[j] = Bb[0, j, :, c]
            if j > 0:
                an[j - 1] = C[0, j - 1, :, c]
            if j < NP - 1:
                an[j + 1] = A[0, j + 1, :, c]
            assert np.all(np.abs((Fp - Fm)[0] / (2 * h) - an) <= bar(Fp)), (j, c)
            assert np.allclose((gp - gm)[0] / (2 * h), W[0, :, j, c], rtol=0,
                               atol=1e-7 * np.max(np.abs(W)) + 1e-30), (j, c)
    for k in range(logs.shape[1]):
        lp, lm = logs.copy(), logs.copy()
        lp[0, k] += h
        lm[0, k] -= h
        Fp, gp, _ = system(y, lp)
        Fm, gm, _ = system(y, lm)
        assert np.all(np.abs((Fp - Fm)[0] / (2 * h) - U[0, :, :, k]) <= bar(Fp)), k


def test_the_integral_current_in_time_is_the_one_the_equations_balance():
    """In time the integral form sums each point's `U` over its control volume, in which its
    continuity equation and Poisson's hold: the current of the differential form of the same
    solution to 1e-9 of the scale, on the graded grid (its spacing changes from point to point),
    through the light switched on (tests/test_solver.py:583-605, here without the surface
    recombination that case adds). ZimT's sums (`zimt_current`) are off by more than 1e-3 of
    the scale there, and leave the differential form as it is."""
    import dataclasses
    setup, tvg, _ = zimt_case("zimt_photo_light")
    differential = dataclasses.replace(setup, raw=dict(setup.raw, currDiffInt="1"))
    b = dd.prepare([build_device(s, grid="graded") for s in (setup, differential)])
    S = 40
    steps = (tvg.t[:S], tvg.Vext[:S], tvg.G_frac[:S], tvg.track[:S], tvg.failure_mode)
    r = transient.solve_transient(b, *steps)
    assert r["converged"].all()
    scale = np.max(np.abs(r["J_ext"][1]))
    assert np.max(np.abs(r["J_ext"][0] - r["J_ext"][1])) < 1e-9 * scale
    z = transient.solve_transient(b, *steps, zimt_current=True)
    assert np.max(np.abs(z["J_ext"][0] - r["J_ext"][1])) > 1e-3 * scale
    assert np.array_equal(z["J_ext"][1], r["J_ext"][1])


def test_transients_with_and_without_ions_in_one_batch():
    """Devices with mobile ions (one region of two layers, with the differential current)
    beside devices with traps and with neither, in one batch of 5x5 blocks (the others' ion rows
    held), each with its own steps and failure mode: each device's `Jext` is ZimT's to the
    bar of its own case (tests/test_solver.py:698-712)."""
    names = ("zimt_ions_slow_light", "zimt_region_diff_light", "zimt_photo_light",
             "zimt_traps_photo_light")
    cases = [zimt_case(c) for c in names]
    tvgs = [tvg for _, tvg, _ in cases]
    b = dd.prepare([build_device(setup, grid="simss") for setup, _, _ in cases])
    r = transient.solve_transient(b, *(np.stack([getattr(t, f) for t in tvgs])
                                       for f in ("t", "Vext", "G_frac", "track")),
                                  np.array([t.failure_mode for t in tvgs]),
                                  bernoulli_name="simss", zimt_current=True)
    assert r["converged"].all()
    for k, (name, (_, _, ref)) in enumerate(zip(names, cases)):
        scale = np.max(np.abs(ref["Jext"]))
        assert np.max(np.abs(r["J_ext"][k] - ref["Jext"])) < ZIMT[name] * scale, name
