"""`solve_states` on the GPU against the oracle's restatement (jaxdd batch.py:1165-1191): the
profiles, the quasi-Fermi level splitting, the ions and the radiative measures of each state, in
the caller's voltage order, for devices with frozen and with free ions."""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from jaxdd_b200 import prepare, solve_states  # noqa: E402
from jaxdd_b200.workloads import drawn_devices  # noqa: E402
from oracle import dd  # noqa: E402

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA GPU")]


def test_states_match_the_oracle():
    devs = drawn_devices(6, NP=120)
    V = [0.9, -0.1, 0.5, 1.1]
    got = solve_states(prepare(devs), V)
    ref = dd.solve_states(dd.prepare(devs), V)
    assert np.array_equal(got["converged"], ref["converged"])
    assert got["converged"].all()
    scale = dd.prepare(devs)["J_scale"][:, None]
    assert np.all(np.abs(got["J"] - ref["J"]) < 1e-6 * scale)
    assert np.max(np.abs(got["V"] - ref["V"])) < 1e-8
    for key in ("n", "p", "anion", "cation"):
        rel = np.abs(got[key] - ref[key]) / np.maximum(np.abs(ref[key]), 1e-30)
        assert np.max(rel) < 1e-6, key
    assert np.max(np.abs(got["qfls"] - ref["qfls"])) < 1e-8
    assert np.allclose(got["implied_voc"], ref["implied_voc"], rtol=0, atol=1e-9)
    assert np.allclose(got["plqy"], ref["plqy"], rtol=1e-6, atol=0)
    # the splitting is V_T ln(n p / n_i^2) of the profiles it comes with
    ni2 = np.array([d.ni ** 2 for d in devs])[:, None, :]
    Vt = np.array([d.Vt for d in devs])[:, None, None]
    assert np.allclose(got["qfls"], Vt * np.log(got["n"] * got["p"] / ni2), rtol=0, atol=1e-12)


def test_one_state_matches_the_oracle():
    """`solve_state` (jaxdd solver.py:2063-2093) on the GPU, solve_jv's scan at one voltage,
    against the oracle's restatement: the SimSS cell of `none_light` (NP 400), the p-i-n cell and
    a frozen and a free-ion drawn device (NP 120), at 0 and 0.8 V and at half the generation, and
    the shunted cell of `resist_light` at 0.8 V:
    converged as the oracle, J within 1e-6 of the current scale and without the shunt's current,
    the potential, ions and radiative measures to the bars of the batch test above, the
    densities and their splitting there where Newton weighs them (above its floor, as the
    reference compares states: tests/test_free_surface.py:290-310)."""
    from jaxdd_b200 import StateResult, build_device, read_setup, solve_state
    from jaxdd_b200.workloads import pin_stack
    from conftest import GOLDEN
    cell = build_device(read_setup(GOLDEN / "inputs" / "none_light" / "simulation_setup.txt"))
    shunted = build_device(read_setup(GOLDEN / "inputs" / "resist_light" / "simulation_setup.txt"))
    cases = [(d, V, None) for d in [cell, pin_stack(NP=120)] + drawn_devices(2, NP=120)
             for V in (0.0, 0.8)] + [(cell, 0.0, 0.5), (shunted, 0.8, None)]
    for d, V, g in cases:
        got = solve_state(d, V, g_frac=g)
        ref = dd.solve_state(d, V, g_frac=g)
        assert isinstance(got, StateResult)
        assert got.converged and ref["converged"]
        assert np.array_equal(got.x, ref["x"])
        scale = float(dd.prepare([d])["J_scale"][0])
        assert abs(got.J - ref["J"]) < 1e-6 * scale, (got.J, ref["J"])
        assert np.max(np.abs(got.V - ref["V"])) < 1e-8
        floor = 1e-12 * np.max(d.N_c)
        weighed = (ref["n"] > floor) & (ref["p"] > floor)
        for key in ("n", "p", "anion", "cation"):
            a, b = getattr(got, key), ref[key]
            assert a.shape == b.shape == (len(d.x),)
            w = b > floor if key in ("n", "p") else np.ones(len(b), bool)
            assert np.max(np.abs(a - b)[w] / np.maximum(np.abs(b[w]), 1e-30)) < 1e-6, key
        assert np.max(np.abs(got.qfls - ref["qfls"])[weighed]) < 1e-8
        assert np.allclose(got.qfls, d.Vt * np.log(got.n * got.p / d.ni ** 2), rtol=0, atol=1e-12)
        assert abs(got.implied_voc - ref["implied_voc"]) < 1e-9
        assert abs(got.plqy / ref["plqy"] - 1) < 1e-6
