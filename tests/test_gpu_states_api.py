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
