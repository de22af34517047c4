"""The transient on the GPU (`dd_transient` through `jaxdd_b200.solve_transient`) against the
oracle (`oracle.transient`) on the same devices and steps, and against ZimT 5.36's own `Jext`
(the reference's tests/data) at the reference's tolerances: electrons and holes, the bulk traps
in time, mobile ions over 2 x 50 ms and 2 x 5 s; config 5's transient (drawn devices with mobile
ions, a step to 0.9 V, log-spaced steps) on fewer steps; ZimT's failure modes; and at config 5's
2000 steps the properties that hold at any size (every step converged and kept, each region's
ions kept to their total, the current finite)."""

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


def test_config5_transient_matches_the_oracle():
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


def test_config5_full_steps_hold_their_invariants():
    devs = [drawn_device(k) for k in range(1, 129, 2)]
    r = solve_transient(prepare(devs), transient_steps(2000))
    assert r.converged.mean() > 0.999 and r.accepted.all()
    assert np.all(np.isfinite(r.J_ext))
    for k, d in enumerate(devs):
        assert abs(_number(r.final.anion[k], d.anion_mask, d) / d.anion_total - 1) < 1e-8
