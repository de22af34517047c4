"""The C++ restatement of the oracle (oracle/dd_cpu.cpp) pinned to the NumPy oracle: the same
devices through both `solve_batch`s give J within 1e-10 of each device's current scale and the
same converged flags and iteration counts — drawn devices of the benchmark (frozen after a
pre-bias and with free ions), the p-i-n cell, and golden cases with interface traps, several ion
regions, the differential current and SIMsalabim's Bernoulli function. Iteration counts are equal
on nearly every point; they may differ where a step's size sits at the tolerance within
round-off."""

import numpy as np
import pytest

from conftest import GOLDEN
from jaxdd_b200.device import build_device
from jaxdd_b200.simss_input import read_setup
from oracle import cpu, dd

TOL = 1e-10


def _same(tree, V, **kw):
    J, ok, its = cpu.solve_batch(tree, V, **kw)
    Jo, oko, itso = dd.solve_batch(tree, V, **kw)
    err = np.max(np.abs(J - Jo), axis=1) / tree["J_scale"]
    assert np.array_equal(ok, oko)
    # the counts may differ where a stop test sits at its threshold within round-off (a start
    # already at the root, a slow point ended by the settled current): at most one point of a
    # device, or 5 % of them
    assert np.all(np.sum(its != itso, axis=1) <= max(1, 0.05 * its.shape[1])), (its, itso)
    assert np.all(err < TOL), err


def test_drawn_devices_and_the_pin_cell():
    from jaxdd_b200.workloads import V_SCAN, drawn_devices, pin_stack
    _same(dd.prepare(drawn_devices(6, NP=120)), V_SCAN)
    _same(dd.prepare([pin_stack(NP=150)]), V_SCAN)


@pytest.mark.parametrize("case,bern", [("iface_charged_light", "simss"),
                                       ("two_regions_light", "simss"),
                                       ("diff_iface_light", "simss"),
                                       ("region_htl_frozen_light", "exact")])
def test_golden_cases(case, bern):
    dev = build_device(read_setup(GOLDEN / "inputs" / case / "simulation_setup.txt"),
                       grid="simss")
    _same(dd.prepare([dev]), np.linspace(-0.2, 1.2, 15), bernoulli_name=bern)


def test_refuses_a_device_it_cannot_solve():
    from jaxdd_b200.workloads import drawn_devices
    tree = dd.prepare(drawn_devices(1, NP=60))
    with pytest.raises(ValueError):
        cpu.solve_batch(tree, np.array([]))


def test_the_mixed_precision_experiment_without_fp32_is_the_fp64_solve():
    """`solve_batch_mixed` with no FP32 sweep (theta < 0) is one pass of `solve_batch`; with
    FP32 sweeps on large steps it still reaches the same curves where both converge."""
    from jaxdd_b200.workloads import V_SCAN, drawn_devices
    tree = dd.prepare(drawn_devices(2, NP=100))
    J, ok, its = cpu.solve_batch(tree, V_SCAN, first_max_iter=60)
    Jm, okm, itsm, st = cpu.solve_batch_mixed(tree, V_SCAN, -1.0)
    assert np.array_equal(J, Jm) and np.array_equal(ok, okm) and np.array_equal(its, itsm)
    assert np.all(st[:, 0] == 0) and np.all(st[:, 1] > 0)
    J3, ok3, _, st3 = cpu.solve_batch_mixed(tree, V_SCAN, 0.1)
    assert np.all(st3[:, 0] > 0)
    both = ok3 & ok
    assert np.all(np.abs(J3 - J)[both] <= 1e-8 * np.repeat(tree["J_scale"], V_SCAN.size)[both.ravel()])
