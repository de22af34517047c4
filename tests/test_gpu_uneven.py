"""Devices of uneven grid size and voltage count in one launch (`solve_uneven`) against the
oracle solving each device on its own, as jaxdd must (one grid size and voltage list per
`prepare`/`solve_batch`, batch.py:151-155): J within 1e-6 of each device's current scale,
converged flags equal."""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from jaxdd_b200.batch import concat, prepare, solve_uneven  # noqa: E402
from jaxdd_b200.workloads import drawn_device  # noqa: E402
from oracle import dd  # noqa: E402

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA GPU")]


def _check(devs, lists, got):
    for dev, V, (J, ok, its) in zip(devs, lists, got):
        od = dd.prepare([dev])
        Jo, oko, itso = dd.solve_batch(od, V)
        assert np.array_equal(ok, oko[0])
        assert np.max(np.abs(J - Jo[0])) < 1e-6 * od["J_scale"][0]


def test_uneven_grids_and_voltage_lists_match_the_oracle():
    """Ten devices, NP from 150 to 260, each with its own voltage list: some unsorted, one of a
    single voltage, one below its pre-bias only."""
    rng = np.random.default_rng(5)
    devs = [drawn_device(k, NP=(150, 260)) for k in range(10)]
    lists = []
    for k in range(10):
        n = int(rng.integers(4, 12))
        V = np.round(rng.uniform(-0.2, 1.2, n), 6)
        lists.append(V if k % 3 else np.sort(V))
    lists[4] = np.array([0.55])
    lists[6] = np.array([0.9, 0.2, -0.1])
    got = solve_uneven(prepare(devs, ragged=True), lists)
    _check(devs, lists, got)


def test_uneven_parts_concatenated_into_one_launch():
    """Two separately packed parts of different grid sizes in one launch (how the uneven
    benchmark packs its chunks)."""
    a = [drawn_device(k, NP=(150, 170)) for k in range(32)]
    b = [drawn_device(k, NP=(280, 300)) for k in range(32, 64)]
    both = concat([prepare(a, ragged=True), prepare(b, ragged=True)], ragged=True)
    V = np.round(np.linspace(-0.2, 1.3, 7), 10)
    lists = [V[: 3 + k % 5] for k in range(64)]
    got = solve_uneven(both, lists)
    pick = [0, 5, 31, 32, 40, 63]
    _check([(a + b)[k] for k in pick], [lists[k] for k in pick], [got[k] for k in pick])
