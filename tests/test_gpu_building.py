"""Devices built on the GPU (`dd_build`) against the host builder and packer for the same
parameters on the same grid structure (jaxdd's `device_tree(structure, params)`): every field of
the record, the scalars, the interface table and the start state; and a sweep built and solved
on the GPU against `solve_batch` of the host-built devices."""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from jaxdd_b200 import _lib  # noqa: E402
from jaxdd_b200.batch import initial_state, prepare, solve_batch  # noqa: E402
from jaxdd_b200.building import SweepStructure, build, parameters, solve_sweep  # noqa: E402
from jaxdd_b200.device import build_device  # noqa: E402
from jaxdd_b200.simss_input import setup_from_texts  # noqa: E402
from jaxdd_b200.workloads import SEED_DRAWN, drawn_texts  # noqa: E402

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA GPU")]


def _setups(parity: int, n: int = 6, NP: int = 120):
    """Drawn devices of one pre-bias pattern (even or odd index): one structure."""
    ks = [2 * i + parity for i in range(n)]
    return [setup_from_texts(drawn_texts(k, np.random.default_rng([SEED_DRAWN, k]), NP))
            for k in ks]


@pytest.mark.parametrize("parity", [0, 1])
def test_records_equal_the_host_builder(parity):
    setups = _setups(parity)
    st = SweepStructure(setups[0])
    P, D = parameters(st, setups, first=np.full(len(setups), -0.2))
    stat, scal, iface, y0, Bp = build(st, P, D)
    devs = [build_device(s, layout=st.layout) for s in setups]
    n = len(devs)
    for k, dev in enumerate(devs):
        b = prepare([dev])
        got_s = stat[:, :, k].cpu().numpy()
        ref_s = b["stat"][:, :, 0]
        rel = np.abs(got_s - ref_s) / np.maximum(np.abs(ref_s), 1e-300)
        assert rel.max() < 1e-12, (k, np.argwhere(rel >= 1e-12)[:5])
        got_c = scal[:, k].cpu().numpy()
        ref_c = b["scal"][:, 0]
        relc = np.abs(got_c - ref_c) / np.maximum(np.abs(ref_c), 1e-300)
        assert relc.max() < 1e-13, (k, np.argwhere(relc >= 1e-13))
        assert np.allclose(iface[:, :, k].cpu().numpy(), b["iface"][:, :, 0], rtol=1e-13, atol=0)
        first = dev.V_pre if dev.pre_cond else -0.2
        # ln n and ln p cross zero inside the device: an absolute floor at their operands'
        # round-off (values up to ~60; CUDA's log and FMA contraction against NumPy's)
        assert np.allclose(y0[:, :, k].cpu().numpy(), initial_state(dev, first), rtol=1e-13,
                           atol=1e-12)
    assert n == len(setups)


def test_a_sweep_solves_as_the_host_built_batch():
    setups = _setups(1, n=8, NP=100)
    st = SweepStructure(setups[0])
    V = np.round(np.linspace(-0.2, 1.2, 9), 10)
    J, ok, its = solve_sweep(st, setups, V)
    devs = [build_device(s, layout=st.layout) for s in setups]
    b = prepare(devs)
    Jh, okh, itsh = solve_batch(b, V)
    assert np.array_equal(ok, okh)
    assert np.all(np.abs(J - Jh) <= 1e-9 * b["J_scale"][:, None])
