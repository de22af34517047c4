"""dd_solve_noalloc (the solve on the library's fixed scratch array) against dd_solve (the solve
on a caller's workspace), through the C ABI on a B200.

Three calls in a row on the fixed array, each against dd_solve on the same inputs: a batch of
drawn devices, then the reference's golden devices (another lane stride, node count and
Bernoulli form, in solve_jv mode), then the first batch again. Each later call finds the
previous call's contents in the array. Runs alone or after the other tests.
"""

import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from conftest import GOLDEN  # noqa: E402
from jaxdd_b200 import _lib  # noqa: E402
from jaxdd_b200.batch import _gpu, descriptor, initial_state, prepare  # noqa: E402
from jaxdd_b200.device import build_device  # noqa: E402
from jaxdd_b200.simss_input import read_setup  # noqa: E402

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA GPU")]

GOLDEN_CASES = ["thin_l1_light", "steady_1e17_thin_light", "iface_charged_light",
                "two_regions_light", "diff_iface_light", "region_etl_light"]


def _inputs(batch, volts, jv):
    """Device inputs of one solve: every device at the voltages `volts` (ascending), started at
    its pre-bias, or at the first voltage without one."""
    B, Bp, npmax = batch["n"], batch["Bp"], batch["np_max"]
    y0 = np.zeros((npmax + 2, 3, Bp))
    counts = np.zeros(Bp, dtype=np.int32)
    for k, dev in enumerate(batch["devices"]):
        lane = batch["lane_of"][k]
        first = dev.V_pre if dev.pre_cond else volts[0]
        y0[:len(dev.x), :, lane] = initial_state(dev, float(first), jv=jv)
        counts[lane] = len(volts)
    offsets = np.zeros(Bp, dtype=np.int32)
    offsets[1:] = np.cumsum(counts)[:-1]
    flat = np.zeros(int(counts.sum()))
    for k in range(B):
        lane = batch["lane_of"][k]
        flat[offsets[lane]:offsets[lane] + counts[lane]] = volts
    g = _gpu(batch)
    cuda = torch.device("cuda")
    t = {"y0": torch.from_numpy(y0).to(cuda), "v": torch.from_numpy(flat).to(cuda),
         "off": torch.from_numpy(offsets).to(cuda), "cnt": torch.from_numpy(counts).to(cuda)}
    desc = descriptor(batch, g, t["y0"])
    v = _lib.DdVoltages(t["v"].data_ptr(), t["off"].data_ptr(), t["cnt"].data_ptr())
    return g, desc, v, t, flat.size


def _solve(batch, volts, *, jv, bern, noalloc):
    g, desc, v, keep, n = _inputs(batch, volts, jv)
    cuda = torch.device("cuda")
    J = torch.full((n,), float("nan"), dtype=torch.float64, device=cuda)
    ok = torch.zeros(n, dtype=torch.uint8, device=cuda)
    its = torch.zeros(n, dtype=torch.int32, device=cuda)
    status = torch.zeros(batch["Bp"], dtype=torch.int32, device=cuda)
    steps = torch.zeros((3, batch["Bp"]), dtype=torch.int32, device=cuda)
    mode = _lib.DD_MODE_JV if jv else _lib.DD_MODE_BATCH
    its_max = 200 if jv else 60
    opts = _lib.DdOpts(1e-10, its_max, its_max, 0, _lib.DD_BERNOULLI[bern], mode, 0, 0)
    stream = torch.cuda.current_stream().cuda_stream
    so = _lib.lib()
    outs = (J.data_ptr(), ok.data_ptr(), its.data_ptr(), status.data_ptr(), steps.data_ptr())
    if noalloc:
        st = so.dd_solve_noalloc(ctypes.byref(desc), ctypes.byref(v), ctypes.byref(opts), *outs,
                                 stream)
    else:
        ws = g.workspace(desc)
        st = so.dd_solve(ctypes.byref(desc), ctypes.byref(v), ctypes.byref(opts), *outs,
                         ws.data_ptr(), ws.numel(), stream)
    _lib.check(st, "dd_solve_noalloc" if noalloc else "dd_solve")
    torch.cuda.synchronize()
    return (J.cpu().numpy(), ok.cpu().numpy(), its.cpu().numpy(), status.cpu().numpy(),
            steps.cpu().numpy())


def _assert_same(batch, got, ref):
    J, ok, its, status, steps = got
    Jr, okr, itsr, statusr, stepsr = ref
    lanes = batch["lane_of"]
    nv = len(J) // batch["n"]
    scale = np.repeat(batch["J_scale"][np.argsort(lanes)], nv)
    assert np.array_equal(np.isnan(J), np.isnan(Jr))
    fin = ~np.isnan(Jr)
    assert np.all(np.abs(J[fin] - Jr[fin]) <= 1e-6 * scale[fin])
    assert np.array_equal(ok, okr) and np.array_equal(its, itsr)
    assert np.array_equal(status[lanes], statusr[lanes])
    assert np.array_equal(steps[:, lanes], stepsr[:, lanes])


def test_fixed_scratch_solve_matches_the_workspace_solve():
    from jaxdd_b200.workloads import V_SCAN, drawn_devices
    drawn = prepare(drawn_devices(8))
    golden = prepare([build_device(read_setup(GOLDEN / "inputs" / c / "simulation_setup.txt"),
                                   grid="simss") for c in GOLDEN_CASES])
    v_golden = np.linspace(0.0, 1.1, 12)
    size = ctypes.c_size_t(0)
    for b in (drawn, golden):
        _lib.check(_lib.lib().dd_workspace_bytes(
            ctypes.byref(descriptor(b, _gpu(b), _gpu(b).stat)), ctypes.byref(size)),
            "dd_workspace_bytes")
        assert size.value <= _lib.DD_NOALLOC_SCRATCH_BYTES
    calls = [(drawn, V_SCAN, False, "exact"), (golden, v_golden, True, "simss"),
             (drawn, V_SCAN, False, "exact")]
    for batch, volts, jv, bern in calls:
        got = _solve(batch, volts, jv=jv, bern=bern, noalloc=True)
        ref = _solve(batch, volts, jv=jv, bern=bern, noalloc=False)
        _assert_same(batch, got, ref)
        assert got[1].mean() > 0.9  # the curves converged: a comparison of solved states
