"""The solve's launch forms on a B200: the work queue (a batch of more devices than the GPU holds
at once, each pair of threads taking the next device when its own is done) gives every device
the curve it gets on its own, bit for bit; the autotuner times every form, keeps one, and the
solves after it give the same curves."""

import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from jaxdd_b200 import _lib  # noqa: E402
from jaxdd_b200.batch import prepare, solve_batch, tune  # noqa: E402
from jaxdd_b200.building import SweepStructure, build, parameters  # noqa: E402
from jaxdd_b200.simss_input import setup_from_texts  # noqa: E402
from jaxdd_b200.workloads import SEED_DRAWN, drawn_devices, drawn_texts  # noqa: E402

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA GPU")]


def _solve(st, P, D, V):
    """dd_solve of the devices of parameter columns P, D (built on the GPU) at voltages V."""
    stat, scal, iface, y0, Bp = build(st, P, D)
    n = P.shape[-1]
    nv = len(V)
    cuda = stat.device
    counts = np.zeros(Bp, dtype=np.int32)
    counts[:n] = nv
    tv = torch.as_tensor(np.tile(V, Bp), device=cuda)
    toff = torch.as_tensor((np.arange(Bp) * nv).astype(np.int32), device=cuda)
    tcnt = torch.as_tensor(counts, device=cuda)
    J = torch.full((Bp * nv,), float("nan"), dtype=torch.float64, device=cuda)
    ok = torch.zeros(Bp * nv, dtype=torch.uint8, device=cuda)
    its = torch.zeros(Bp * nv, dtype=torch.int32, device=cuda)
    status = torch.zeros(Bp, dtype=torch.int32, device=cuda)
    steps = torch.zeros((3, Bp), dtype=torch.int32, device=cuda)
    desc = _lib.DdBatch(n, Bp, st.NP, st.ka, st.kc, stat.data_ptr(), scal.data_ptr(),
                        iface.data_ptr(), y0.data_ptr())
    volts = _lib.DdVoltages(tv.data_ptr(), toff.data_ptr(), tcnt.data_ptr())
    opts = _lib.DdOpts(1e-10, 60, 60, 0, 0, _lib.DD_MODE_BATCH, 0, 0)
    so = _lib.lib()
    size = ctypes.c_size_t(0)
    _lib.check(so.dd_workspace_bytes(ctypes.byref(desc), ctypes.byref(size)), "workspace")
    ws = torch.empty(size.value, dtype=torch.uint8, device=cuda)
    _lib.check(so.dd_solve(ctypes.byref(desc), ctypes.byref(volts), ctypes.byref(opts),
                           J.data_ptr(), ok.data_ptr(), its.data_ptr(), status.data_ptr(),
                           steps.data_ptr(), ws.data_ptr(), ws.numel(),
                           torch.cuda.current_stream().cuda_stream), "dd_solve")
    torch.cuda.synchronize()
    shape = (Bp, nv)
    return (J.cpu().numpy().reshape(shape)[:n], ok.cpu().numpy().reshape(shape)[:n],
            its.cpu().numpy().reshape(shape)[:n], steps.cpu().numpy()[:, :n])


def test_the_work_queue_gives_every_device_its_own_curve():
    """24576 devices, more than the 148 SMs hold at once (about 19000 pairs of threads at the
    solve's 255 registers a thread), so the default form solves them from the work queue: each
    is one of six distinct devices (free ions, NP 40), and each device's curve, flags, iteration
    counts and step counts equal those of the six solved alone, bit for bit."""
    ks = [2 * i + 1 for i in range(6)]
    setups = [setup_from_texts(drawn_texts(k, np.random.default_rng([SEED_DRAWN, k]), 40))
              for k in ks]
    st = SweepStructure(setups[0])
    V = np.round(np.linspace(-0.2, 1.2, 8), 10)
    P, D = parameters(st, setups, first=np.full(len(setups), V[0]))
    n = 24576
    pick = np.arange(n) % len(setups)
    Jq, okq, itq, stq = _solve(st, P[:, :, pick], D[:, pick], V)
    J1, ok1, it1, st1 = _solve(st, P, D, V)
    assert ok1.mean() > 0.9
    assert np.array_equal(Jq, J1[pick], equal_nan=True)
    assert np.array_equal(okq, ok1[pick]) and np.array_equal(itq, it1[pick])
    assert np.array_equal(stq, st1[:, pick])


def test_the_autotuner_times_every_form_and_keeps_the_curves():
    from jaxdd_b200.workloads import V_SCAN
    b = prepare(drawn_devices(8, NP=60))
    ref = solve_batch(b, V_SCAN)
    choice = tune(b, V_SCAN)
    assert 0 <= choice["form"] < _lib.DD_SOLVE_FORMS
    assert all(t > 0 for t in choice["times_ms"])
    assert {"block", "queue"} <= set(choice)
    after = solve_batch(b, V_SCAN)
    for x, y in zip(ref, after):
        assert np.array_equal(x, y, equal_nan=True)
