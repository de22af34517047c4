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


def test_a_solve_captured_in_a_cuda_graph_replays_the_direct_launch():
    """`dd_solve` (the queue counter's reset, the specialised and the generic kernel) captured
    once into a CUDA graph, as `bench.py` replays config 3's solve: each replay gives the direct
    launch's curves, flags and iterations bit for bit, also after the outputs were overwritten
    between replays, on uneven grids and voltage lists."""
    from jaxdd_b200.batch import descriptor, _gpu
    from jaxdd_b200.workloads import ragged_plan, ragged_voltages
    idx = np.arange(64)
    _, Nvs = ragged_plan(idx)
    devs = drawn_devices(64, NP=(60, 160))
    batch = prepare(devs, ragged=True)
    lists = [ragged_voltages(nv) for nv in Nvs]
    g = _gpu(batch)
    Bp, npmax, lanes = batch["Bp"], batch["np_max"], batch["lane_of"]
    from jaxdd_b200.batch import initial_state
    y0 = np.zeros((npmax + 2, 3, Bp))
    counts = np.zeros(Bp, dtype=np.int32)
    for k, d in enumerate(devs):
        first = d.V_pre if d.pre_cond else lists[k][0]
        y0[:len(d.x), :, lanes[k]] = initial_state(d, first)
        counts[lanes[k]] = len(lists[k])
    offsets = np.zeros(Bp, dtype=np.int32)
    offsets[1:] = np.cumsum(counts)[:-1]
    flat = np.zeros(int(counts.sum()))
    for k in range(len(devs)):
        flat[offsets[lanes[k]]:offsets[lanes[k]] + counts[lanes[k]]] = lists[k]
    cuda = torch.device("cuda")
    t_y0 = torch.from_numpy(y0).to(cuda)
    t_v, t_off, t_cnt = (torch.from_numpy(a).to(cuda) for a in (flat, offsets, counts))
    J = torch.empty(flat.size, dtype=torch.float64, device=cuda)
    ok = torch.empty(flat.size, dtype=torch.uint8, device=cuda)
    its = torch.empty(flat.size, dtype=torch.int32, device=cuda)
    status = torch.empty(Bp, dtype=torch.int32, device=cuda)
    steps = torch.zeros((3, Bp), dtype=torch.int32, device=cuda)
    desc = descriptor(batch, g, t_y0)
    volts = _lib.DdVoltages(t_v.data_ptr(), t_off.data_ptr(), t_cnt.data_ptr())
    opts = _lib.DdOpts(1e-10, 60, 60, 0, 0, _lib.DD_MODE_BATCH, 0, 0)
    ws = g.workspace(desc)
    so = _lib.lib()

    def launch(stream):
        _lib.check(so.dd_solve(ctypes.byref(desc), ctypes.byref(volts), ctypes.byref(opts),
                               J.data_ptr(), ok.data_ptr(), its.data_ptr(), status.data_ptr(),
                               steps.data_ptr(), ws.data_ptr(), ws.numel(), stream.cuda_stream),
                   "dd_solve")

    launch(torch.cuda.current_stream())
    torch.cuda.synchronize()
    direct = [t.cpu().numpy().copy() for t in (J, ok, its)]
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, capture_error_mode="relaxed"):
        launch(torch.cuda.current_stream())
    for _ in range(2):
        J.fill_(float("nan"))
        ok.zero_()
        its.zero_()
        graph.replay()
        torch.cuda.synchronize()
        for a, b in zip(direct, (J, ok, its)):
            np.testing.assert_array_equal(a, b.cpu().numpy())
    assert direct[1].all()
