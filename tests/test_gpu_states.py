"""dd_solve_states: the same curves as dd_solve, and checkpoints that are the solutions those
curves were read at: one more Newton step from a checkpoint is negligible, and the current there
is the reported one (the shunt's aside). dd_newton_step solves with the ions mobile, so the scan's
checkpoints are checked on the devices whose ions stay mobile, and a frozen device's pre-bias
checkpoint at its pre-bias (before the freeze)."""

import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from gpu_inputs import pack  # noqa: E402
from jaxdd_b200 import _lib  # noqa: E402
from jaxdd_b200.batch import prepare  # noqa: E402
from jaxdd_b200.workloads import drawn_devices  # noqa: E402

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA GPU")]

V = np.round(np.linspace(-0.2, 1.3, 11), 10)


def _solve(batch, states: bool):
    g, desc, volts, keep, offsets, counts, n = pack(batch, [V] * batch["n"])
    cuda = torch.device("cuda")
    Bp, nodes = batch["Bp"], batch["np_max"] + 2
    out = {"J": torch.zeros(n, dtype=torch.float64, device=cuda),
           "ok": torch.zeros(n, dtype=torch.uint8, device=cuda),
           "its": torch.zeros(n, dtype=torch.int32, device=cuda),
           "status": torch.zeros(Bp, dtype=torch.int32, device=cuda),
           "steps": torch.zeros((3, Bp), dtype=torch.int32, device=cuda)}
    opts = _lib.DdOpts(1e-10, 60, 60, 0, 0, _lib.DD_MODE_BATCH, 0, 0)
    ws = g.workspace(desc)
    stream = torch.cuda.current_stream().cuda_stream
    so = _lib.lib()
    args = [ctypes.byref(desc), ctypes.byref(volts), ctypes.byref(opts)] + [
        out[k].data_ptr() for k in ("J", "ok", "its", "status", "steps")]
    if states:
        out["states"] = torch.full((len(V), nodes, 3, Bp), np.nan, dtype=torch.float64, device=cuda)
        out["logs"] = torch.full((len(V), _lib.DD_MAXK, Bp), np.nan, dtype=torch.float64, device=cuda)
        out["pre"] = torch.full((nodes, 3, Bp), np.nan, dtype=torch.float64, device=cuda)
        out["pre_logs"] = torch.full((_lib.DD_MAXK, Bp), np.nan, dtype=torch.float64, device=cuda)
        _lib.check(so.dd_solve_states(*args, out["states"].data_ptr(), out["logs"].data_ptr(),
                                      out["pre"].data_ptr(), out["pre_logs"].data_ptr(), len(V),
                                      ws.data_ptr(), ws.numel(), stream), "dd_solve_states")
    else:
        _lib.check(so.dd_solve(*args, ws.data_ptr(), ws.numel(), stream), "dd_solve")
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in out.items()}, offsets, g


def _step(batch, g, y, logs, vint, share):
    """dd_newton_step from lane-ordered (y, logs): the step's size and the current after it."""
    cuda = torch.device("cuda")
    from jaxdd_b200.batch import descriptor
    K = 2 if batch["ka"] + batch["kc"] <= 2 else 4
    y = np.nan_to_num(y, nan=0.0)  # the contacts' rows are not checkpointed (nor read)
    ty = torch.from_numpy(np.ascontiguousarray(y)).to(cuda)
    tl = torch.from_numpy(np.ascontiguousarray(logs[:K])).to(cuda)
    tv = torch.from_numpy(vint).to(cuda)
    size = torch.zeros(batch["Bp"], dtype=torch.float64, device=cuda)
    J = torch.zeros(batch["Bp"], dtype=torch.float64, device=cuda)
    desc = descriptor(batch, g, ty)
    ws = g.workspace(desc)
    opts = _lib.DdOpts(1e-10, 60, 60, 0, 0, 0, 0, 0)
    _lib.check(_lib.lib().dd_newton_step(
        ctypes.byref(desc), ty.data_ptr(), tl.data_ptr(), tv.data_ptr(), float(share),
        ctypes.byref(opts), size.data_ptr(), J.data_ptr(), ws.data_ptr(), ws.numel(),
        torch.cuda.current_stream().cuda_stream), "dd_newton_step")
    torch.cuda.synchronize()
    return size.cpu().numpy(), J.cpu().numpy()


def test_checkpoints_are_the_solutions_of_the_curves():
    devs = drawn_devices(8)
    batch = prepare(devs)
    ref, _, _ = _solve(batch, False)
    got, offsets, g = _solve(batch, True)
    for key in ("J", "ok", "its", "status"):
        assert np.array_equal(got[key], ref[key], equal_nan=True), key
    mobile = [k for k, d in enumerate(devs) if not (d.pre_cond and d.fix_ions)]
    assert mobile
    lanes = batch["lane_of"][mobile]
    scale = batch["J_scale"][mobile]
    for j in (0, 4, 10):
        vint = np.zeros(batch["Bp"])
        vint[batch["lane_of"][:batch["n"]]] = V[j]
        size, Jn = _step(batch, g, got["states"][j], got["logs"][j], vint, 1.0)
        pos = offsets[lanes] + j
        ok = got["ok"][pos] > 0
        assert ok.all()
        assert np.all(size[lanes] < 1e-6), size[lanes]
        shunt = batch["G_shunt"][mobile] * V[j]
        assert np.all(np.abs(Jn[lanes] - (got["J"][pos] - shunt)) <= 1e-8 * scale)


def test_prebias_checkpoint_of_frozen_devices():
    devs = drawn_devices(8)
    batch = prepare(devs)
    got, _, g = _solve(batch, True)
    frozen = [k for k, d in enumerate(devs) if d.pre_cond and d.fix_ions]
    assert frozen
    lanes = batch["lane_of"][frozen]
    vint = np.zeros(batch["Bp"])
    vint[batch["lane_of"][:batch["n"]]] = [d.V_pre if d.pre_cond else 0.0 for d in devs]
    size, _ = _step(batch, g, got["pre"], got["pre_logs"], vint, 1.0)
    assert np.all(np.isfinite(got["pre"][1:401, :, lanes]))
    assert np.all(size[lanes] < 1e-6), size[lanes]
