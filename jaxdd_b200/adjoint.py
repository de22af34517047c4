"""The J-V curves as a differentiable function of the packed inputs, on the GPU.

`curves(stat, scal, iface, plan)` solves the batch (`dd_solve_states`, keeping the converged
solution of every voltage) and returns the curves as a torch tensor; its backward pass is the
adjoint kernel (`dd_adjoint`): one transposed bordered solve per converged voltage, by implicit
differentiation at the solution, which is what jaxdd's custom JVP of `_converged` gives under
`jax.grad` (batch.py:661-737). The gradient reaches every continuous input the solve reads (see
include/jaxdd_b200.h, `dd_adjoint`), so a differentiable map from device parameters to the packed
record (`jaxdd_b200.fitting.records`) carries it on to the parameters, as jaxdd's `device_tree`
(batch.py:142-148) does under `jax.grad`.

A voltage that did not converge has zero derivatives, as in jaxdd (`_converged_jvp`'s `valid`).
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib
from .batch import Batch, initial_state


@dataclass
class Plan:
    """What a differentiable solve needs besides the packed record: the voltages of each lane
    (flat, ascending per lane, offsets and counts), the start state, the solver's options."""
    batch: Batch
    v: object          # torch float64 [nflat]
    offsets: object    # torch int32 [Bp]
    counts: object     # torch int32 [Bp]
    y0: object         # torch float64 [np_max + 2][3][Bp]
    nv_max: int
    nflat: int
    tol: float = 1e-10
    max_iter: int = 60
    bernoulli: str = "exact"
    strict: bool = False
    mode: int = _lib.DD_MODE_BATCH  # DD_MODE_JV: solve_jv's scan (`solver.solve_state`)


def plan(batch: Batch, voltages, tol: float = 1e-10, max_iter: int = 60,
         bernoulli_name: str = "exact", strict: bool = False) -> Plan:
    """A plan for `batch` with the ascending `voltages` for every device (or a list of one
    ascending list per device)."""
    import torch
    devs = batch["devices"]
    if len(voltages) and np.ndim(voltages[0]) == 0:
        lists = [np.asarray(voltages, dtype=float)] * len(devs)
    else:
        lists = [np.asarray(v, dtype=float) for v in voltages]
    if len(lists) != len(devs):
        raise ValueError(f"{len(lists)} voltage lists for {len(devs)} devices")
    for v in lists:
        if v.size == 0 or np.any(np.diff(v) < 0):
            raise ValueError("each device's voltages must be ascending and not empty")
    Bp, npmax, lanes = batch["Bp"], batch["np_max"], batch["lane_of"]
    y0 = np.zeros((npmax + 2, 3, Bp))
    counts = np.zeros(Bp, dtype=np.int32)
    for k, d in enumerate(devs):
        first = d.V_pre if d.pre_cond else lists[k][0]
        y0[:len(d.x), :, lanes[k]] = initial_state(d, float(first))
        counts[lanes[k]] = len(lists[k])
    offsets = np.zeros(Bp, dtype=np.int32)
    offsets[1:] = np.cumsum(counts)[:-1]
    flat = np.zeros(int(counts.sum()))
    for k in range(len(devs)):
        flat[offsets[lanes[k]]:offsets[lanes[k]] + counts[lanes[k]]] = lists[k]
    cuda = torch.device("cuda")
    return Plan(batch=batch, v=torch.from_numpy(flat).to(cuda),
                offsets=torch.from_numpy(offsets).to(cuda),
                counts=torch.from_numpy(counts).to(cuda), y0=torch.from_numpy(y0).to(cuda),
                nv_max=int(counts.max()), nflat=int(flat.size), tol=tol, max_iter=max_iter,
                bernoulli=bernoulli_name, strict=strict)


def _desc(p: Plan, stat, scal, iface):
    b = p.batch
    return _lib.DdBatch(b["n"], b["Bp"], b["np_max"], b["ka"], b["kc"], stat.data_ptr(),
                        scal.data_ptr(), iface.data_ptr(), p.y0.data_ptr())


def _opts(p: Plan):
    return _lib.DdOpts(float(p.tol), int(p.max_iter), int(p.max_iter), int(bool(p.strict)),
                       _lib.DD_BERNOULLI[p.bernoulli], p.mode, 0, 0)


def solve_states(p: Plan, stat, scal, iface):
    """The curves and the checkpoints: `(J, ok, its, ckpt)`, J/ok/its flat in lane order;
    `ckpt["status"]` each lane's status (`DD_LANE_*`)."""
    import torch
    b = p.batch
    cuda = stat.device
    Bp, nodes = b["Bp"], b["np_max"] + 2
    for t, shape in ((stat, (nodes, _lib.DD_NF, Bp)), (scal, (_lib.DD_NS_BASE + _lib.DD_MAXK, Bp)),
                     (iface, (_lib.DD_MAXIF, _lib.DD_NIF, Bp))):
        if tuple(t.shape) != shape or t.dtype != torch.float64 or not t.is_contiguous():
            raise ValueError(f"a packed input of shape {tuple(t.shape)}: {shape} float64 wanted")
    J = torch.empty(p.nflat, dtype=torch.float64, device=cuda)
    ok = torch.empty(p.nflat, dtype=torch.uint8, device=cuda)
    its = torch.empty(p.nflat, dtype=torch.int32, device=cuda)
    status = torch.empty(Bp, dtype=torch.int32, device=cuda)
    ckpt = {"states": torch.empty((p.nv_max, nodes, 3, Bp), dtype=torch.float64, device=cuda),
            "logs": torch.zeros((p.nv_max, _lib.DD_MAXK, Bp), dtype=torch.float64, device=cuda),
            "pre": torch.empty((nodes, 3, Bp), dtype=torch.float64, device=cuda),
            "pre_logs": torch.zeros((_lib.DD_MAXK, Bp), dtype=torch.float64, device=cuda)}
    desc = _desc(p, stat, scal, iface)
    volts = _lib.DdVoltages(p.v.data_ptr(), p.offsets.data_ptr(), p.counts.data_ptr())
    opts = _opts(p)
    size = ctypes.c_size_t(0)
    _lib.check(_lib.lib().dd_workspace_bytes(ctypes.byref(desc), ctypes.byref(size)),
               "dd_workspace_bytes")
    ws = torch.empty(size.value, dtype=torch.uint8, device=cuda)
    stream = torch.cuda.current_stream(cuda).cuda_stream
    _lib.check(_lib.lib().dd_solve_states(
        ctypes.byref(desc), ctypes.byref(volts), ctypes.byref(opts), J.data_ptr(), ok.data_ptr(),
        its.data_ptr(), status.data_ptr(), None, ckpt["states"].data_ptr(),
        ckpt["logs"].data_ptr(), ckpt["pre"].data_ptr(), ckpt["pre_logs"].data_ptr(), p.nv_max,
        ws.data_ptr(), ws.numel(), stream), "dd_solve_states")
    ckpt["status"] = status
    return J, ok, its, ckpt


def adjoint(p: Plan, stat, scal, iface, ok, ckpt, J_bar):
    """`dd_adjoint`: the gradients of `sum(J_bar * J)` in the packed inputs."""
    import torch
    cuda = stat.device
    desc = _desc(p, stat, scal, iface)
    volts = _lib.DdVoltages(p.v.data_ptr(), p.offsets.data_ptr(), p.counts.data_ptr())
    opts = _opts(p)
    size = ctypes.c_size_t(0)
    _lib.check(_lib.lib().dd_adjoint_workspace_bytes(ctypes.byref(desc), ctypes.byref(size)),
               "dd_adjoint_workspace_bytes")
    ws = torch.empty(size.value, dtype=torch.uint8, device=cuda)
    J_bar = J_bar.to(torch.float64).contiguous()
    out = (torch.empty_like(stat), torch.empty_like(scal), torch.empty_like(iface))
    stream = torch.cuda.current_stream(cuda).cuda_stream
    _lib.check(_lib.lib().dd_adjoint(
        ctypes.byref(desc), ctypes.byref(volts), ctypes.byref(opts), ok.data_ptr(),
        J_bar.data_ptr(), ckpt["states"].data_ptr(), ckpt["logs"].data_ptr(),
        ckpt["pre"].data_ptr(), ckpt["pre_logs"].data_ptr(), p.nv_max, out[0].data_ptr(),
        out[1].data_ptr(), out[2].data_ptr(), ws.data_ptr(), ws.numel(), stream), "dd_adjoint")
    return out


def _function():
    import torch

    class Curves(torch.autograd.Function):
        """J (flat, lane order, the shunt's current added) of the packed inputs; backward by the
        adjoint kernel. `ok` and the iteration counts ride along, not differentiable."""

        @staticmethod
        def forward(ctx, stat, scal, iface, p):
            stat, scal, iface = stat.contiguous(), scal.contiguous(), iface.contiguous()
            J, ok, its, ckpt = solve_states(p, stat, scal, iface)
            ctx.save_for_backward(stat, scal, iface)
            ctx.p, ctx.ok, ctx.ckpt = p, ok, ckpt
            ctx.mark_non_differentiable(ok, its)
            return J, ok, its

        @staticmethod
        def backward(ctx, J_bar, _ok_bar, _its_bar):
            stat, scal, iface = ctx.saved_tensors
            gs, gc, gi = adjoint(ctx.p, stat, scal, iface, ctx.ok, ctx.ckpt, J_bar)
            return gs, gc, gi, None

    return Curves


_CURVES = None


def curves(stat, scal, iface, p: Plan):
    """`(J, ok, its)` of the packed inputs (torch float64 tensors on the GPU, laid out as
    `prepare` packs them) at the plan's voltages, flat in lane order; differentiable in the three
    inputs through the adjoint kernel."""
    global _CURVES
    if _CURVES is None:
        _CURVES = _function()
    return _CURVES.apply(stat, scal, iface, p)


def per_device(p: Plan, flat):
    """A flat lane-order tensor as devices x voltages (every device with the same count)."""
    b = p.batch
    off = p.offsets.cpu().numpy()[b["lane_of"]]
    n = int(p.counts.cpu().numpy()[b["lane_of"][0]])
    import torch
    idx = torch.as_tensor(off[:, None] + np.arange(n)[None, :], device=flat.device)
    return flat[idx]
