"""One device's J-V curve and steady state: the drop-ins for jaxdd's `solve_jv` and
`solve_state` (jaxdd src/jaxdd/solver.py:2041-2093), run by the same kernel as `solve_batch` in
its solve_jv mode: each voltage in the caller's order from the last converged solution (no
extrapolation), Newton to `tol`, the round-off floor or the problem's own noise floor
(`_noise_step`, solver.py:1728-1751), `RuntimeError` where a pre-bias does not converge
(solver.py:2228-2229)."""

from __future__ import annotations

from dataclasses import dataclass, replace

import numpy as np

from . import _lib
from .adjoint import Plan
from .adjoint import solve_states as _solve_states
from .batch import _gather, _gpu, initial_state, observables, prepare, run

__all__ = ["JVResult", "StateResult", "solve_jv", "solve_state"]


@dataclass(frozen=True)
class JVResult:
    """jaxdd's `JVResult` (solver.py:171-177)."""

    V: np.ndarray
    J: np.ndarray
    converged: np.ndarray
    iterations: np.ndarray
    V_ext: np.ndarray | None = None


def solve_jv(dev, voltages, g_frac: float | None = None, tol: float = 1e-10,
             max_iter: int = 200, bernoulli_name: str = "exact",
             precision: str = "fp64") -> JVResult:
    """The J-V curve at `voltages` (internal = external without a series resistance), each
    solved from the last converged one (jaxdd solver.py:2041-2060)."""
    if g_frac is not None:
        dev = replace(dev, G_frac=float(g_frac))
    V = np.asarray(voltages, dtype=float).reshape(-1)
    batch = prepare([dev])
    first = dev.V_pre if dev.pre_cond else float(V[0])
    J, ok, its, status, offsets, _ = run(
        batch, [V], np.array([first]), tol=tol, max_iter=max_iter, start_iter=max_iter,
        strict=False, bernoulli_name=bernoulli_name, mode=_lib.DD_MODE_JV,
        precision=precision, jv_start=True)
    if int(status.cpu()[batch["lane_of"][0]]) == _lib.DD_LANE_PREBIAS_FAILED:
        raise RuntimeError(f"no convergence at the pre-bias {dev.V_pre} V")
    Jv, okv, itv = _gather(batch, J, ok, its, offsets, len(V), np.arange(len(V)))
    J0 = Jv[0]
    return JVResult(V, J0, okv[0], itv[0], V + J0 * dev.R_series)


@dataclass(frozen=True)
class StateResult:
    """jaxdd's `StateResult` (solver.py:181-202): one steady state on the device's NP + 2
    points (`V` in V, `n`, `p`, `anion`, `cation` in m^-3, `qfls` = V_T ln(n p / n_i^2) in eV)
    and what photoluminescence measures of it: `implied_voc` (V) and `plqy` of direct
    recombination (NaN where the device has none, or no generation); `J` in A/m^2."""

    x: np.ndarray
    V: np.ndarray
    n: np.ndarray
    p: np.ndarray
    qfls: np.ndarray
    implied_voc: float
    plqy: float
    J: float
    anion: np.ndarray
    cation: np.ndarray
    converged: bool
    iterations: int


def solve_state(dev, Vint: float = 0.0, g_frac: float | None = None, tol: float = 1e-10,
                max_iter: int = 200, bernoulli_name: str = "exact") -> StateResult:
    """The steady state at the internal voltage `Vint` (jaxdd solver.py:2063-2093): the scan of
    `solve_jv` at that one voltage (`dd_solve_states` in its solve_jv mode: the start, any
    pre-bias and freeze first), then the state's profiles, splitting, ions and radiative
    measures (`dd_observables`). `J` is the device's own current, without the shunt's, as
    jaxdd's `solve_state` reports it (`_current`); `RuntimeError` where a pre-bias does not
    converge."""
    import torch
    if g_frac is not None:
        dev = replace(dev, G_frac=float(g_frac))
    Vint = float(Vint)
    batch = prepare([dev])
    g = _gpu(batch)  # the GPU's copy of the record; raises where there is no GPU
    lane, Bp, nodes = int(batch["lane_of"][0]), batch["Bp"], len(dev.x)
    y0 = np.zeros((batch["np_max"] + 2, 3, Bp))
    y0[:nodes, :, lane] = initial_state(dev, dev.V_pre if dev.pre_cond else Vint, jv=True)
    counts = np.zeros(Bp, dtype=np.int32)
    counts[lane] = 1
    offsets = np.zeros(Bp, dtype=np.int32)
    offsets[1:] = np.cumsum(counts)[:-1]
    cuda = torch.device("cuda")
    p = Plan(batch=batch, v=torch.tensor([Vint], dtype=torch.float64, device=cuda),
             offsets=torch.from_numpy(offsets).to(cuda), counts=torch.from_numpy(counts).to(cuda),
             y0=torch.from_numpy(y0).to(cuda), nv_max=1, nflat=1, tol=tol, max_iter=max_iter,
             bernoulli=bernoulli_name, strict=False, mode=_lib.DD_MODE_JV)
    J, ok, its, ckpt = _solve_states(p, g.stat, g.scal, g.iface)
    if int(ckpt["status"][lane]) == _lib.DD_LANE_PREBIAS_FAILED:
        raise RuntimeError(f"no convergence at the pre-bias {dev.V_pre} V")
    prof, meas = observables(batch, p, ckpt)
    at = int(offsets[lane])
    shunt = Vint / dev.R_shunt if dev.R_shunt > 0 else 0.0
    prof = {k: v[0, :nodes, lane].cpu().numpy() for k, v in prof.items()}
    return StateResult(
        x=np.asarray(dev.x), V=prof["V"], n=prof["n"], p=prof["p"], qfls=prof["qfls"],
        implied_voc=float(meas["implied_voc"][0, lane]), plqy=float(meas["plqy"][0, lane]),
        J=float(J[at]) - shunt, anion=prof["anion"], cation=prof["cation"],
        converged=bool(ok[at]), iterations=int(its[at]))
