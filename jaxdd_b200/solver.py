"""One device's J-V curve: the drop-in for jaxdd's `solve_jv` (jaxdd src/jaxdd/solver.py:2041-2060),
run by the same kernel as `solve_batch` in its solve_jv mode: each voltage in the caller's order
from the last converged solution (no extrapolation), Newton to `tol`, the round-off floor or the
problem's own noise floor (`_noise_step`, solver.py:1728-1751), `RuntimeError` where a pre-bias
does not converge (solver.py:2228-2229)."""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _lib
from .batch import _gather, prepare, run

__all__ = ["JVResult", "solve_jv"]


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
        from dataclasses import replace
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
