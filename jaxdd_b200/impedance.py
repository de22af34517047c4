"""Impedance in the frequency domain from the steady state's Jacobian: jaxdd's
`solve_impedance` (src/jaxdd/impedance.py:365-409).

At the steady state of each device at `voltage` (the solve's own, `dd_solve_states`) a small
voltage drives `(J + iωM)·δy = −(∂F/∂V)·δV`, the traps' occupations following at their own rates;
`dd_admittance` solves it for every (device, frequency) on the GPU and linearises the current of
a time step (`Y = δJ/δV`). A batch with free mobile ions goes through `dd_admittance_ions`: the
ions are unknowns of their own (5×5 blocks, each region's number kept by a border), and the
linearised current has each region's ion current. With a series resistance and a shunt the
external `Z = 1/(Y + G_shunt) + R_series`.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib
from .batch import Batch, _gpu, descriptor


@dataclass(frozen=True)
class ImpedanceResult:
    """Per device and frequency (devices x frequencies): `Z` the external impedance (Ω·m²),
    `Y` the internal admittance δJ/δV_int (S/m², SIMsalabim's sign); per device the steady
    state's `J` (A/m²) and `converged` (jaxdd impedance.py:46-64)."""

    frequencies: np.ndarray
    Z: np.ndarray
    Y: np.ndarray
    J: np.ndarray
    converged: np.ndarray

    @property
    def capacitance(self) -> np.ndarray:
        return self.Y.imag / (2 * np.pi * self.frequencies)


def _mobile(batch: Batch) -> bool:
    """Whether any device of the batch has mobile ions (jaxdd impedance.py:391)."""
    return any(d.anion_total > 0 or d.cation_total > 0 for d in batch["devices"])


class Work:
    """The device-side inputs of one impedance run, packed once: the plan of the steady solve at
    `voltage`, the permittivities, the frequencies, the output and the workspace. `run()` solves
    the steady states and the admittances on the current stream and returns the device tensors
    `(J, converged, Y)` (J, converged flat in lane order; Y [frequency][re, im][lane])."""

    def __init__(self, batch: Batch, frequencies, voltage: float, tol: float = 1e-10,
                 max_iter: int = 60, bernoulli_name: str = "exact", dt: float | None = None):
        import torch
        from .adjoint import plan as _plan
        self.batch = batch
        self.plan = _plan(batch, [float(voltage)], tol=tol, max_iter=max_iter,
                          bernoulli_name=bernoulli_name)
        self.g = _gpu(batch)
        self.bern = _lib.DD_BERNOULLI[bernoulli_name]
        Bp, nodes, lanes = batch["Bp"], batch["np_max"] + 2, batch["lane_of"]
        cuda = self.g.stat.device
        self.ions = _mobile(batch)
        # the permittivity (and, with ions, the ions' mobilities) at every point
        X = np.zeros((nodes, _lib.DD_NT, Bp))
        for k, d in enumerate(batch["devices"]):
            m = len(d.x)
            X[:m, 0, lanes[k]] = d.eps
            if d.mu_anion is not None:
                X[:m, 1, lanes[k]] = d.mu_anion
            if d.mu_cation is not None:
                X[:m, 2, lanes[k]] = d.mu_cation
        self.X = torch.from_numpy(X).to(cuda)
        self.eps = self.X[:, 0, :].contiguous()
        self.vint = torch.full((Bp,), float(voltage), dtype=torch.float64, device=cuda)
        omega = 2 * np.pi * np.asarray(frequencies, dtype=float)
        # iω, or over implicit Euler's steps of dt (1 − e^(−iω dt))/dt (impedance.py:379-383)
        lap = 1j * omega if dt is None else -np.expm1(-1j * omega * dt) / dt
        laps = np.stack([lap.real, lap.imag], -1)
        self.dt = 0.0 if dt is None else float(dt)
        self.laps = torch.from_numpy(laps).to(cuda)
        self.nf = len(frequencies)
        self.Y = torch.empty((self.nf, 2, Bp), dtype=torch.float64, device=cuda)
        size = ctypes.c_size_t(0)
        desc = descriptor(batch, self.g, self.plan.y0)
        query = (_lib.lib().dd_admittance_ions_workspace_bytes if self.ions
                 else _lib.lib().dd_admittance_workspace_bytes)
        _lib.check(query(ctypes.byref(desc), self.nf, ctypes.byref(size)),
                   "dd_admittance_workspace_bytes")
        self.ws = torch.empty(size.value, dtype=torch.uint8, device=cuda)

    def run(self):
        import torch
        from .adjoint import solve_states as _solve_states
        g = self.g
        J, ok, _, ckpt = _solve_states(self.plan, g.stat, g.scal, g.iface)
        state = ckpt["states"][0]
        desc = descriptor(self.batch, g, state)
        stream = torch.cuda.current_stream(g.stat.device).cuda_stream
        if self.ions:
            _lib.check(_lib.lib().dd_admittance_ions(
                ctypes.byref(desc), state.data_ptr(), ckpt["logs"][0].data_ptr(),
                self.X.data_ptr(), self.vint.data_ptr(), self.laps.data_ptr(), self.nf,
                self.bern, self.dt, self.Y.data_ptr(), self.ws.data_ptr(), self.ws.numel(),
                stream), "dd_admittance_ions")
        else:
            _lib.check(_lib.lib().dd_admittance(
                ctypes.byref(desc), state.data_ptr(), self.eps.data_ptr(), self.vint.data_ptr(),
                self.laps.data_ptr(), self.nf, self.bern, self.dt, self.Y.data_ptr(),
                self.ws.data_ptr(), self.ws.numel(), stream), "dd_admittance")
        return J, ok, self.Y


def solve_impedance(batch: Batch, frequencies, voltage: float = 0.0, tol: float = 1e-10,
                    max_iter: int = 60, bernoulli_name: str = "exact",
                    ion_flux: str = "electrochemical",
                    dt: float | None = None) -> ImpedanceResult:
    """The impedance of a batch at the internal voltage `voltage` (V) at each of `frequencies`
    (Hz), from the steady state there by one complex linear solve per frequency (jaxdd
    impedance.py:371-409, same arguments). Free mobile ions move with the voltage as unknowns of
    their own. Several ion regions of a species each keep their own number; a region that
    reaches a contact takes the contact's ions from its neighbour's (jaxdd's `_ion_full`). With
    the differential current (`currDiffInt = 1`) the current's tangent is each interval's
    Scharfetter–Gummel flux's, the ions' too. Refused (`NotImplementedError`), as the reference
    refuses them: ions frozen at a pre-bias. `ion_flux`: one of jaxdd's two ion fluxes
    (`ValueError` otherwise); without ion sites both are the Scharfetter–Gummel flux, the only
    case built. `dt` (s): instead of the continuous response, what `solve_transient` sees
    through implicit Euler at steps of `dt` (its time terms at `(1 − e^(−iω dt))/dt`, the traps'
    occupations over each step as it solves them)."""
    if ion_flux not in ("electrochemical", "modified-drift"):
        raise ValueError(f"ion_flux {ion_flux!r}: one of ('electrochemical', 'modified-drift')")
    devs = batch["devices"]
    if _mobile(batch) and any(d.pre_cond and d.fix_ions for d in devs):
        raise NotImplementedError("impedance with ions frozen at a pre-bias")
    frequencies = np.atleast_1d(np.asarray(frequencies, dtype=float))
    if dt is not None and not dt > 0:
        raise ValueError(f"dt must be positive, got {dt}")
    work = Work(batch, frequencies, voltage, tol=tol, max_iter=max_iter,
                bernoulli_name=bernoulli_name, dt=dt)
    J, ok, Y = work.run()
    lanes = batch["lane_of"]
    p = work.plan
    Yc = Y.cpu().numpy()
    Yd = (Yc[:, 0, :] + 1j * Yc[:, 1, :])[:, lanes].T
    offsets = p.offsets.cpu().numpy()[lanes]
    Jd = J.cpu().numpy()[offsets]
    okd = ok.cpu().numpy()[offsets].astype(bool)
    Z = 1.0 / (Yd + batch["G_shunt"][:, None]) + batch["R_series"][:, None]
    return ImpedanceResult(frequencies=frequencies, Z=Z, Y=Yd, J=Jd, converged=okd)
