"""Transients of a batch: jaxdd's `solve_transient` (src/jaxdd/transient.py:537-637) on the GPU.

Each device starts from its steady state at the first step (`t = 0`; `dd_solve_states` at the
first voltage and generation factor, no pre-bias), then `dd_transient` takes every device
through all its steps in one launch: per step one Newton solve of implicit Euler with the mobile
ions as unknowns of their own (5×5 blocks bordered by the ion slots), the traps' occupations
carried from step to step, the current with each density's change, the ions' currents and the
displacement current, and ZimT's main loop (which steps are kept, each step's Δt from the last
one kept).

With `profiles=True` every step's state is written beside its current (`TransientResult.state`);
with `initial=` (a `TransientState`) the devices start from that state instead of a steady one.

The voltage is given at every step, or with an open circuit or a series resistance the internal
voltage is an unknown of each step's Newton solve. Refused (`NotImplementedError`), not
approximated: photon recycling.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib
from .batch import Batch, _gpu, descriptor, initial_state
from .simss_input import TVG

__all__ = ["STOP_FAILED", "STOP_STATIC", "ChargeGradients", "TransientResult", "TransientState",
           "Work", "charge_gradients", "solve_transient", "tj_columns"]

#: `TransientResult.stop`: a failed step ended the run (transient.py:240)
STOP_STATIC, STOP_FAILED = 1, 2


@dataclass(frozen=True)
class TransientState:
    """The last state kept, per device (jaxdd transient.py:72-94): `t`, the potential `V` and
    the densities `n`, `p`, `anion`, `cation` on every point (the ions 0 outside their regions),
    `V_int`, `J_ext`, `dti`, and the traps' occupations `f_bulk` (interior points) and
    `f_interface` (intervals)."""

    t: np.ndarray
    V: np.ndarray
    n: np.ndarray
    p: np.ndarray
    anion: np.ndarray
    cation: np.ndarray
    V_int: np.ndarray
    J_ext: np.ndarray
    dti: np.ndarray
    f_bulk: np.ndarray
    f_interface: np.ndarray


@dataclass(frozen=True)
class TransientResult:
    """Per device and step (devices × steps), as jaxdd's (transient.py:97-135): `J` the internal
    current density (A/m²), `J_ext` with the shunt, `V_int`, `V_ext`, `converged`, `iterations`,
    `accepted` (the steps ZimT keeps); per device `stop` (0, `STOP_STATIC` where ZimT's automatic
    stop found the state static, or `STOP_FAILED`); `t` each step's
    time; `final` the last state kept; with `profiles=True` `profiles` `{"V", "n", "p", "anion",
    "cation", "f_bulk", "f_interface", "dti"}` (devices × steps × points, or per device where
    the grids differ), from which `state(k)` is step k's state. `columns` ZimT's other tJFile
    columns (jaxdd transient.py:163-222; devices × steps, the per-layer ones devices × steps ×
    the batch's most layers), `n_layers` each device's; `tj_columns` names them as ZimT does."""

    J: np.ndarray
    J_ext: np.ndarray
    V_int: np.ndarray
    V_ext: np.ndarray
    converged: np.ndarray
    iterations: np.ndarray
    accepted: np.ndarray
    stop: np.ndarray
    t: np.ndarray
    final: TransientState
    columns: dict
    profiles: dict | None = None
    n_layers: np.ndarray | None = None

    def state(self, k: int) -> TransientState:
        """Every device's state at step `k` (jaxdd transient.py:124-135): the step's solution,
        as the next step starts from it where the step was kept."""
        if self.profiles is None:
            raise ValueError("a step's state needs the profiles: solve_transient(profiles=True)")
        prof = self.profiles

        def at(a):
            if a.dtype == object:
                return _stack([row[k] for row in a])
            return a[:, k]
        return TransientState(
            t=self.t[:, k], V=at(prof["V"]), n=at(prof["n"]), p=at(prof["p"]),
            anion=at(prof["anion"]), cation=at(prof["cation"]), V_int=self.V_int[:, k],
            J_ext=self.J_ext[:, k], dti=prof["dti"][:, k], f_bulk=at(prof["f_bulk"]),
            f_interface=at(prof["f_interface"]))


def _stack(xs):
    """Per-device arrays stacked, or an object array of them where their lengths differ."""
    if len({np.shape(x) for x in xs}) == 1:
        return np.stack(xs)
    out = np.empty(len(xs), dtype=object)
    out[:] = xs
    return out


def _per_device(name, value, lengths):
    """`initial.<name>` as one float array per device of the given lengths."""
    shape = (len(lengths), *sorted(set(lengths)))
    bad = ValueError(f"initial.{name}: one value per device and point, {shape}, got "
                     f"{np.shape(value) if np.asarray(value).dtype != object else 'ragged'}")
    if isinstance(value, np.ndarray) and value.dtype != object and value.ndim != 2:
        raise bad
    try:
        rows = list(value)
    except TypeError:
        raise bad from None
    if len(rows) != len(lengths):
        raise bad
    out = [np.asarray(r, dtype=float) for r in rows]
    if any(r.shape != (m,) for r, m in zip(out, lengths)):
        raise bad
    return out


def _checked_initial(initial: TransientState, devs, t) -> dict:
    """`solve_transient`'s `initial` checked against the devices and their steps as jaxdd
    checks it (transient.py:498-534), with the same messages: one value per device and point,
    per device for the scalars; the bulk traps' occupations on the interior points, the
    interface traps' on the intervals (not read where no device has interface traps); every
    first time after the state's; the densities positive, the ions where they are mobile."""
    n = len(devs)
    points = [len(d.x) for d in devs]
    st = {f: _per_device(f, getattr(initial, f), points)
          for f in ("V", "n", "p", "anion", "cation")}
    for f in ("t", "V_int", "J_ext", "dti"):
        v = np.asarray(getattr(initial, f), dtype=float)
        if v.shape != (n,):
            raise ValueError(f"initial.{f}: one value per device ({n}), got {v.shape}")
        st[f] = v
    st["f_bulk"] = _per_device("f_bulk", initial.f_bulk, [m - 2 for m in points])
    fi = initial.f_interface
    if not any(d.interface is not None for d in devs):
        st["f_interface"] = [np.zeros(m - 1) for m in points]
    else:
        st["f_interface"] = _per_device("f_interface", fi, [m - 1 for m in points])
    if not np.all(np.asarray(t)[:, 0] > st["t"]):
        raise ValueError("a transient from a state starts after it: every device's first time "
                         "must exceed its state's t")
    if not all(np.all(a > 0) for a in st["n"] + st["p"]):
        raise ValueError("initial.n and initial.p must be positive on every point")
    for name, mask in (("anion", "anion_mask"), ("cation", "cation_mask")):
        for d, a in zip(devs, st[name]):
            m = getattr(d, mask)
            if m is not None and np.any(np.asarray(m, bool) & ~(a > 0)):
                raise ValueError(f"initial.{name} must be positive where the device's "
                                 f"{name}s are mobile")
    return st


def _steps(tvgs: list[TVG]):
    if len({len(x.t) for x in tvgs}) != 1:
        raise ValueError("one tVG for the batch, or one per device, all of one length")
    t, V, G, track = (np.stack([np.asarray(getattr(x, k), dtype=float) for x in tvgs])
                      for k in ("t", "Vext", "G_frac", "track"))
    oc = np.stack([np.asarray(x.oc, dtype=bool) for x in tvgs])
    fm = np.array([x.failure_mode for x in tvgs], dtype=np.int32)
    tols = np.array([[x.tol_pois, x.tol_dens, x.tol_curr, x.conv_var] for x in tvgs],
                    dtype=float)
    return t, np.where(oc, 0.0, V), G, track.astype(np.int32), fm, oc, tols


def reaches_contact(d) -> bool:
    """Whether a region of mobile ions of device `d` reaches a contact."""
    return any(m is not None and bool(m[0] or m[-1]) for m in (d.anion_mask, d.cation_mask))


def _check_batch(batch: Batch, vint: bool) -> None:
    devs = batch["devices"]
    if vint and any(reaches_contact(d) for d in devs):
        raise NotImplementedError("the internal voltage an unknown (an open circuit, a series "
                                  "resistance) with an ion region that reaches a contact: not "
                                  "built")


class Work:
    """The device-side inputs of one transient run, packed once: the start's plan (the steady
    state at the first step), the per-point record, the steps, the outputs and the workspace.
    `run()` solves the start and the transient on the current stream; the outputs stay on the
    device (`out`)."""

    def __init__(self, batch: Batch, tvg, tol: float = 1e-10, max_iter: int = 200,
                 bernoulli_name: str = "exact", zimt_current: bool = False,
                 gradients: bool = False, profiles: bool = False, initial=None,
                 zimt_ion_currents: bool = False, vint: bool = False,
                 columns: bool = False):
        import torch
        from .adjoint import plan as _plan
        devs = batch["devices"]
        tvgs = list(tvg) if isinstance(tvg, (list, tuple)) else [tvg] * len(devs)
        if len(tvgs) != len(devs):
            raise ValueError("one tVG for the batch, or one per device, all of one length")
        t, V, G, track, fm, oc, tols = _steps(tvgs)
        R = np.array([d.R_series for d in devs])
        # the internal voltage an unknown of every device's steps where any is at the open
        # circuit or has a series resistance (transient.py:600-601)
        self.vint = vint = bool(vint or oc.any() or np.any(R > 0))
        _check_batch(batch, vint)
        init = None if initial is None else _checked_initial(initial, devs, t)
        self.batch, self.tol, self.max_iter = batch, tol, max_iter
        self.bern = _lib.DD_BERNOULLI[bernoulli_name]
        self.g = g = _gpu(batch)
        cuda = g.stat.device
        Bp, nodes, lanes = batch["Bp"], batch["np_max"] + 2, batch["lane_of"]
        self.S = S = t.shape[1]
        self.t, self.V = t, V
        # the start: the steady state at the first step's voltage (0 V at the open circuit) and
        # generation, no pre-bias
        V0 = np.where(oc[:, 0], 0.0, V[:, 0])
        self.plan = _plan(batch, [[float(v)] for v in V0], tol=tol, max_iter=max_iter,
                          bernoulli_name=bernoulli_name)
        y0 = np.zeros((nodes, 3, Bp))
        for k, d in enumerate(devs):
            y0[:len(d.x), :, lanes[k]] = initial_state(d, float(V0[k]))
        self.plan.y0.copy_(torch.from_numpy(y0))
        scal = g.scal.clone()
        gf = scal[_lib.C["GFRAC"]].cpu().numpy()
        gf[lanes] = G[:, 0]
        scal[_lib.C["GFRAC"]] = torch.from_numpy(gf).to(cuda)
        scal[_lib.C["PRECOND"]] = 0.0
        self.scal0 = scal
        # the per-point record: permittivity and the ions' mobilities
        X = np.zeros((nodes, _lib.DD_NT, Bp))
        for k, d in enumerate(devs):
            m = len(d.x)
            X[:m, 0, lanes[k]] = d.eps
            if d.mu_anion is not None:
                X[:m, 1, lanes[k]] = d.mu_anion
            if d.mu_cation is not None:
                X[:m, 2, lanes[k]] = d.mu_cation
        self.X = torch.from_numpy(X).to(cuda)
        # the steps: one list for all lanes where every device has the same
        same = all(np.array_equal(a[0], a[j]) for a in (t, V, G, track, oc)
                   for j in range(len(a)))
        if same:
            self.stride = 0
            cols, tr, ocs = (t[0], V[0], G[0]), track[0], oc[0]
        else:
            self.stride = Bp

            def lane_major(a):
                out = np.zeros((S, Bp), dtype=a.dtype)
                out[:, lanes] = a.T
                return out
            cols, tr = (lane_major(t), lane_major(V), lane_major(G)), lane_major(track)
            ocs = lane_major(oc)
        self.ocv = torch.from_numpy(np.ascontiguousarray(ocs, dtype=np.uint8)).to(cuda)
        rl = np.zeros(Bp)
        rl[lanes] = R
        self.rser = torch.from_numpy(rl).to(cuda)
        gv0 = np.zeros(Bp)  # the shunt's current at the start, where its solve failed
        gv0[lanes] = batch["G_shunt"] * V0
        self.gv0 = torch.from_numpy(gv0).to(cuda)
        self.jext0 = torch.zeros(Bp, dtype=torch.float64, device=cuda)
        # ZimT's tJFile columns: each lane's layers (first and last point, thickness)
        self.n_layers = np.array([len(d.i0) for d in devs])
        self.nl = int(self.n_layers.max()) if columns else 0
        if columns:
            if self.nl > _lib.DD_COL_MAXL:
                raise NotImplementedError(f"the tJFile columns of more than "
                                          f"{_lib.DD_COL_MAXL} layers")
            lay = np.zeros((3, self.nl, Bp))
            lay[0] = -1.0
            for k, d in enumerate(devs):
                m = len(d.i0)
                lay[0, :m, lanes[k]] = d.i0
                lay[1, :m, lanes[k]] = d.i1
                lay[2, :m, lanes[k]] = [d.x[b] - d.x[a] for a, b in zip(d.i0, d.i1)]
            self.lay = torch.from_numpy(lay).to(cuda)
        tl = np.zeros((3, Bp))  # the automatic stop's tolPois, tolDens and tolCurr
        tl[:, lanes] = tols[:, :3].T
        self.tols = torch.from_numpy(tl).to(cuda)
        cvl = np.ones(Bp, dtype=np.int32)  # and its convVar
        cvl[lanes] = tols[:, 3].astype(np.int32)
        self.cv = torch.from_numpy(cvl).to(cuda)
        self.tv, self.vv, self.gv = (torch.from_numpy(np.ascontiguousarray(c)).to(cuda)
                                     for c in cols)
        self.trk = torch.from_numpy(np.ascontiguousarray(tr, dtype=np.int32)).to(cuda)
        fml = np.ones(Bp, dtype=np.int32)
        fml[lanes] = fm
        self.fm = torch.from_numpy(fml).to(cuda)
        self.zimt = int(bool(zimt_current))
        self.ion_last = int(bool(zimt_ion_currents))
        f64, u8, i32 = torch.float64, torch.uint8, torch.int32
        self.out = {
            "J": torch.empty((S, Bp), dtype=f64, device=cuda),
            "J_ext": torch.empty((S, Bp), dtype=f64, device=cuda),
            "converged": torch.empty((S, Bp), dtype=u8, device=cuda),
            "iterations": torch.empty((S, Bp), dtype=i32, device=cuda),
            "accepted": torch.empty((S, Bp), dtype=u8, device=cuda),
            "stop": torch.empty(Bp, dtype=i32, device=cuda),
            "V_int": torch.empty((S, Bp), dtype=f64, device=cuda),
            **({"columns": torch.zeros((S, _lib.DD_COL_SCALARS + 8 * self.nl, Bp), dtype=f64,
                                       device=cuda)} if self.nl else {}),
            "state": torch.empty((nodes, 5, Bp), dtype=f64, device=cuda),
            "logs": torch.zeros((_lib.DD_MAXK, Bp), dtype=f64, device=cuda),
            "f_bulk": torch.empty((nodes, Bp), dtype=f64, device=cuda),
            "f_iface": torch.empty((nodes, Bp), dtype=f64, device=cuda),
        }
        self.gradients = gradients
        if gradients:
            self.out["Q"] = torch.empty(Bp, dtype=f64, device=cuda)
            self.out["dQ"] = torch.empty((2, Bp), dtype=f64, device=cuda)
        if profiles:
            self.out["prof_state"] = torch.empty((S, nodes, 5, Bp), dtype=f64, device=cuda)
            self.out["prof_f_bulk"] = torch.empty((S, nodes, Bp), dtype=f64, device=cuda)
            self.out["prof_f_iface"] = torch.empty((S, nodes, Bp), dtype=f64, device=cuda)
            self.out["prof_dti"] = torch.empty((S, Bp), dtype=f64, device=cuda)
        # the given state to start from: V, ln n, ln p, and ln a, ln c where the ions are mobile
        self.initial = init
        if init is not None:
            st = np.zeros((nodes, 5, Bp))
            fb, fi, sc = np.zeros((nodes, Bp)), np.zeros((nodes, Bp)), np.zeros((4, Bp))
            for k, d in enumerate(devs):
                m, ln = len(d.x), lanes[k]
                st[:m, 0, ln] = init["V"][k]
                st[:m, 1, ln] = np.log(init["n"][k])
                st[:m, 2, ln] = np.log(init["p"][k])
                for c, (name, mask) in enumerate((("anion", d.anion_mask),
                                                  ("cation", d.cation_mask)), start=3):
                    if mask is not None:
                        mob = np.asarray(mask, bool)
                        st[:m, c, ln] = np.where(mob, np.log(np.where(mob, init[name][k], 1.0)),
                                                 0.0)
                fb[1:m - 1, ln] = init["f_bulk"][k]
                fi[:m - 1, ln] = init["f_interface"][k]
                sc[:, ln] = [init[f][k] for f in ("t", "V_int", "J_ext", "dti")]
            self.init = {name: torch.from_numpy(a).to(cuda)
                         for name, a in (("state", st), ("f_bulk", fb), ("f_iface", fi),
                                         ("scalars", sc))}
        size = ctypes.c_size_t(0)
        desc = descriptor(batch, g, self.plan.y0)
        _lib.check(_lib.lib().dd_transient_workspace_bytes(ctypes.byref(desc),
                                                           ctypes.byref(size)),
                   "dd_transient_workspace_bytes")
        self.ws = torch.empty(size.value, dtype=torch.uint8, device=cuda)

    def run(self):
        """The start and the transient, on the current stream: `(out, start_converged)`
        (`start_converged` None from a given state)."""
        import torch
        from .adjoint import solve_states as _solve_states
        g = self.g
        if self.initial is None:
            J0, ok0, _, ckpt = _solve_states(self.plan, g.stat, self.scal0, g.iface)
            start, start_logs = ckpt["states"][0].data_ptr(), ckpt["logs"][0].data_ptr()
            init = None
            # the start's external current (the shunt's included), its shunt's alone where the
            # start failed (transient.py:453-456)
            off = self.plan.offsets.long().clamp(max=J0.numel() - 1)
            self.jext0.copy_(torch.where(ok0[off] > 0, J0[off], self.gv0))
        else:
            ok0, start, start_logs = None, None, None
            init = ctypes.byref(_lib.DdTransientInit(*(self.init[k].data_ptr() for k in (
                "state", "f_bulk", "f_iface", "scalars"))))
        steps = _lib.DdSteps(self.S, self.stride, self.tv.data_ptr(), self.vv.data_ptr(),
                             self.gv.data_ptr(), self.trk.data_ptr(), self.fm.data_ptr(),
                             self.zimt, self.ion_last, int(self.vint), self.ocv.data_ptr(),
                             self.rser.data_ptr(), self.jext0.data_ptr(), self.tols[0].data_ptr(),
                             self.tols[1].data_ptr(), self.nl,
                             self.lay.data_ptr() if self.nl else None, self.cv.data_ptr(),
                             self.tols[2].data_ptr())
        o = self.out
        out = _lib.DdTransientOut(*(o[k].data_ptr() if k in o else None for k in (
            "J", "J_ext", "converged", "iterations", "accepted", "stop", "state", "logs",
            "f_bulk", "f_iface", "Q", "dQ", "prof_state", "prof_f_bulk", "prof_f_iface",
            "prof_dti", "V_int", "columns")))
        opts = _lib.DdOpts(float(self.tol), int(self.max_iter), int(self.max_iter), 0,
                           self.bern, _lib.DD_MODE_BATCH, 0, 0)
        desc = descriptor(self.batch, g, self.plan.y0)
        _lib.check(_lib.lib().dd_transient(
            ctypes.byref(desc), self.X.data_ptr(), ctypes.byref(steps), start, start_logs, init,
            ctypes.byref(opts), ctypes.byref(out), self.ws.data_ptr(), self.ws.numel(),
            torch.cuda.current_stream(g.stat.device).cuda_stream),
            "dd_transient")
        return o, ok0


def solve_transient(batch: Batch, tvg, tol: float = 1e-10, max_iter: int = 200,
                    bernoulli_name: str = "exact", zimt_ion_currents: bool = False,
                    ions=None, vint=None, zimt_current: bool = False, recycle=None,
                    profiles: bool = False, ion_flux: str = "electrochemical",
                    initial=None, columns: bool = True) -> TransientResult:
    """A batch (`prepare`) through ZimT's time steps `tvg` (a `TVG`, or one per device, all of
    one length): jaxdd's `solve_transient` (transient.py:537-637) with the same arguments.
    `zimt_current`: ZimT's sums in the integral current (each point's change over the interval
    after it); by default over each point's control volume. `ion_flux`: both of jaxdd's are the
    Scharfetter–Gummel flux without ion sites, the only case built. `profiles`: every step's
    state (`TransientResult.profiles`, `state(k)`). `initial` (a `TransientState`, e.g. a
    result's `final` or `state(k)`): every device starts from it instead of from a steady state,
    its slots' scales 1 and the first step's guess the state itself (no extrapolation), checked
    as jaxdd checks it (`ValueError`). `zimt_ion_currents`: with several ion regions of a
    species each species' last region's current alone, as ZimT 5.36 has it; by default every
    region's. An ion region that reaches a contact takes the contact's density from its
    neighbour, nothing flowing over the contact's interval (jaxdd's `_ion_full`). Where any step
    is at the open circuit (`TVG.oc`) or any device has a series resistance, the internal
    voltage is an unknown of every device's steps (`vint`, also forced by `vint=True`): its row
    the external current at the open circuit, else `V_int + J_ext R_series = V_ext`. Not built
    (raise `NotImplementedError`): `recycle`; the internal voltage an unknown with an ion region
    that reaches a contact. `columns` (this build's switch, on by default as jaxdd always forms
    them): ZimT's tJFile columns of every step in `TransientResult.columns`, from one more pass
    over each step's solution on the GPU. `ions` is accepted for the
    reference's signature: the ions are unknowns of every step here, which leaves devices
    without mobile ions as they are."""
    if recycle is not None:
        raise NotImplementedError("photon recycling in transients: not built")
    if ion_flux not in ("electrochemical", "modified-drift"):
        raise ValueError(f"ion_flux {ion_flux!r}: one of ('electrochemical', 'modified-drift')")
    del ions
    work = Work(batch, tvg, tol=tol, max_iter=max_iter, bernoulli_name=bernoulli_name,
                zimt_current=zimt_current, profiles=profiles, initial=initial,
                zimt_ion_currents=zimt_ion_currents, vint=bool(vint), columns=columns)
    o, _ = work.run()
    return result(work, o)


def result(work: Work, o) -> TransientResult:
    """`Work.run()`'s device outputs as a `TransientResult` in the caller's device order."""
    batch = work.batch
    lanes = batch["lane_of"]
    devs = batch["devices"]

    def per_step(name, dtype=None):
        a = o[name].cpu().numpy()[:, lanes].T
        return a if dtype is None else a.astype(dtype)

    J, J_ext = per_step("J"), per_step("J_ext")
    ok, its = per_step("converged", bool), per_step("iterations", int)
    acc = per_step("accepted", bool)
    stop = o["stop"].cpu().numpy()[lanes]
    V_int = per_step("V_int")
    R = np.array([d.R_series for d in devs])
    V_ext = V_int + J_ext * R[:, None]
    state = o["state"].cpu().numpy()[:, :, lanes]  # nodes × 5 × devices
    fb = o["f_bulk"].cpu().numpy()[:, lanes]
    fi = o["f_iface"].cpu().numpy()[:, lanes]
    t = work.t
    n = len(devs)
    init = work.initial
    # the last kept step of each device, its time and 1/Δt (Δt from the step kept before it);
    # from a given state its time and 1/Δt until a step is kept
    last = np.full(n, -1)
    kept_t = np.zeros(n) if init is None else init["t"].copy()
    kept_dti = np.zeros(n) if init is None else init["dti"].copy()
    for k in range(n):
        prev = kept_t[k]
        for s in range(t.shape[1]):
            if acc[k, s]:
                tk = t[k, s]
                kept_dti[k] = 0.0 if tk == 0 else 1.0 / (tk - prev if tk > prev else 1.0)
                prev = tk
                last[k] = s
        kept_t[k] = prev
    rows = np.arange(n)
    fields = _states(devs, state, fb, fi)
    at = np.maximum(last, 0)
    V0 = V_int[:, 0] if init is None else init["V_int"]
    J0 = np.full(n, np.nan) if init is None else init["J_ext"]
    final = TransientState(
        t=kept_t, **fields, V_int=np.where(last >= 0, V_int[rows, at], V0),
        J_ext=np.where(last >= 0, J_ext[rows, at], J0), dti=kept_dti)
    profiles = None
    if "prof_state" in o:
        ps = o["prof_state"].cpu().numpy()[..., lanes]  # steps × nodes × 5 × devices
        pfb = o["prof_f_bulk"].cpu().numpy()[..., lanes]
        pfi = o["prof_f_iface"].cpu().numpy()[..., lanes]
        steps = [_states(devs, ps[s], pfb[s], pfi[s]) for s in range(t.shape[1])]
        profiles = {name: _stack([np.stack([st[name][k] for st in steps]) for k in range(n)])
                    for name in steps[0]}
        profiles["dti"] = o["prof_dti"].cpu().numpy()[:, lanes].T
    columns = {}
    if "columns" in o:
        c = o["columns"].cpu().numpy()[..., lanes]  # steps × columns × devices
        nl = work.nl
        for q, name in enumerate(_lib.COL_SCALARS):
            columns[name] = c[:, q].T
        for q, name in enumerate(_lib.COL_LAYER):
            base = _lib.DD_COL_SCALARS + q * nl
            columns[name] = np.transpose(c[:, base:base + nl], (2, 0, 1))
    return TransientResult(J=J, J_ext=J_ext, V_int=V_int, V_ext=V_ext, converged=ok,
                           iterations=its, accepted=acc, stop=stop, t=t, final=final,
                           columns=columns, profiles=profiles, n_layers=work.n_layers)


def tj_columns(result: TransientResult, k: int = 0, spv: bool = False) -> dict:
    """Device `k`'s steps as ZimT 5.36's tJFile names its columns, in its order (jaxdd
    transient.py:228-250): `Vext Jext errJ Vint Jint`, per layer `QFLS`, `Jphoto`, `Jdir`,
    `JbulkElec`, `JbulkHoles`, per interface `JintElec`, `JintHoles`, then `JminLeft JminRight
    JShunt Jnion Jpion JD`; with `spv` each layer's voltage drop `VL1`, `VL2`, ..."""
    if not result.columns:
        raise ValueError("no columns: solve_transient(..., columns=True)")
    c = {name: np.asarray(v)[k] for name, v in result.columns.items()}
    nl = int(result.n_layers[k])
    out = {"Vext": result.V_ext[k], "Jext": result.J_ext[k], "errJ": c["errJ"],
           "Vint": result.V_int[k], "Jint": result.J[k]}
    for name in ("QFLS", "Jphoto", "Jdir", "JbulkElec", "JbulkHoles"):
        out.update({f"{name}L{j + 1}": c[name][:, j] for j in range(nl)})
    for name in ("JintElec", "JintHoles"):
        out.update({f"{name}L{j + 1}L{j + 2}": c[name][:, j] for j in range(nl - 1)})
    out.update({name: c[name] for name in ("JminLeft", "JminRight", "JShunt", "Jnion", "Jpion",
                                           "JD")})
    if spv:
        out.update({f"VL{j + 1}": c["VL"][:, j] for j in range(nl)})
    return out


def _states(devs, state, fb, fi) -> dict:
    """`TransientState`'s arrays from the kernel's (state nodes × 5 × devices, the traps'
    occupations nodes × devices): the densities from their logarithms, the ions where they are
    mobile, the bulk traps' occupations on the interior points, the interface traps' on the
    intervals."""
    Vs, ns, ps, As, Cs, fbs, fis = [], [], [], [], [], [], []
    for k, d in enumerate(devs):
        m = len(d.x)
        st = state[:m, :, k]
        Vs.append(st[:, 0])
        ns.append(np.exp(st[:, 1]))
        ps.append(np.exp(st[:, 2]))
        am = np.asarray(d.anion_mask, bool) if d.anion_mask is not None else np.zeros(m, bool)
        cm = np.asarray(d.cation_mask, bool) if d.cation_mask is not None else np.zeros(m, bool)
        As.append(np.where(am, np.exp(st[:, 3]), 0.0))
        Cs.append(np.where(cm, np.exp(st[:, 4]), 0.0))
        fbs.append(fb[1:m - 1, k])
        fis.append(fi[:m - 1, k])
    return {"V": _stack(Vs), "n": _stack(ns), "p": _stack(ps), "anion": _stack(As),
            "cation": _stack(Cs), "f_bulk": _stack(fbs), "f_interface": _stack(fis)}


@dataclass(frozen=True)
class ChargeGradients:
    """Per device: `Q` the integrated current `sum_k J_k (t_k - t_(k-1))` over the kept steps
    (C/m², J the internal current), and its derivatives in the log of the ion density (both
    species' totals scaled together) and of the ion mobility (both species'); `result` the
    transient itself."""

    Q: np.ndarray
    dQ_dlnN_ion: np.ndarray
    dQ_dlnmu_ion: np.ndarray
    result: TransientResult


def charge_gradients(batch: Batch, tvg, tol: float = 1e-10, max_iter: int = 200,
                     bernoulli_name: str = "exact", zimt_current: bool = False,
                     vint: bool = False) -> ChargeGradients:
    """The integrated transient current and its gradient in the ion density and the ion mobility
    (the transient workload's gradients), in forward mode through every step as jaxdd differentiates
    its transients (`jax.jvp` through each step's `_converged_jvp`, batch.py:661-737): one
    `dd_transient` launch with the tangents carried beside the state. With the internal voltage
    an unknown (`vint`, as `solve_transient` decides it: an open circuit, a series resistance)
    it has a tangent of its own, from the tangent system's voltage row."""
    work = Work(batch, tvg, tol=tol, max_iter=max_iter, bernoulli_name=bernoulli_name,
                zimt_current=zimt_current, gradients=True, vint=vint)
    o, _ = work.run()
    lanes = batch["lane_of"]
    dQ = o["dQ"].cpu().numpy()[:, lanes]
    return ChargeGradients(Q=o["Q"].cpu().numpy()[lanes], dQ_dlnN_ion=dQ[0], dQ_dlnmu_ion=dQ[1],
                           result=result(work, o))

