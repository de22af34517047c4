"""Many devices at once: `prepare` packs them for the kernel, `solve_batch` solves their J-V
curves on the GPU. The drop-in for jaxdd's `prepare` / `solve_batch` (jaxdd
src/jaxdd/batch.py:151-223, 1136-1162), same arguments and results.

`prepare` writes the lane-interleaved layout of jaxdd_b200/csrc/dd_layout.h: per node the
stencils jaxdd's `_stencils` computes (solver.py:210-278) and the arrays its current reads, per
lane the scalars, per lane a small table of interface traps. Lanes are ordered by grid size and
by whether their ions are frozen after the pre-bias, so that the lanes of one warp take the same
path; results come back in the caller's device order.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .constants import Q

__all__ = ["Batch", "prepare", "solve_batch", "external_voltages"]

DENSITY_FLOOR = 1e-12  # solver.py:52


class Batch(dict):
    """A packed batch. Its keys include the per-device arrays the reference's batch pytree
    exposes to callers (`J_scale`, `R_series`, `G_shunt`, `Vt`, `NP`), in the caller's device
    order; the packed kernel inputs are `stat`, `scal`, `iface` (lane order `lane_of`)."""


def _slot_index(mask, slots):
    """Each point's slot index (-1 outside every mobile region)."""
    if slots is None:
        return np.where(mask, 0.0, -1.0), 1
    idx = np.full(mask.shape, -1.0)
    for k, m in enumerate(slots):
        idx[np.asarray(m, bool)] = k
    return idx, len(slots)


def _totals(total, totals):
    return np.array([float(total)]) if totals is None else np.asarray(totals, dtype=float)


def _pack_one(dev, stat, scal, iface, lane, ka_all, kc_all):
    """Write one device into lane `lane` of the packed arrays."""
    NP = len(dev.x) - 2
    h, L, eps = dev.h, dev.L, dev.eps
    i = np.arange(1, NP + 1)
    hm, hp = h[i - 1], h[i]
    w = hp + hm
    L2 = L * L
    facu = 2 * eps[i] / (hp * w * L2)
    facl = 2 * eps[i] / (hm * w * L2) - (eps[i] - eps[i - 1]) / (hm ** 2 * L2)
    facm = (eps[i] - eps[i - 1]) / (hm ** 2 * L2) - 2 * eps[i] * (1 / (hp * w * L2) + 1 / (hm * w * L2))
    S = _lib.S
    col = stat[:, :, lane]
    nodes = slice(0, NP + 2)
    rows = slice(1, NP + 1)
    col[nodes, S["OFFN"]] = dev.offset_n
    col[nodes, S["OFFP"]] = dev.offset_p
    col[nodes, S["MUN"]] = dev.mu_n
    col[nodes, S["MUP"]] = dev.mu_p
    col[nodes, S["H"]] = h
    dx = np.zeros(NP + 2)
    dx[:NP] = np.diff(dev.x[:NP + 1])
    col[nodes, S["DX"]] = dx
    col[rows, S["FACL"]] = facl
    col[rows, S["FACM"]] = facm
    col[rows, S["FACU"]] = facu
    col[rows, S["FAC"]] = 0.5 * L2 * hp * hm * w
    col[rows, S["SP"]] = 1.0 / (Q * dev.N_c[i])
    col[rows, S["SC"]] = 1.0 / (np.maximum(dev.mu_n[i], dev.mu_p[i]) * dev.Vt * dev.N_c[i] * hp)
    col[rows, S["DOP"]] = dev.N_A[i] - dev.N_D[i]
    col[nodes, S["KD"]] = dev.k_direct
    col[nodes, S["NI2"]] = dev.ni ** 2
    col[nodes, S["NT"]] = dev.srh_Nt
    col[nodes, S["CNT"]] = dev.srh_Cn
    col[nodes, S["CPT"]] = dev.srh_Cp
    col[nodes, S["NT0"]] = dev.srh_nt0
    col[nodes, S["PT0"]] = dev.srh_pt0
    col[nodes, S["G"]] = dev.G
    aslot, _ = _slot_index(np.asarray(dev.anion_mask, bool), dev.anion_slots)
    cslot, _ = _slot_index(np.asarray(dev.cation_mask, bool), dev.cation_slots)
    col[nodes, S["ASLOT"]] = aslot
    col[nodes, S["CSLOT"]] = cslot
    col[rows, S["AFIX"]] = dev.anion_fixed[i]
    col[rows, S["CFIX"]] = dev.cation_fixed[i]
    ifk = np.full(NP + 2, -2.0)
    ifk[list(dev.i1[:-1])] = -1.0
    if dev.interface is not None:
        edges = np.flatnonzero(np.asarray(dev.interface["Nt"]) > 0)
        if len(edges) > _lib.DD_MAXIF:
            raise NotImplementedError(f"more than {_lib.DD_MAXIF} trapped interfaces")
        for r, e in enumerate(edges):
            ifk[e] = r
            for name, key in (("NT", "Nt"), ("CN", "Cn"), ("CP", "Cp"), ("NT0LO", "nt0_lo"),
                              ("PT0LO", "pt0_lo"), ("NT0HI", "nt0_hi"), ("PT0HI", "pt0_hi"),
                              ("IW", "iw"), ("CHARGE", "charge"), ("CWE", "cwe")):
                iface[r, _lib.I[name], lane] = dev.interface[key][e]
    col[nodes, S["IFK"]] = ifk
    # per-lane scalars
    C = _lib.C
    generated = Q * L * np.sum(h[:-1] * dev.G[:-1]) / np.sum(h[:-1])
    sc = scal[:, lane]
    sc[C["VT"]] = dev.Vt
    sc[C["L"]] = L
    sc[C["V0"]] = dev.V0
    sc[C["VL"]] = dev.VL
    sc[C["LEFT"]] = float(dev.left_elec)
    sc[C["LNNL"]] = np.log(dev.n_left)
    sc[C["LNPL"]] = np.log(dev.p_left)
    sc[C["LNNR"]] = np.log(dev.n_right)
    sc[C["LNPR"]] = np.log(dev.p_right)
    sc[C["JSCALE"]] = max(generated, 1.0)
    sc[C["GSHUNT"]] = 1.0 / dev.R_shunt if dev.R_shunt > 0 else 0.0
    sc[C["PRECOND"]] = float(dev.pre_cond)
    sc[C["VPRE"]] = dev.V_pre
    sc[C["FIXIONS"]] = float(dev.fix_ions)
    sc[C["GFRAC"]] = dev.G_frac
    sc[C["NFLOOR"]] = DENSITY_FLOOR * np.max(dev.N_c)
    sc[C["NP"]] = NP
    sc[C["CURRDIFF"]] = float(dev.curr_diff)
    sc[C["HSUM"]] = np.sum(h[:NP + 1])
    sc[C["MID"]] = split_row(NP, ifk)
    ta = _totals(dev.anion_total, dev.anion_totals)
    tc = _totals(dev.cation_total, dev.cation_totals)
    sc[_lib.DD_NS_BASE:_lib.DD_NS_BASE + len(ta)] = ta
    sc[_lib.DD_NS_BASE + ka_all:_lib.DD_NS_BASE + ka_all + len(tc)] = tc
    # cation slot indices count from 0 within the cations; the kernel adds k_anion
    return max(generated, 1.0)


def split_row(NP: int, ifk: np.ndarray) -> int:
    """The row where the two halves of the kernel's twisted sweep meet: near the middle, with
    no layer interface on the three intervals around it (so that no interface term straddles
    the two halves)."""
    m0 = NP // 2
    for d in range(NP):
        for m in (m0 - d, m0 + d):
            if 2 <= m <= NP - 2 and all(ifk[e] == -2 for e in (m - 1, m, m + 1)):
                return m
    raise NotImplementedError(f"no row to split a grid of {NP} points between its interfaces")


def _empty_stat(nodes: int, Bp: int) -> np.ndarray:
    """Static records of nodes no device has: outside every ion slot and interface, unit row
    scales."""
    stat = np.zeros((nodes, _lib.DD_NF, Bp))
    stat[:, _lib.S["ASLOT"], :] = -1.0
    stat[:, _lib.S["CSLOT"], :] = -1.0
    stat[:, _lib.S["IFK"], :] = -2.0
    stat[:, _lib.S["SP"], :] = 1.0
    stat[:, _lib.S["SC"], :] = 1.0
    return stat


def prepare(devices, ragged: bool = False) -> Batch:
    """A batch of devices for `solve_batch` (jaxdd batch.py:151-223). Like jaxdd's, every device
    must have one grid size (`ValueError` otherwise) unless `ragged` is true: then devices of
    different NP share the launch, each lane sweeping its own grid."""
    devices = list(devices)
    if not devices:
        raise ValueError("an empty batch")
    sizes = sorted({len(d.x) for d in devices})
    if len(sizes) != 1 and not ragged:
        raise ValueError(f"a batch needs one grid size, got NP + 2 in {sizes}")
    B = len(devices)
    Bp = (B + 31) // 32 * 32
    npmax = max(len(d.x) for d in devices) - 2
    ka = max(1 if d.anion_slots is None else len(d.anion_slots) for d in devices)
    kc = max(1 if d.cation_slots is None else len(d.cation_slots) for d in devices)
    if ka + kc > _lib.DD_MAXK:
        raise NotImplementedError(f"{ka + kc} ion slots: at most {_lib.DD_MAXK}")
    # lanes: larger grids first, then frozen-after-pre-bias, then with mobile ions
    key = [(-(len(d.x)), not (d.pre_cond and d.fix_ions), d.anion_total + d.cation_total == 0)
           for d in devices]
    lane_order = sorted(range(B), key=lambda k: key[k])
    lane_of = np.empty(B, dtype=np.int64)
    lane_of[lane_order] = np.arange(B)
    stat = _empty_stat(npmax + 2, Bp)
    scal = np.zeros((_lib.DD_NS_BASE + _lib.DD_MAXK, Bp))
    iface = np.zeros((_lib.DD_MAXIF, _lib.DD_NIF, Bp))
    J_scale = np.zeros(B)
    for k, dev in enumerate(devices):
        J_scale[k] = _pack_one(dev, stat, scal, iface, int(lane_of[k]), ka, kc)
    # padding lanes: a harmless copy of lane 0's scalars (never run: n_lanes excludes them)
    out = Batch(
        stat=stat, scal=scal, iface=iface, lane_of=lane_of, n=B, Bp=Bp, np_max=npmax, ka=ka,
        kc=kc, devices=devices,
        J_scale=J_scale, R_series=np.array([d.R_series for d in devices]),
        G_shunt=np.array([1.0 / d.R_shunt if d.R_shunt > 0 else 0.0 for d in devices]),
        Vt=np.array([d.Vt for d in devices]), NP=np.array([len(d.x) - 2 for d in devices]),
    )
    return out


def concat(parts: list[Batch], ragged: bool = False) -> Batch:
    """One batch of several packed ones (each packed by `prepare` with the same grid size and
    slot counts), their devices in order; each part's lane order is kept, so a part packed in
    its own process needs no repacking. With `ragged`, parts of different grid sizes too (the
    smaller ones padded with empty nodes)."""
    first = parts[0]
    npmax = max(p["np_max"] for p in parts)
    for p in parts:
        if (p["ka"], p["kc"]) != (first["ka"], first["kc"]) or (
                p["np_max"] != npmax and not ragged):
            raise ValueError("concat needs parts of one grid size and slot counts")
        if p["n"] != p["Bp"]:
            raise ValueError("concat needs parts whose device count is a multiple of 32")

    def padded(p):
        if p["np_max"] == npmax:
            return p["stat"]
        out = _empty_stat(npmax + 2, p["Bp"])
        out[:p["np_max"] + 2] = p["stat"]
        return out

    lane_of, base, devs = [], 0, []
    for p in parts:
        lane_of.append(p["lane_of"] + base)
        base += p["Bp"]
        devs += p["devices"]
    out = Batch(
        stat=np.concatenate([padded(p) for p in parts], axis=2),
        scal=np.concatenate([p["scal"] for p in parts], axis=1),
        iface=np.concatenate([p["iface"] for p in parts], axis=2),
        lane_of=np.concatenate(lane_of), Bp=base, np_max=npmax, ka=first["ka"],
        kc=first["kc"], devices=devs)
    out["n"] = base
    for key in ("J_scale", "R_series", "G_shunt", "Vt", "NP"):
        out[key] = np.concatenate([p[key] for p in parts])
    return out


def initial_state(dev, Vint: float, jv: bool = False) -> np.ndarray:
    """SIMsalabim's `Init_Pot_Dens_Ions_Traps`: a linear potential and Fermi level
    (`batch._initial`, batch.py:276-299; `solver._initial`, solver.py:1882-1893, with
    `jv`), (NP + 2) x 3."""
    x, L, e = dev.x, dev.L, dev.left_elec
    V = dev.V0 + 0.5 * e * Vint + x * (dev.VL - dev.V0 - e * Vint) / L
    EF = dev.W_L - x * (dev.W_L - dev.W_R) / L
    if jv:
        n = dev.N_c * np.exp(-(EF - dev.E_c) / dev.Vt)
        return np.stack([V, np.log(n), np.log(dev.ni ** 2 / n)], -1)
    ln_n = np.log(dev.N_c) - (EF - dev.E_c) / dev.Vt
    return np.stack([V, ln_n, 2 * np.log(dev.ni) - ln_n], -1)


class _Device:
    """The GPU side of a batch: packed inputs uploaded once, a workspace reused."""

    def __init__(self, batch: Batch):
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("jaxdd_b200 needs a CUDA GPU (sm_100a); none is available")
        self.torch = torch
        dev = torch.device("cuda")
        self.stat = torch.from_numpy(batch["stat"]).to(dev)
        self.scal = torch.from_numpy(batch["scal"]).to(dev)
        self.iface = torch.from_numpy(batch["iface"]).to(dev)
        self.ws = None

    def workspace(self, desc) -> "object":
        size = ctypes.c_size_t(0)
        _lib.check(_lib.lib().dd_workspace_bytes(ctypes.byref(desc), ctypes.byref(size)),
                   "dd_workspace_bytes")
        if self.ws is None or self.ws.numel() < size.value:
            self.ws = self.torch.empty(size.value, dtype=self.torch.uint8, device="cuda")
        return self.ws


def _gpu(batch: Batch) -> _Device:
    if "_gpu" not in batch:
        batch["_gpu"] = _Device(batch)
    return batch["_gpu"]


def descriptor(batch: Batch, g, y0) -> _lib.DdBatch:
    return _lib.DdBatch(batch["n"], batch["Bp"], batch["np_max"], batch["ka"], batch["kc"],
                        g.stat.data_ptr(), g.scal.data_ptr(), g.iface.data_ptr(), y0.data_ptr())


def run(batch: Batch, volts_lane: list[np.ndarray], firsts: np.ndarray, *, tol: float,
        max_iter: int, start_iter: int, strict: bool, bernoulli_name: str, mode: int,
        precision: str = "fp64", jv_start: bool = False, sync: bool = True,
        tune: bool = False):
    """Launch the solve on the packed batch. `volts_lane[k]`: device k's voltages in the order
    the kernel takes them; `firsts[k]`: its start voltage. Returns device tensors
    (J, ok, its, status) in lane order and the flat offsets. `tune`: through the autotuner
    (`dd_tune`, every launch form timed once), its choice left in `batch["_tuned"]`."""
    import torch
    g = _gpu(batch)
    B, Bp, npmax = batch["n"], batch["Bp"], batch["np_max"]
    lane_of = batch["lane_of"]
    y0 = np.zeros((npmax + 2, 3, Bp))
    counts = np.zeros(Bp, dtype=np.int32)
    for k, dev in enumerate(batch["devices"]):
        lane = lane_of[k]
        NP = len(dev.x) - 2
        y0[:NP + 2, :, lane] = initial_state(dev, float(firsts[k]), jv=jv_start)
        counts[lane] = len(volts_lane[k])
    offsets = np.zeros(Bp, dtype=np.int32)
    offsets[1:] = np.cumsum(counts)[:-1]
    flat = np.zeros(max(int(counts.sum()), 1))
    for k in range(B):
        lane = lane_of[k]
        flat[offsets[lane]:offsets[lane] + counts[lane]] = volts_lane[k]
    dev = torch.device("cuda")
    t_y0 = torch.from_numpy(y0).to(dev)
    t_v = torch.from_numpy(flat).to(dev)
    t_off = torch.from_numpy(offsets).to(dev)
    t_cnt = torch.from_numpy(counts).to(dev)
    nflat = flat.size
    J = torch.full((nflat,), float("nan"), dtype=torch.float64, device=dev)
    ok = torch.zeros(nflat, dtype=torch.uint8, device=dev)
    its = torch.zeros(nflat, dtype=torch.int32, device=dev)
    status = torch.zeros(Bp, dtype=torch.int32, device=dev)
    steps = torch.zeros((3, Bp), dtype=torch.int32, device=dev)
    desc = descriptor(batch, g, t_y0)
    volts = _lib.DdVoltages(t_v.data_ptr(), t_off.data_ptr(), t_cnt.data_ptr())
    opts = _lib.DdOpts(float(tol), int(max_iter), int(start_iter), int(bool(strict)),
                       _lib.DD_BERNOULLI[bernoulli_name], mode, _lib.DD_PRECISION[precision], 0)
    ws = g.workspace(desc)
    stream = torch.cuda.current_stream().cuda_stream
    outs = (J.data_ptr(), ok.data_ptr(), its.data_ptr(), status.data_ptr(), steps.data_ptr(),
            ws.data_ptr(), ws.numel(), stream)
    if tune:
        form = ctypes.c_int32(-1)
        times = (ctypes.c_float * _lib.DD_SOLVE_FORMS)()
        _lib.check(_lib.lib().dd_tune(ctypes.byref(desc), ctypes.byref(volts), ctypes.byref(opts),
                                      *outs, ctypes.byref(form), times), "dd_tune")
        batch["_tuned"] = dict(_lib.SOLVE_FORMS[form.value], form=form.value,
                               times_ms=[float(t) for t in times])
    else:
        _lib.check(_lib.lib().dd_solve(ctypes.byref(desc), ctypes.byref(volts),
                                       ctypes.byref(opts), *outs), "dd_solve")
    batch["_last_steps"] = steps
    if sync:
        torch.cuda.synchronize()
    return J, ok, its, status, offsets, counts


def solve_batch(batch: Batch, voltages, tol: float = 1e-10, max_iter: int = 60,
                first_max_iter: int | None = 6, bernoulli_name: str = "exact",
                strict: bool = False, devices=None, precision: str = "fp64"):
    """J-V curves of a batch at `voltages` (internal, V): `(J, converged, iterations)`, each
    devices x voltages in the order of `voltages`, J with the shunt's current (jaxdd
    batch.py:1136-1162).

    Each device's scan runs outwards from its pre-bias (up, then down from the pre-bias solution
    again), each voltage started from the last two converged solutions extrapolated. jaxdd runs
    two passes, `first_max_iter` steps per voltage and then the devices that missed it with
    `max_iter`, to keep its lockstep batch cheap; its results are those of one pass at
    `max_iter`, which is what the kernel runs (every lane advances on its own).
    `devices` (jaxdd's accelerators to split across) is accepted for compatibility; the solve
    runs on the current CUDA device."""
    del first_max_iter, devices
    voltages = np.asarray(voltages, dtype=float).reshape(-1)
    order = np.argsort(voltages, kind="stable")
    inv = np.argsort(order, kind="stable")
    vs = voltages[order]
    devs = batch["devices"]
    firsts = np.array([d.V_pre if d.pre_cond else vs[0] for d in devs])
    J, ok, its, status, offsets, counts = run(
        batch, [vs] * len(devs), firsts, tol=tol, max_iter=max_iter, start_iter=max_iter,
        strict=strict, bernoulli_name=bernoulli_name, mode=_lib.DD_MODE_BATCH,
        precision=precision)
    return _gather(batch, J, ok, its, offsets, len(vs), inv)


def tune(batch: Batch, voltages, tol: float = 1e-10, max_iter: int = 60,
         bernoulli_name: str = "exact") -> dict:
    """Time every launch form of the solve on this batch at `voltages` (`dd_tune`) and keep the
    fastest for later solves of batches of its shape in this process: `{"form", "block",
    "queue", "times_ms"}`. `voltages` one list for every device, or one list per device (as
    `solve_uneven` takes them)."""
    devs = batch["devices"]
    if len(voltages) == len(devs) and np.ndim(voltages[0]) == 1:
        lists = [np.sort(np.asarray(v, dtype=float).reshape(-1)) for v in voltages]
    else:
        lists = [np.sort(np.asarray(voltages, dtype=float).reshape(-1))] * len(devs)
    firsts = np.array([d.V_pre if d.pre_cond else v[0] for d, v in zip(devs, lists)])
    run(batch, lists, firsts, tol=tol, max_iter=max_iter, start_iter=max_iter, strict=False,
        bernoulli_name=bernoulli_name, mode=_lib.DD_MODE_BATCH, tune=True)
    return batch.pop("_tuned")


def solve_uneven(batch: Batch, voltages: list, tol: float = 1e-10, max_iter: int = 60,
                 bernoulli_name: str = "exact", strict: bool = False):
    """`solve_batch` with a voltage list of its own for every device (`voltages[k]`, any
    length), in one launch; with `prepare(..., ragged=True)` the devices' grid sizes may differ
    too. jaxdd needs one `prepare` and one `solve_batch` per (grid size, voltage list)
    (batch.py:151-155, 1136-1162) and gets the same curves that way. Returns one
    `(J, converged, iterations)` per device, each in the order of its voltages."""
    devs = batch["devices"]
    if len(voltages) != len(devs):
        raise ValueError(f"{len(voltages)} voltage lists for {len(devs)} devices")
    lists = [np.asarray(v, dtype=float).reshape(-1) for v in voltages]
    if any(v.size == 0 for v in lists):
        raise ValueError("every device needs at least one voltage")
    orders = [np.argsort(v, kind="stable") for v in lists]
    firsts = np.array([d.V_pre if d.pre_cond else v[o[0]]
                       for d, v, o in zip(devs, lists, orders)])
    J, ok, its, status, offsets, counts = run(
        batch, [v[o] for v, o in zip(lists, orders)], firsts, tol=tol, max_iter=max_iter,
        start_iter=max_iter, strict=strict, bernoulli_name=bernoulli_name,
        mode=_lib.DD_MODE_BATCH)
    J, ok, its = J.cpu().numpy(), ok.cpu().numpy().astype(bool), its.cpu().numpy()
    out = []
    for k, (v, o) in enumerate(zip(lists, orders)):
        at = offsets[batch["lane_of"][k]] + np.argsort(o, kind="stable")
        out.append((J[at], ok[at], its[at]))
    return out


def solve_states(batch: Batch, voltages=0.0, tol: float = 1e-10, max_iter: int = 60,
                 first_max_iter: int | None = 6, bernoulli_name: str = "exact",
                 strict: bool = False, devices=None) -> dict:
    """The steady states of a batch at `voltages` (one or several, internal) and what
    photoluminescence measures of them (jaxdd batch.py:1165-1191): a dict of `V`, `n`, `p`,
    `qfls`, `anion`, `cation` (devices x voltages x NP + 2), `implied_voc`, `plqy`, `J`,
    `converged`, `iterations` (devices x voltages), in the order of `voltages`. Solved as
    `solve_batch` (one pass at `max_iter`, which gives jaxdd's two passes' results); the
    states are the checkpoints of `dd_solve_states`, the profiles and measures those of
    `dd_observables`. One grid size per batch, as jaxdd's `prepare` has it."""
    from .adjoint import plan as _plan
    from .adjoint import solve_states as _solve_states
    del first_max_iter, devices
    if len(set(int(n) for n in batch["NP"])) != 1:
        raise ValueError("solve_states needs one grid size (prepare without ragged)")
    voltages = np.atleast_1d(np.asarray(voltages, dtype=float)).reshape(-1)
    order = np.argsort(voltages, kind="stable")
    inv = np.argsort(order, kind="stable")
    vs = voltages[order]
    p = _plan(batch, vs, tol=tol, max_iter=max_iter, bernoulli_name=bernoulli_name,
              strict=strict)
    g = _gpu(batch)
    J, ok, its, ckpt = _solve_states(p, g.stat, g.scal, g.iface)
    prof, meas = observables(batch, p, ckpt)
    lanes = batch["lane_of"]
    offsets = p.offsets.cpu().numpy()
    Jd, okd, itd = _gather(batch, J, ok, its, offsets, p.nv_max, inv)
    out = {k: np.transpose(v.cpu().numpy()[:, :, lanes], (2, 0, 1))[:, inv]
           for k, v in prof.items()}
    out.update({k: v.cpu().numpy()[:, lanes].T[:, inv] for k, v in meas.items()})
    out.update({"J": Jd, "converged": okd, "iterations": itd})
    return out


def observables(batch: Batch, p, ckpt) -> tuple[dict, dict]:
    """`dd_observables` of the checkpoints `ckpt` that `dd_solve_states` wrote for the plan `p`
    (`adjoint.Plan`): the profiles `V`, `n`, `p`, `qfls`, `anion`, `cation` (voltages x NP + 2 x
    lanes) and the measures `implied_voc`, `plqy` (voltages x lanes), device tensors in lane
    order, the stream synchronised."""
    import torch
    g = _gpu(batch)
    nv, nodes, Bp = p.nv_max, batch["np_max"] + 2, batch["Bp"]
    cuda = p.v.device
    prof = {k: torch.empty((nv, nodes, Bp), dtype=torch.float64, device=cuda)
            for k in ("V", "n", "p", "qfls", "anion", "cation")}
    meas = {k: torch.empty((nv, Bp), dtype=torch.float64, device=cuda)
            for k in ("implied_voc", "plqy")}
    desc = descriptor(batch, g, p.y0)
    volts = _lib.DdVoltages(p.v.data_ptr(), p.offsets.data_ptr(), p.counts.data_ptr())
    _lib.check(_lib.lib().dd_observables(
        ctypes.byref(desc), ctypes.byref(volts), ckpt["states"].data_ptr(),
        ckpt["logs"].data_ptr(), ckpt["pre"].data_ptr(), ckpt["pre_logs"].data_ptr(), nv,
        *[prof[k].data_ptr() for k in ("V", "n", "p", "qfls", "anion", "cation")],
        meas["implied_voc"].data_ptr(), meas["plqy"].data_ptr(),
        torch.cuda.current_stream(cuda).cuda_stream), "dd_observables")
    torch.cuda.synchronize()
    return prof, meas


def _gather(batch, J, ok, its, offsets, nv, inv):
    J, ok, its = J.cpu().numpy(), ok.cpu().numpy().astype(bool), its.cpu().numpy()
    lanes = batch["lane_of"]
    idx = offsets[lanes][:, None] + np.arange(nv)[None, :]
    return J[idx][:, inv], ok[idx][:, inv], its[idx][:, inv]


def external_voltages(batch: Batch, voltages, J):
    """`V_ext = V_int + J·R_series` (jaxdd batch.py:1104-1108)."""
    return np.asarray(voltages)[None, :] + np.asarray(J) * batch["R_series"][:, None]
