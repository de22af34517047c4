"""Device building on the GPU for parameter sweeps.

jaxdd builds the devices of a sweep in JAX on the accelerator (`batch.device_tree(structure,
params)`, batch.py:142-148, over `device.device_arrays`, device.py:877-1063): the grid's
structure (points per layer) is fixed by one setup, and each device's parameters only scale the
spacings and fill the arrays. Here `SweepStructure(setup)` is that structure on the GPU,
`parameters(setups)` the per-layer and per-device parameter tables of many setups of the same
stack, and `build(...)` runs `dd_build` to write the packed record (and each device's start
state) on the GPU; `solve_sweep` solves them without a host-side `Device` per device. The host
builder (`device.build_device`) builds one device in milliseconds; a batch of thousands would
keep the GPU waiting (jaxdd docs/batching.md:64-66 estimates 1800 devices/s are needed to feed an
A100).
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .batch import prepare
from .device import build_device, grid_layout
from .simss_input import Setup


class SweepStructure:
    """The structure all devices of a sweep share, from one reference setup: the grid's layout,
    the layers' ion slots and fixed ions, the trapped joins and their trap types, which contacts
    are flat-band, the record's interface index and the twisted sweep's meeting row."""

    def __init__(self, setup: Setup, grid: str = "graded", grid_split: str = "exact"):
        import torch
        self.setup = setup
        self.layout = grid_layout(setup, grid, grid_split)
        dev = build_device(setup, grid=grid, grid_split=grid_split, layout=self.layout)
        b = prepare([dev])
        self.NP = len(dev.x) - 2
        layers = setup.layers
        self.n_layers = len(layers)
        if self.n_layers > _lib.DD_MAXLAYERS:
            raise NotImplementedError(f"{self.n_layers} layers: at most {_lib.DD_MAXLAYERS}")
        if setup.raw.get("genProfile", "none").strip().lower() != "none":
            raise NotImplementedError("a generation profile from a file: built on the host only")
        S, C = _lib.S, _lib.C
        col = b["stat"][:, :, 0]
        lay = self.layout
        self.ka, self.kc = b["ka"], b["kc"]
        aslot = np.array([col[lay.i0[j] + (1 if j == 0 else 0), S["ASLOT"]]
                          for j in range(self.n_layers)])
        cslot = np.array([col[lay.i0[j] + (1 if j == 0 else 0), S["CSLOT"]]
                          for j in range(self.n_layers)])
        held = bool(setup.i("fixIons", 0)) and not bool(setup.i("preCond", 0))
        conc = {sp: np.array([ly.f(f"N_{sp}") for ly in layers]) for sp in ("anion", "cation")}
        mob = {sp: np.array([ly.f(f"mu_{sp}") for ly in layers]) for sp in ("anion", "cation")}
        afixed = ((conc["anion"] != 0) & ((mob["anion"] == 0) | held)).astype(np.uint8)
        cfixed = ((conc["cation"] != 0) & ((mob["cation"] == 0) | held)).astype(np.uint8)
        row = np.full(self.n_layers, -1, dtype=np.int32)
        kind = np.zeros(self.n_layers)
        if dev.interface is not None:
            edges = list(np.flatnonzero(np.asarray(dev.interface["Nt"]) > 0))
            for j in range(self.n_layers - 1):
                if lay.i1[j] in edges:
                    row[j] = edges.index(lay.i1[j])
                    kind[j] = float(layers[j].raw.get("intTrapType", "0"))
        at_iface = np.zeros(self.NP + 2, dtype=np.uint8)
        at_iface[list(lay.i1[:-1])] = 1
        self.sfb = [setup.raw[k].strip().lower() == "sfb" for k in ("W_L", "W_R")]
        sc = b["scal"][:, 0]
        cuda = torch.device("cuda")
        self._keep = {
            "lid": torch.as_tensor(lay.lid.astype(np.int32), device=cuda),
            "raw": torch.as_tensor(lay.raw, device=cuda),
            "norm": torch.as_tensor(lay.norm, device=cuda),
            "i0": torch.as_tensor(np.array(lay.i0, np.int32), device=cuda),
            "i1": torch.as_tensor(np.array(lay.i1, np.int32), device=cuda),
            "at_iface": torch.as_tensor(at_iface, device=cuda),
            "ifk": torch.as_tensor(np.ascontiguousarray(col[:, S["IFK"]]), device=cuda),
            "aslot": torch.as_tensor(aslot, device=cuda),
            "cslot": torch.as_tensor(cslot, device=cuda),
            "afixed": torch.as_tensor(afixed, device=cuda),
            "cfixed": torch.as_tensor(cfixed, device=cuda),
            "iface_row": torch.as_tensor(row, device=cuda),
            "iface_kind": torch.as_tensor(kind, device=cuda),
        }
        k = self._keep
        self.c_struct = _lib.DdStructure(
            self.NP, self.n_layers, *[k[n].data_ptr() for n in (
                "lid", "raw", "norm", "i0", "i1", "at_iface", "ifk", "aslot", "cslot", "afixed",
                "cfixed", "iface_row", "iface_kind")],
            int(self.sfb[0]), int(self.sfb[1]), float(sc[C["LEFT"]]), float(sc[C["PRECOND"]]),
            float(sc[C["FIXIONS"]]), float(sc[C["CURRDIFF"]]), float(sc[C["MID"]]))

    def check(self, setup: Setup) -> None:
        """`ValueError` unless `setup` is a device of this structure: the same grid size and
        layers, contacts, ion pattern, trapped joins and pre-bias."""
        ref = self.setup
        same = (setup.i("NP") == ref.i("NP") and len(setup.layers) == len(ref.layers)
                and [setup.raw[k].strip().lower() == "sfb" for k in ("W_L", "W_R")] == self.sfb
                and setup.i("preCond", 0) == ref.i("preCond", 0)
                and setup.i("fixIons", 0) == ref.i("fixIons", 0)
                and setup.i("leftElec") == ref.i("leftElec"))
        for a, b in zip(setup.layers, ref.layers):
            for key in ("mu_anion", "mu_cation", "N_anion", "N_cation", "N_t_int"):
                same = same and ((a.f(key) != 0) == (b.f(key) != 0))
            same = same and a.i("ionsMayEnter") == b.i("ionsMayEnter")
        if not same:
            raise ValueError("a setup of another structure than the sweep's")


def parameters(structure: SweepStructure, setups: list[Setup], first=None):
    """The parameter tables of `setups` (each checked against the structure):
    `(layer_params [layers][DD_LF][n], device_params [DD_DF][n])`; `first` the voltage each
    device's start state is for (the pre-bias where there is one; default 0 V)."""
    n = len(setups)
    P = np.zeros((structure.n_layers, len(_lib.LAYER_FIELDS), n))
    D = np.zeros((len(_lib.DEVICE_FIELDS), n))
    for k, s in enumerate(setups):
        structure.check(s)
        for j, ly in enumerate(s.layers):
            for f, name in enumerate(_lib.LAYER_FIELDS):
                P[j, f, k] = float(ly.raw.get(name, "0"))
        D[0, k] = s.f("T")
        D[1, k] = 0.0 if structure.sfb[0] else s.f("W_L")
        D[2, k] = 0.0 if structure.sfb[1] else s.f("W_R")
        D[3, k] = s.f("G_frac", 1.0)
        D[4, k] = float(s.raw.get("R_shunt", "-1"))
        D[5, k] = s.f("Vpre", 0.0)
        pre = bool(s.i("preCond", 0))
        D[6, k] = D[5, k] if pre else (0.0 if first is None else float(np.atleast_1d(first)[k]))
    return P, D


def build(structure: SweepStructure, P: np.ndarray, D: np.ndarray, stream=None):
    """`dd_build` on the GPU: `(stat, scal, iface, y0, lane_stride)` torch tensors of the devices
    in lanes 0..n-1."""
    import torch
    n = P.shape[-1]
    Bp = (n + 31) // 32 * 32
    nodes = structure.NP + 2
    cuda = torch.device("cuda")
    tP = torch.as_tensor(np.ascontiguousarray(P), device=cuda)
    tD = torch.as_tensor(np.ascontiguousarray(D), device=cuda)
    stat = torch.zeros((nodes, _lib.DD_NF, Bp), dtype=torch.float64, device=cuda)
    stat[:, _lib.S["ASLOT"]] = -1.0
    stat[:, _lib.S["CSLOT"]] = -1.0
    stat[:, _lib.S["IFK"]] = -2.0
    stat[:, _lib.S["SP"]] = 1.0
    stat[:, _lib.S["SC"]] = 1.0
    scal = torch.zeros((_lib.DD_NS_BASE + _lib.DD_MAXK, Bp), dtype=torch.float64, device=cuda)
    iface = torch.zeros((_lib.DD_MAXIF, _lib.DD_NIF, Bp), dtype=torch.float64, device=cuda)
    y0 = torch.zeros((nodes, 3, Bp), dtype=torch.float64, device=cuda)
    ws = torch.empty(nodes * n, dtype=torch.float64, device=cuda)
    s = stream if stream is not None else torch.cuda.current_stream(cuda).cuda_stream
    _lib.check(_lib.lib().dd_build(
        ctypes.byref(structure.c_struct), tP.data_ptr(), tD.data_ptr(), n, Bp, structure.ka,
        structure.kc, stat.data_ptr(), scal.data_ptr(), iface.data_ptr(), y0.data_ptr(),
        ws.data_ptr(), ws.numel() * 8, s), "dd_build")
    return stat, scal, iface, y0, Bp


def solve_sweep(structure: SweepStructure, setups: list[Setup], voltages, tol: float = 1e-10,
                max_iter: int = 60, bernoulli_name: str = "exact"):
    """The J-V curves of the sweep's devices at `voltages` (internal, V), built and solved on the
    GPU: `(J, converged, iterations)`, devices x voltages in the order of `voltages`, the shunt's
    current added (`solve_batch`'s results for the same devices)."""
    import torch
    voltages = np.asarray(voltages, dtype=float).reshape(-1)
    order = np.argsort(voltages, kind="stable")
    inv = np.argsort(order, kind="stable")
    vs = voltages[order]
    n = len(setups)
    P, D = parameters(structure, setups, first=np.full(n, vs[0]))
    stat, scal, iface, y0, Bp = build(structure, P, D)
    cuda = stat.device
    nv = len(vs)
    counts = np.zeros(Bp, dtype=np.int32)
    counts[:n] = nv
    offsets = (np.arange(Bp) * nv).astype(np.int32)
    tv = torch.as_tensor(np.tile(vs, Bp), device=cuda)
    toff = torch.as_tensor(offsets, device=cuda)
    tcnt = torch.as_tensor(counts, device=cuda)
    J = torch.empty(Bp * nv, dtype=torch.float64, device=cuda)
    ok = torch.empty(Bp * nv, dtype=torch.uint8, device=cuda)
    its = torch.empty(Bp * nv, dtype=torch.int32, device=cuda)
    status = torch.empty(Bp, dtype=torch.int32, device=cuda)
    desc = _lib.DdBatch(n, Bp, structure.NP, structure.ka, structure.kc, stat.data_ptr(),
                        scal.data_ptr(), iface.data_ptr(), y0.data_ptr())
    volts = _lib.DdVoltages(tv.data_ptr(), toff.data_ptr(), tcnt.data_ptr())
    opts = _lib.DdOpts(float(tol), int(max_iter), int(max_iter), 0,
                       _lib.DD_BERNOULLI[bernoulli_name], _lib.DD_MODE_BATCH, 0, 0)
    size = ctypes.c_size_t(0)
    so = _lib.lib()
    _lib.check(so.dd_workspace_bytes(ctypes.byref(desc), ctypes.byref(size)), "dd_workspace_bytes")
    ws = torch.empty(size.value, dtype=torch.uint8, device=cuda)
    _lib.check(so.dd_solve(ctypes.byref(desc), ctypes.byref(volts), ctypes.byref(opts),
                           J.data_ptr(), ok.data_ptr(), its.data_ptr(), status.data_ptr(), None,
                           ws.data_ptr(), ws.numel(), torch.cuda.current_stream(cuda).cuda_stream),
               "dd_solve")
    J = J.cpu().numpy().reshape(Bp, nv)[:n][:, inv]
    ok = ok.cpu().numpy().reshape(Bp, nv)[:n][:, inv].astype(bool)
    its = its.cpu().numpy().reshape(Bp, nv)[:n][:, inv]
    return J, ok, its
