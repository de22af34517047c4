"""Parameter gradients of J-V misfits: the adjoint workload (14 log-parameters per device).

jaxdd fits device parameters by differentiating its solve: it builds a device in JAX from its
parameters (`batch.device_tree`, batch.py:142-148, over `device.device_arrays`, device.py:877-1063,
with the grid's structure held fixed) and differentiates `solve_batch` through the custom JVP of
its converged solutions (validation/fit.py:92-108). Here the same chain runs as
parameters -> packed record (`records`, torch, differentiable) -> curves (`adjoint.curves`, the
CUDA solve, backward by the adjoint kernel) -> loss.

The parameters (`PARAMS`), each in its logarithm: the absorber's electron and hole mobilities, the
hole transport layer's mobility (both carriers), the absorber's bulk trap density, the interface
trap density (both interfaces), the three thicknesses, the two work functions, the absorber's ion
density (anions = cations), its generation rate, and the transport layers' doping (N_A of the
HTL, N_D of the ETL). `records` restates, for these inputs, the formulas of the device builder
(`device.build_device`) and the packer (`batch._pack_one`); the tests check it against them.
"""

from __future__ import annotations

import numpy as np

from . import _lib
from .batch import prepare
from .constants import EPS_0, K_B, Q
from .device import build_device, grid_layout
from .simss_input import setup_from_texts

#: (name, file, keys): each parameter's logarithm sets every key in its file
PARAMS = (
    ("mu_n_absorber", "L2.txt", ("mu_n",)),
    ("mu_p_absorber", "L2.txt", ("mu_p",)),
    ("mu_htl", "L1.txt", ("mu_n", "mu_p")),
    ("N_t_bulk", "L2.txt", ("N_t_bulk",)),
    ("N_t_interface", ("L1.txt", "L2.txt"), ("N_t_int",)),
    ("L_htl", "L1.txt", ("L",)),
    ("L_absorber", "L2.txt", ("L",)),
    ("L_etl", "L3.txt", ("L",)),
    ("W_L", "simulation_setup.txt", ("W_L",)),
    ("W_R", "simulation_setup.txt", ("W_R",)),
    ("N_ion", "L2.txt", ("N_anion", "N_cation")),
    ("G", "L2.txt", ("G_ehp",)),
    ("N_A_htl", "L1.txt", ("N_A",)),
    ("N_D_etl", "L3.txt", ("N_D",)),
)
NAMES = tuple(p[0] for p in PARAMS)
#: seed of the target curves' parameter perturbation
SEED_TARGET = 20261204
TARGET_SIGMA = 0.2


def _files(spec):
    return spec if isinstance(spec, tuple) else (spec,)


def _get(text: str, key: str) -> str:
    for line in text.splitlines():
        k, _, v = line.partition("=")
        if k.strip() == key:
            return v.split("*")[0].strip()
    raise KeyError(key)


def _set(text: str, key: str, value: float) -> str:
    out = []
    for line in text.splitlines():
        k, _, _ = line.partition("=")
        out.append(f"{key} = {value!r}" if k.strip() == key else line)
    return "\n".join(out) + "\n"


def theta_of(texts: dict) -> np.ndarray:
    """A device's parameters (logarithms) from its input texts."""
    return np.array([np.log(float(_get(texts[_files(f)[0]], keys[0])))
                     for _, f, keys in PARAMS])


def texts_with(texts: dict, theta) -> dict:
    """The input texts with the parameters set to `exp(theta)` (written exactly)."""
    out = dict(texts)
    for (_, f, keys), t in zip(PARAMS, theta):
        for name in _files(f):
            for key in keys:
                out[name] = _set(out[name], key, float(np.exp(t)))
    return out


def fit_texts(k: int, seed: int = 20261203, NP: int = 400) -> dict:
    """Device `k` of the adjoint workload: the drawn stack (its distributions and pre-bias
    pattern) with both interfaces' traps of one density and the contacts' work functions given
    as numbers (each the flat-band value of its layer's drawn doping), so that every parameter of
    `PARAMS` is an input of the device."""
    from .workloads import drawn_texts
    rng = np.random.default_rng([seed, k])
    texts = drawn_texts(k, rng, NP)
    nti = float(_get(texts["L1.txt"], "N_t_int"))
    texts["L2.txt"] = _set(texts["L2.txt"], "N_t_int", nti)
    Vt = K_B * 300.0 / Q
    NA, ND = float(_get(texts["L1.txt"], "N_A")), float(_get(texts["L3.txt"], "N_D"))
    W_L = float(5.6 - Vt * np.log(2.2e24 / NA))
    W_R = float(4.0 + Vt * np.log(2.2e24 / ND))
    s = texts["simulation_setup.txt"]
    s = s.replace("W_L = sfb", f"W_L = {W_L!r}").replace("W_R = sfb", f"W_R = {W_R!r}")
    texts["simulation_setup.txt"] = s
    return texts


def flat_band(theta: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """The contacts' flat-band work functions of the parameters' doping (`fit_texts`'s)."""
    Vt = K_B * 300.0 / Q
    NA, ND = np.exp(theta[..., NAMES.index("N_A_htl")]), np.exp(theta[..., NAMES.index("N_D_etl")])
    return 5.6 - Vt * np.log(2.2e24 / NA), 4.0 + Vt * np.log(2.2e24 / ND)


def target_theta(theta: np.ndarray, seed: int = SEED_TARGET, sigma: float = TARGET_SIGMA,
                 start: int = 0) -> np.ndarray:
    """The target curves' parameters: each device's, every factor times exp(sigma N(0, 1)) (device
    `start + k` drawing from its own stream) — but the work functions, which a 20 % factor would
    put outside their layers' gaps: those are the flat-band values of the target's doping."""
    out = np.array(theta, dtype=float, copy=True)
    for k in range(out.shape[0]):
        out[k] += sigma * np.random.default_rng([seed, start + k]).standard_normal(out.shape[1])
    W_L, W_R = flat_band(out)
    out[:, NAMES.index("W_L")] = np.log(W_L)
    out[:, NAMES.index("W_R")] = np.log(W_R)
    return out


class Structure:
    """What `records` holds fixed: the devices' grids (points per layer, unscaled spacings), the
    layers' constants and the packed record at the reference parameters, on the GPU."""

    def __init__(self, texts: list[dict], theta0: np.ndarray | None = None, device=None):
        import torch
        self.texts = texts
        setups = [setup_from_texts(t) for t in texts]
        self.layouts = [grid_layout(s) for s in setups]
        self.theta0 = np.stack([theta_of(t) for t in texts]) if theta0 is None else theta0
        devs = [build_device(setup_from_texts(texts_with(t, th)), layout=lay)
                for t, th, lay in zip(texts, self.theta0, self.layouts)]
        self.batch = prepare(devs)
        b = self.batch
        NPs = {len(d.x) - 2 for d in devs}
        if len(NPs) != 1:
            raise ValueError("the adjoint workload needs one grid size")
        self.NP = NPs.pop()
        n = len(devs)
        cuda = torch.device(device or ("cuda" if torch.cuda.is_available() else "cpu"))
        self.device = cuda
        f64 = dict(dtype=torch.float64, device=cuda)
        self.lanes = torch.as_tensor(b["lane_of"], device=cuda)
        self.stat0 = torch.from_numpy(b["stat"]).to(cuda)
        self.scal0 = torch.from_numpy(b["scal"]).to(cuda)
        self.iface0 = torch.from_numpy(b["iface"]).to(cuda)
        lid = np.stack([lay.lid for lay in self.layouts])
        self.lid = torch.as_tensor(lid, device=cuda)
        self.raw = torch.as_tensor(np.stack([lay.raw for lay in self.layouts]), **f64)
        self.norm = torch.as_tensor(np.stack([lay.norm for lay in self.layouts]), **f64)
        self.joins = torch.as_tensor(np.stack([lay.i0[1:] for lay in self.layouts]), device=cuda)
        ends = np.stack([lay.i1[:-1] for lay in self.layouts])
        at_iface = np.zeros(lid.shape, dtype=bool)
        np.put_along_axis(at_iface, ends, True, axis=1)
        self.at_iface = torch.as_tensor(at_iface, device=cuda)
        layer = {key: np.array([[float(_get(t[f"L{j + 1}.txt"], key)) for j in range(3)]
                                for t in texts])
                 for key in ("eps_r", "E_c", "E_v", "N_c", "nu_int_n", "nu_int_p", "mu_n",
                             "mu_p")}
        self.layer = {k: torch.as_tensor(v, **f64) for k, v in layer.items()}
        self.Vt = torch.as_tensor(np.array([d.Vt for d in devs]), **f64)
        # where the parameters act: bulk traps, generation, interface rows and their edges
        S, I = _lib.S, _lib.I
        st = b["stat"][:, :, b["lane_of"]]  # nodes x fields x devices
        self.trap = torch.as_tensor(st[:, S["NT"], :].T > 0, device=cuda)
        self.gen = torch.as_tensor(st[:, S["G"], :].T > 0, device=cuda)
        ifk = st[:, S["IFK"], :].T  # devices x nodes
        rows = b["iface"][:, I["NT"], :][:, b["lane_of"]].T > 0  # devices x rows
        edge = np.zeros(rows.shape, dtype=np.int64)
        for k in range(n):
            for r in range(rows.shape[1]):
                hit = np.flatnonzero(ifk[k] == r)
                edge[k, r] = hit[0] if len(hit) else 1
        self.rows = torch.as_tensor(rows, device=cuda)
        self.row_edge = torch.as_tensor(edge, device=cuda)
        self.n = n


def _smooth(h, joins):
    """`_scaled`'s three spacings around each layer join set to their mean."""
    import torch
    for j in range(joins.shape[1]):
        idx = joins[:, j:j + 1] + torch.tensor([0, -1, -2], device=h.device)[None, :]
        three = torch.gather(h, 1, idx)
        mean = (three[:, 0] + three[:, 1] + three[:, 2]) / 3.0
        h = h.scatter(1, idx, mean[:, None].expand(-1, 3))
    return h


def records(theta, st: Structure):
    """The packed record `(stat, scal, iface)` of the devices at the parameters `theta`
    (devices x 14, torch float64 on the GPU), differentiable in `theta`; every other input as
    at `st.theta0`."""
    import torch
    S, C, I = _lib.S, _lib.C, _lib.I
    e = torch.exp(theta)
    Ls = e[:, 5:8]
    total = Ls.sum(1)
    lid = st.lid
    layer = st.layer
    h = st.raw * torch.gather(Ls, 1, lid) / (total[:, None] * torch.gather(st.norm, 1, lid))
    h = _smooth(h, st.joins)
    NP = st.NP
    Vt = st.Vt

    def per_layer(values):  # devices x 3 -> devices x nodes
        return torch.gather(values, 1, lid)

    eps = per_layer(layer["eps_r"]) * EPS_0
    Nc = per_layer(layer["N_c"])
    one = torch.ones_like(e[:, 0])
    mun_l = torch.stack([e[:, 2], e[:, 0], layer["mu_n"][:, 2]], 1)
    mup_l = torch.stack([e[:, 2], e[:, 1], layer["mu_p"][:, 2]], 1)
    at = st.at_iface
    th = total[:, None] * h
    mu_n = torch.where(at, th * per_layer(layer["nu_int_n"]) / Vt[:, None], per_layer(mun_l))
    mu_p = torch.where(at, th * per_layer(layer["nu_int_p"]) / Vt[:, None], per_layer(mup_l))
    i = torch.arange(1, NP + 1, device=theta.device)
    hm, hp = h[:, i - 1], h[:, i]
    w = hp + hm
    L2 = (total * total)[:, None]
    ei, em = eps[:, i], eps[:, i - 1]
    facu = 2 * ei / (hp * w * L2)
    facl = 2 * ei / (hm * w * L2) - (ei - em) / (hm ** 2 * L2)
    facm = (ei - em) / (hm ** 2 * L2) - 2 * ei * (1 / (hp * w * L2) + 1 / (hm * w * L2))
    fac = 0.5 * L2 * hp * hm * w
    sc = 1.0 / (torch.maximum(mu_n[:, i], mu_p[:, i]) * Vt[:, None] * Nc[:, i] * hp)
    NA_l = torch.stack([e[:, 12], 0 * one, 0 * one], 1)
    ND_l = torch.stack([0 * one, 0 * one, e[:, 13]], 1)
    dop = per_layer(NA_l - ND_l)[:, i]
    dx = torch.cat([th[:, :NP], torch.zeros_like(th[:, :2])], 1)
    Nt = torch.where(st.trap, e[:, 3:4].expand_as(h), torch.zeros_like(h))
    G = torch.where(st.gen, e[:, 11:12].expand_as(h), torch.zeros_like(h))

    def rows_of(v):  # devices x NP -> devices x nodes, zero at the contacts
        z = torch.zeros_like(v[:, :1])
        return torch.cat([z, v, z], 1)

    new = {S["MUN"]: mu_n, S["MUP"]: mu_p, S["H"]: h, S["DX"]: dx, S["FACL"]: rows_of(facl),
           S["FACM"]: rows_of(facm), S["FACU"]: rows_of(facu), S["FAC"]: rows_of(fac),
           S["SC"]: rows_of(sc), S["DOP"]: rows_of(dop), S["NT"]: Nt, S["G"]: G}
    lanes = st.lanes
    fields = []
    for f in range(_lib.DD_NF):
        col = st.stat0[:, f, :]
        if f in new:
            v = new[f].T  # nodes x devices
            if f == S["SC"]:  # the contacts' rows keep the packer's unit scale
                v = torch.cat([col[:1, lanes], v[1:NP + 1], col[NP + 1:, lanes]], 0)
            col = col.clone()
            col[:, lanes] = v
        fields.append(col)
    stat = torch.stack(fields, 1)
    # scalars
    W_L, W_R = e[:, 8], e[:, 9]
    Ec, Ev, Ncl = layer["E_c"], layer["E_v"], layer["N_c"]
    tot = Ls[:, 1] * e[:, 10]
    sv = {C["L"]: total, C["V0"]: 0.5 * (-W_L + W_R), C["VL"]: 0.5 * (W_L - W_R),
          C["LNNL"]: torch.log(Ncl[:, 0]) - (W_L - Ec[:, 0]) / Vt,
          C["LNPL"]: torch.log(Ncl[:, 0]) + (W_L - Ev[:, 0]) / Vt,
          C["LNNR"]: torch.log(Ncl[:, 2]) - (W_R - Ec[:, 2]) / Vt,
          C["LNPR"]: torch.log(Ncl[:, 2]) - (Ev[:, 2] - W_R) / Vt,
          C["HSUM"]: h[:, :NP + 1].sum(1),
          _lib.DD_NS_BASE: tot, _lib.DD_NS_BASE + st.batch["ka"]: tot}
    rows = []
    for f in range(st.scal0.shape[0]):
        r = st.scal0[f]
        if f in sv:
            r = r.clone()
            r[lanes] = sv[f]
        rows.append(r)
    scal = torch.stack(rows, 0)
    # interface table: the density and the inverse width of each trapped edge
    ed = st.row_edge
    hE = lambda off: torch.gather(h, 1, (ed + off).clamp(0, NP + 1))  # noqa: E731
    width = 0.5 * total[:, None] * (0.5 * hE(1) + hE(0) + 0.5 * hE(-1))
    iw = torch.where(st.rows, 1.0 / width, torch.zeros_like(width))
    ntr = torch.where(st.rows, e[:, 4:5].expand_as(width), torch.zeros_like(width))
    blocks = []
    for r in range(_lib.DD_MAXIF):
        fl = []
        for f in range(_lib.DD_NIF):
            col = st.iface0[r, f]
            if r < ntr.shape[1] and f in (I["NT"], I["IW"]):
                col = col.clone()
                col[lanes] = (ntr if f == I["NT"] else iw)[:, r]
            fl.append(col)
        blocks.append(torch.stack(fl, 0))
    iface = torch.stack(blocks, 0)
    return stat.contiguous(), scal.contiguous(), iface.contiguous()


def misfit(J, ok, target, scale):
    """jaxdd's fit residual (validation/fit.py:99-104) summed in squares: sum over the converged
    voltages of ((J - J_target) / scale)^2, `scale` each device's current scale at the
    reference parameters (held constant)."""
    import torch
    r = torch.where(ok > 0, (J - target) / scale[:, None], torch.zeros_like(J))
    return (r * r).sum()
