"""A SIMsalabim device on its grid: the static arrays the solver reads.

The drop-in for jaxdd's `build_device` (jaxdd src/jaxdd/device.py:1066-1079). The arrays follow
SIMsalabim 5.36's definitions as jaxdd states them (`Make_Grid`, `Define_Layers`,
`Init_Generation_Profile`, `Init_Trapping`, `Calc_Elec_Mob`), so that a device built here is the
reference's device to the bit: the tests compare every array with fixtures the reference's own
builder wrote.

The scope is the steady-state J-V path: Boltzmann carriers, bulk SRH traps through one neutral
level, interface traps (one level, neutral or charged), direct recombination, mobile ions in
regions (free, frozen after a pre-bias, or held), a generation profile from a file or uniform,
SIMsalabim's or jaxdd's graded grid, either form of the current, series and shunt resistance.
Inputs that need more (finite surface recombination, free ends, field-dependent mobility or
generation, Langevin, trap files, charged bulk traps, ion sites, Auger, other statistics,
transfer-matrix optics) are refused by name with `NotImplementedError`, never approximated.
"""

from __future__ import annotations

import io
from collections.abc import Sequence
from dataclasses import dataclass
from fractions import Fraction

import numpy as np

from .constants import EPS_0, K_B, Q
from .simss_input import Setup, ion_region_problems, ion_regions

__all__ = ["Device", "GRIDS", "GRID_SPLITS", "build_device", "layer_points", "make_grid"]

#: SIMsalabim's `MinGridPointsPerLayer`.
MIN_POINTS = 5
#: SimSS's `myReal` (x87 extended) carries a 64-bit significand.
_EXT_BITS = 64
GRID_SPLITS = ("exact", "simss")
GRIDS = ("simss", "graded")
#: jaxdd's graded grid: points per e-fold of the distance to a layer's end, and the distance (m)
#: at which the grading starts (jaxdd device.py:154-157).
GRADED_PER_EFOLD = 6.0
GRADED_SMALLEST = 3e-12


def _to_extended(q: Fraction) -> Fraction:
    """`q` rounded to the nearest value with a 64-bit significand, ties to even (the x87's
    default rounding, which SimSS's grid split goes through)."""
    if q == 0:
        return q
    neg = q < 0
    a = -q if neg else q
    e = a.numerator.bit_length() - a.denominator.bit_length()
    if a < Fraction(2) ** e:
        e -= 1
    unit = Fraction(2) ** (e - _EXT_BITS + 1)
    m = a / unit
    whole, frac = divmod(m.numerator, m.denominator)
    rem = Fraction(frac, m.denominator)
    if rem > Fraction(1, 2) or (rem == Fraction(1, 2) and whole % 2 == 1):
        whole += 1
    out = whole * unit
    return -out if neg else out


def layer_points(thicknesses: Sequence[str | float], NP: int, split: str = "exact") -> list[int]:
    """Each layer's points beyond its first on SIMsalabim's grid: at least `MIN_POINTS`, else
    `floor((NP − n_thin·MIN_POINTS)·L/(L_tot − L_thin))`, a layer thin where `NP·L/L_tot` is
    below `MIN_POINTS` (jaxdd device.py:66-94). `split` "exact" evaluates the share in rational
    arithmetic of the decimal inputs, "simss" rounds every operation to an extended value as
    SimSS does, which decides `floor` where the share is a whole number."""
    if split not in GRID_SPLITS:
        raise ValueError(f"split {split!r}: one of {GRID_SPLITS}")
    rnd = (lambda q: q) if split == "exact" else _to_extended
    vals = [rnd(Fraction(t if isinstance(t, str) else repr(float(t)))) for t in thicknesses]
    tot = Fraction(0)
    for v in vals:
        tot = rnd(tot + v)
    thin = [v for v in vals if rnd(rnd(NP * v) / tot) < MIN_POINTS]
    thin_tot = Fraction(0)
    for v in thin:
        thin_tot = rnd(thin_tot + v)
    avail = NP - MIN_POINTS * len(thin)
    rest = rnd(tot - thin_tot)
    out = []
    for v in vals:
        share = rnd(avail * rnd(v / rest))
        out.append(max(MIN_POINTS, share.numerator // share.denominator))
    return out


def _simss_sub_grid(m: int, grad: float) -> np.ndarray:
    """SIMsalabim's `Make_Sub_Grid` before scaling: `m + 1` exponentially graded spacings,
    mirrored about the layer's middle."""
    h = np.ones(m + 1)
    half = round(0.5 * m)
    for i in range(half + 1):
        h[i] = h[m - i] = np.exp(grad * (1.0 / half - 1.0 / (i + 1)))
    return h


@dataclass(frozen=True)
class _Layout:
    i0: list[int]
    i1: list[int]
    lid: np.ndarray
    raw: np.ndarray
    norm: np.ndarray


def _fill_layout(counts, NP, spacings) -> _Layout:
    """Lay the layers' point counts out on the `NP + 2` grid; `spacings(k, m)` gives layer `k`'s
    `m` unscaled spacings (the last layer runs to the grid's last point)."""
    n = len(counts)
    raw = np.zeros(NP + 2)
    norm = np.zeros(n)
    lid = np.zeros(NP + 2, dtype=int)
    i0, i1 = [], []
    a = 0
    for k in range(n):
        b = a + int(counts[k])
        i0.append(a)
        i1.append(b)
        if k == n - 1:
            b = NP + 1
        raw[a:b + 1] = spacings(k, b - a + 1)
        norm[k] = raw[a:b + 1].sum()
        lid[a:b + 1] = k
        a = b + 1
    i1[-1] = NP + 1
    return _Layout(i0, i1, lid, raw, norm)


def _simss_layout(thicknesses, NP, grad, split) -> _Layout:
    counts = layer_points(thicknesses, NP, split)
    return _fill_layout(counts, NP, lambda k, m: _simss_sub_grid(m - 1, grad))


def _graded_layout(thicknesses, NP, beta=GRADED_PER_EFOLD, d0=GRADED_SMALLEST) -> _Layout:
    """jaxdd's graded grid (jaxdd device.py:171-214): point density `1/H + β/(d + d0)` from
    each layer end, `H` the mean spacing; each layer gets its share of the density's integral
    (at least `MIN_POINTS`), and its points equidistribute that integral (bisection)."""
    Ls = np.array([float(t) for t in thicknesses])
    H = Ls.sum() / NP
    n = len(Ls)

    def cumulative(x, Lk):
        return x / H + beta * (np.log1p(x / d0) + np.log1p(Lk / d0) - np.log1p((Lk - x) / d0))

    weight = np.array([cumulative(Lk, Lk) for Lk in Ls])
    counts = np.maximum(MIN_POINTS, np.floor((NP + 2 - n) * weight / weight.sum()).astype(int))
    over = int(counts.sum()) + n - (NP + 2)
    if over > 0:
        counts[np.argmax(counts)] -= over

    def spacings(k, m):
        Lk = Ls[k]
        goal = np.arange(m + 1) * weight[k] / m
        lo, hi = np.zeros(m + 1), np.full(m + 1, Lk)
        for _ in range(100):
            mid = 0.5 * (lo + hi)
            below = cumulative(mid, Lk) < goal
            lo = np.where(below, mid, lo)
            hi = np.where(below, hi, mid)
        u = 0.5 * (lo + hi)
        u[0], u[-1] = 0.0, Lk
        return np.diff(u)

    return _fill_layout(counts, NP, spacings)


def _neumaier(values) -> float:
    """`sum` as Python 3.12+ adds floats (compensated), so the total thickness matches to the bit."""
    s, c = 0.0, 0.0
    for v in values:
        v = float(v)
        t = s + v
        c += (s - t) + v if abs(s) >= abs(v) else (v - t) + s
        s = t
    return s + c


def _scaled(lay: _Layout, Ls: np.ndarray, total: float):
    """`(x, h)`: each layer's spacing scaled to its thickness, then the three spacings around
    each interface set to their mean (jaxdd device.py:226-233)."""
    h = lay.raw * (Ls[lay.lid] / (total * lay.norm[lay.lid]))
    for j in lay.i0[1:]:
        h[j - 2:j + 1] = (h[j] + h[j - 1] + h[j - 2]) / 3.0
    x = np.concatenate([[0.0], np.cumsum(total * h[:-1])])
    return x, h


def make_grid(thicknesses, NP: int, grad: float, split: str = "exact"):
    """`(x, h, i0, i1, lid)` of SIMsalabim's `Make_Grid` (jaxdd device.py:236-248)."""
    lay = _simss_layout(thicknesses, NP, grad, split)
    Ls = np.array([float(t) for t in thicknesses])
    x, h = _scaled(lay, Ls, _neumaier(Ls))
    return x, h, lay.i0, lay.i1, lay.lid


@dataclass(frozen=True)
class Device:
    """Every static array of one device on its `NP + 2` points, SI units; the field names and
    meanings of jaxdd's `Device` (jaxdd device.py:251-382) for the supported scope."""

    x: np.ndarray
    h: np.ndarray
    L: float
    T: float
    Vt: float
    eps: np.ndarray
    E_c: np.ndarray
    E_v: np.ndarray
    N_c: np.ndarray
    ni: np.ndarray
    N_D: np.ndarray
    N_A: np.ndarray
    mu_n: np.ndarray  # per interval: mu_n[i] between x[i] and x[i+1]
    mu_p: np.ndarray
    k_direct: np.ndarray
    srh_Nt: np.ndarray
    srh_Cn: np.ndarray
    srh_Cp: np.ndarray
    srh_nt0: np.ndarray
    srh_pt0: np.ndarray
    G: np.ndarray
    offset_n: np.ndarray
    offset_p: np.ndarray
    V0: float
    VL: float
    n_left: float
    n_right: float
    p_left: float
    p_right: float
    W_L: float
    W_R: float
    G_frac: float
    i0: tuple
    i1: tuple
    anion_mask: np.ndarray
    cation_mask: np.ndarray
    anion_total: float
    cation_total: float
    anion_fixed: np.ndarray
    cation_fixed: np.ndarray
    pre_cond: bool
    V_pre: float
    fix_ions: bool
    interface: dict | None = None
    R_series: float = 0.0
    R_shunt: float = -1.0
    left_elec: int = -1
    curr_diff: bool = False
    anion_slots: np.ndarray | None = None
    anion_totals: np.ndarray | None = None
    cation_slots: np.ndarray | None = None
    cation_totals: np.ndarray | None = None
    mu_anion: np.ndarray | None = None
    mu_cation: np.ndarray | None = None
    free: tuple = (False, False)
    statistics: str = "boltzmann"

    @property
    def NP(self) -> int:
        return len(self.x) - 2


def _flag(layer, name, default="0") -> int:
    return int(float(layer.raw.get(name, default)))


def _refusals(setup: Setup) -> list[str]:
    """Inputs outside this build's scope, by name."""
    out = []
    for k in ("W_L", "W_R"):
        if setup.raw[k].strip().lower() == "free":
            out.append(f"{k} = free (a free end)")
    for k in ("S_n_L", "S_p_L", "S_n_R", "S_p_R"):
        if float(setup.raw.get(k, "-1")) >= 0:
            out.append(f"{k} >= 0 (finite surface recombination)")
    if setup.raw.get("genProfile", "none").strip().lower() == "calc":
        out.append("genProfile = calc (transfer-matrix optics)")
    for j, ly in enumerate(setup.layers, start=1):
        for name, what in (("mobnDep", "field-dependent mobility"),
                           ("mobpDep", "field-dependent mobility"),
                           ("useLangevin", "Langevin recombination"),
                           ("fieldDepG", "field-dependent generation")):
            if _flag(ly, name) == 1:
                out.append(f"layer {j}: {name} = 1 ({what})")
        for name in ("bulkTrapFile", "intTrapFile"):
            if ly.raw.get(name, "none").strip().lower() != "none":
                out.append(f"layer {j}: {name} (trap files)")
        if float(ly.raw.get("N_t_bulk", "0")) != 0 and _flag(ly, "bulkTrapType") != 0:
            out.append(f"layer {j}: bulkTrapType = {_flag(ly, 'bulkTrapType')} (charged bulk traps)")
        for name in ("N_max_anion", "N_max_cation"):
            if np.isfinite(float(ly.raw.get(name, "inf"))):
                out.append(f"layer {j}: {name} (ion sites)")
        for name in ("C_n_Auger", "C_p_Auger"):
            if float(ly.raw.get(name, "0")) != 0:
                out.append(f"layer {j}: {name} (Auger recombination)")
    return out


def _sfb(N_A, N_D, E_c, E_v, N_c, Vt):
    """SIMsalabim's `ObtainWorkFunction` for 'sfb': the adjacent layer's equilibrium Fermi level
    from its net doping, mid-gap without any (jaxdd device.py:561-573, Boltzmann)."""
    net = N_A - N_D
    if net > 0:
        return E_v - Vt * np.log(N_c / abs(net))
    if net < 0:
        return E_c + Vt * np.log(N_c / abs(net))
    return 0.5 * (E_c + E_v)


def _profile(table, x, lid, layer_gen, total):
    """`Init_Generation_Profile` from a file: its axis stretched to the device, interpolated
    linearly, each point in the first interval whose end lies beyond it; zero in layers that do
    not generate and beyond the axis's end (jaxdd device.py:804-815)."""
    gx, gG = table[:, 0], table[:, 1]
    a = gx * (total / gx[-1])
    j = np.searchsorted(a[1:], x, side="right")
    jj = np.minimum(j, len(a) - 2)
    g = gG[jj] + (x - a[jj]) * (gG[jj + 1] - gG[jj]) / (a[jj + 1] - a[jj])
    return np.where((j < len(a) - 1) & layer_gen[lid], g, 0.0)


def grid_layout(setup: Setup, grid: str = "graded", grid_split: str = "exact") -> _Layout:
    """The grid's structure for a setup: each layer's points and unscaled spacings (jaxdd's
    `Structure` holds the same, device.py:386-575). The thicknesses only scale it: a device built
    with this layout and other thicknesses keeps its points per layer (as jaxdd's
    `device_arrays(structure, params)` does, device.py:877-885)."""
    if grid not in GRIDS:
        raise ValueError(f"grid {grid!r}: one of {GRIDS}")
    thick = [ly.raw["L"] for ly in setup.layers]
    NP = setup.i("NP")
    if grid == "graded":
        return _graded_layout(thick, NP)
    return _simss_layout(thick, NP, setup.f("grad"), grid_split)


def build_device(setup: Setup, grid_split: str = "exact", surface: str = "extraction",
                 langevin: str = "layer", braun: str = "exact", grid: str = "graded",
                 statistics: str = "boltzmann", layout: _Layout | None = None) -> Device:
    """The device of a SIMsalabim input (jaxdd device.py:1066-1079, same arguments). `grid`
    "graded" (jaxdd's default) or "simss" (`Make_Grid`); `grid_split` as `layer_points`.
    `surface`, `langevin` and `braun` choose among models this build does not carry and are
    accepted only at their defaults; `statistics` only "boltzmann". `layout` (`grid_layout` of
    another setup of the same stack) fixes the grid's structure instead of laying it out for
    this setup's thicknesses."""
    if grid not in GRIDS:
        raise ValueError(f"grid {grid!r}: one of {GRIDS}")
    if statistics != "boltzmann":
        raise NotImplementedError(f"statistics = {statistics!r}: only Boltzmann's is built")
    if (surface, langevin, braun) != ("extraction", "layer", "exact"):
        raise NotImplementedError("surface/langevin/braun models beyond the defaults")
    if setup.i("leftElec") not in (-1, 1):
        raise ValueError("leftElec must be -1 (the left electrode the cathode) or 1 (the anode)")
    problems = _refusals(setup)
    if problems:
        raise NotImplementedError("outside this build's scope: " + "; ".join(problems))
    problems = ion_region_problems(setup)
    if problems:
        raise NotImplementedError("; ".join(problems))

    layers = setup.layers
    NP = setup.i("NP")
    lay = layout if layout is not None else grid_layout(setup, grid, grid_split)
    if len(lay.lid) != NP + 2 or len(lay.norm) != len(layers):
        raise ValueError("the layout is of another grid size or stack")
    lid = lay.lid
    per = {name: np.array([float(ly.raw[name]) for ly in layers])
           for name in ("L", "eps_r", "E_c", "E_v", "N_c", "N_D", "N_A", "mu_n", "mu_p",
                        "k_direct", "N_t_bulk", "N_anion", "N_cation", "mu_anion", "mu_cation")}
    opt = {name: np.array([float(ly.raw.get(name, "0")) for ly in layers])
           for name in ("nu_int_n", "nu_int_p", "C_n_bulk", "C_p_bulk", "E_t_bulk", "N_t_int",
                        "E_t_int", "C_n_int", "C_p_int", "G_ehp")}
    Ls = per["L"]
    total = _neumaier(Ls)
    x, h = _scaled(lay, Ls, total)
    T = setup.f("T")
    Vt = K_B * T / Q
    inner = np.zeros(NP + 2, dtype=bool)
    inner[1:-1] = True

    E_c, E_v, N_c = per["E_c"][lid], per["E_v"][lid], per["N_c"][lid]
    ni = N_c * np.exp(-0.5 * (E_v - E_c) / Vt)
    at_iface = np.zeros(NP + 2, dtype=bool)
    at_iface[list(lay.i1[:-1])] = True
    mu_n = np.where(at_iface, (total * h) * opt["nu_int_n"][lid] / Vt, per["mu_n"][lid])
    mu_p = np.where(at_iface, (total * h) * opt["nu_int_p"][lid] / Vt, per["mu_p"][lid])
    k_direct = np.where(inner, per["k_direct"][lid], 0.0)

    trap = inner & (per["N_t_bulk"] != 0)[lid]
    nt0_l = per["N_c"] * np.exp((per["E_c"] - opt["E_t_bulk"]) / Vt)
    pt0_l = per["N_c"] * np.exp((opt["E_t_bulk"] - per["E_v"]) / Vt)
    srh = {k: np.where(trap, v[lid], 0.0) for k, v in (
        ("Nt", per["N_t_bulk"]), ("Cn", opt["C_n_bulk"]), ("Cp", opt["C_p_bulk"]),
        ("nt0", nt0_l), ("pt0", pt0_l))}

    mode = setup.raw.get("genProfile", "none").strip()
    if mode.lower() == "none":
        G = opt["G_ehp"][lid]
    else:
        table = np.loadtxt(io.StringIO(setup.text("genProfile")), skiprows=1)
        layer_gen = np.array([bool(ly.i("layerGen")) for ly in layers])
        G = _profile(table, x, lid, layer_gen, total)
    G = np.where(inner, G, 0.0)

    held = bool(setup.i("fixIons", 0)) and not bool(setup.i("preCond", 0))
    ions = {}
    for sp in ("anion", "cation"):
        index = -np.ones(len(layers), dtype=int)
        mobile_regions = [(a, b) for a, b, moves in ion_regions(setup, sp) if moves and not held]
        for k, (a, b) in enumerate(mobile_regions):
            index[a:b + 1] = k
        mobile = index >= 0
        conc, mob = per[f"N_{sp}"], per[f"mu_{sp}"]
        fixed = (conc != 0) & ((mob == 0) | held)
        n_regions = int(index.max()) + 1
        many = n_regions > 1
        ions[sp] = dict(
            mask=mobile[lid],
            total=float(np.sum(np.where(mobile, Ls * conc, 0.0))),
            fixed=np.where(fixed[lid], conc[lid], 0.0),
            slots=np.stack([index[lid] == k for k in range(n_regions)]) if many else None,
            totals=np.array([np.sum(np.where(index == k, Ls * conc, 0.0))
                             for k in range(n_regions)]) if many else None,
        )

    dos = Vt * np.log(N_c / N_c[0])
    sfb = [setup.raw[k].strip().lower() == "sfb" for k in ("W_L", "W_R")]
    W_L = _sfb(per["N_A"][0], per["N_D"][0], per["E_c"][0], per["E_v"][0], per["N_c"][0], Vt) \
        if sfb[0] else setup.f("W_L")
    W_R = _sfb(per["N_A"][-1], per["N_D"][-1], per["E_c"][-1], per["E_v"][-1], per["N_c"][-1],
               Vt) if sfb[1] else setup.f("W_R")
    for name, W, ly, is_sfb in (("W_L", W_L, layers[0], sfb[0]), ("W_R", W_R, layers[-1], sfb[1])):
        if not is_sfb and not ly.f("E_c") <= W <= ly.f("E_v"):
            raise ValueError(f"{name} = {W} eV: outside the gap of its layer "
                             f"({ly.f('E_c')} to {ly.f('E_v')} eV)")

    interface = None
    with_traps = [j for j in range(len(layers) - 1) if opt["N_t_int"][j] != 0]
    if with_traps:
        interface = _interface(setup, with_traps, lay, h, total, Vt, per, opt, NP)

    return Device(
        x=x, h=h, L=total, T=T, Vt=Vt, eps=per["eps_r"][lid] * EPS_0, E_c=E_c, E_v=E_v,
        N_c=N_c, ni=ni, N_D=per["N_D"][lid], N_A=per["N_A"][lid], mu_n=mu_n, mu_p=mu_p,
        k_direct=k_direct, srh_Nt=srh["Nt"], srh_Cn=srh["Cn"], srh_Cp=srh["Cp"],
        srh_nt0=srh["nt0"], srh_pt0=srh["pt0"], G=G,
        offset_n=E_c - E_c[0] + dos, offset_p=E_v - E_v[0] - dos,
        V0=0.5 * (-W_L + W_R), VL=0.5 * (W_L - W_R),
        n_left=N_c[0] * np.exp(-(W_L - E_c[0]) / Vt),
        n_right=N_c[-1] * np.exp(-(W_R - E_c[-1]) / Vt),
        p_left=N_c[0] * np.exp((W_L - E_v[0]) / Vt),
        p_right=N_c[-1] * np.exp(-(E_v[-1] - W_R) / Vt),
        W_L=W_L, W_R=W_R, G_frac=setup.f("G_frac", 1.0), i0=tuple(lay.i0), i1=tuple(lay.i1),
        anion_mask=ions["anion"]["mask"], cation_mask=ions["cation"]["mask"],
        anion_total=ions["anion"]["total"], cation_total=ions["cation"]["total"],
        anion_fixed=ions["anion"]["fixed"], cation_fixed=ions["cation"]["fixed"],
        pre_cond=bool(setup.i("preCond", 0)), V_pre=setup.f("Vpre", 0.0),
        fix_ions=bool(setup.i("fixIons", 0)), interface=interface,
        R_series=float(setup.raw.get("R_series", "0")),
        R_shunt=float(setup.raw.get("R_shunt", "-1")), left_elec=setup.i("leftElec"),
        curr_diff=int(float(setup.raw.get("currDiffInt", "2"))) == 1,
        anion_slots=ions["anion"]["slots"], anion_totals=ions["anion"]["totals"],
        cation_slots=ions["cation"]["slots"], cation_totals=ions["cation"]["totals"],
        mu_anion=per["mu_anion"][lid], mu_cation=per["mu_cation"][lid],
    )


def _interface(setup, with_traps, lay, h, total, Vt, per, opt, NP) -> dict:
    """Interface traps on the edge after each trapped layer's last point (SIMsalabim's
    `Init_Trapping`; jaxdd device.py:827-864): per edge their density (m⁻²), capture
    coefficients, each side's SRH densities, the inverse interface width, and whether they
    are charged (with their charge when empty: 1 a donor)."""
    j = np.array(with_traps)
    e = np.array(lay.i1)[j]
    E_t, N_t = opt["E_t_int"][j], opt["N_t_int"][j]
    kind = np.array([int(float(setup.layers[k].raw.get("intTrapType", "0"))) for k in j])
    for k, lo_layer in enumerate(j):
        lo, hi = setup.layers[lo_layer], setup.layers[lo_layer + 1]
        gap = max(lo.f("E_c"), hi.f("E_c")), min(lo.f("E_v"), hi.f("E_v"))
        if not gap[0] < E_t[k] < gap[1]:
            raise ValueError(f"interface trap between layers {lo_layer + 1} and {lo_layer + 2} "
                             f"at {E_t[k]} eV: not within the gaps of both")
        if kind[k] not in (-1, 0, 1):
            raise ValueError(f"layer {lo_layer + 1}: intTrapType {kind[k]}")

    def nt0(k):
        return per["N_c"][k] * np.exp((per["E_c"][k] - E_t) / Vt)

    def pt0(k):
        return per["N_c"][k] * np.exp((E_t - per["E_v"][k]) / Vt)

    width = 0.5 * total * (0.5 * h[e + 1] + h[e] + 0.5 * h[e - 1])

    def edges(v):
        out = np.zeros(NP + 1)
        out[e] = v
        return out

    return {"Nt": edges(N_t), "Cn": edges(opt["C_n_int"][j]), "Cp": edges(opt["C_p_int"][j]),
            "nt0_lo": edges(nt0(j)), "pt0_lo": edges(pt0(j)),
            "nt0_hi": edges(nt0(j + 1)), "pt0_hi": edges(pt0(j + 1)),
            "iw": edges(1.0 / width), "charge": edges(np.abs(kind).astype(float)),
            "cwe": edges((kind == 1).astype(float))}
