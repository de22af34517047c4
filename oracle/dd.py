"""TEST INFRASTRUCTURE ONLY — FP64 NumPy oracle of jaxdd's steady-state J-V path.

A CPU restatement of the reference's arithmetic, vectorised over a batch of devices of one grid
size (as the reference's `vmap`): `solve_batch` (jaxdd src/jaxdd/batch.py:1136-1208) and
`solve_jv` (src/jaxdd/solver.py:2041-2245). The CUDA path is checked against it; nothing in the
product imports it. Each function cites the reference lines it follows.

Scope: the product's scope (Boltzmann carriers, neutral SRH bulk traps, interface traps, direct
recombination, mobile ions in slots, pre-bias with frozen or free ions, integral or differential
current, shunt). Derivatives that the reference takes by autodiff (`jax.jvp` of the Bernoulli
function and of the interface traps, `jax.jacrev` of the ion constraints) are written out by hand
here; they are exact, as autodiff is, and tests/test_oracle.py checks them against central
differences of the residual.

Pinning: the reference cannot run in this container (no JAX). The oracle is pinned against the
reference's golden J-V curves (SimSS runs under the reference's tests/data) at the reference's
own tolerances (tests/test_oracle.py); see oracle/__init__.py.
"""

from __future__ import annotations

import numpy as np

Q = 1.6022e-19

# solver.py:44-61, 2009; batch.py:79-87
ROUND_OFF_FLOOR = 1e-6
STALL_STEPS = 3
NOISE_FLOOR_CAP = 1e-3
DENSITY_FLOOR = 1e-12
STEP_CAPS = (10.0, 5.0, 5.0)
ION_LOG_CAP = 5.0
FLOOR_DROP_CAP = 50.0
CURRENT_TOL = 1e-5
CURRENT_STEP_CAP = 1e-3
QUADRATIC_TOL = 1e-5
QUADRATIC_RATIO = 1e-2
ION_DENSITY_STAGES = (1 / 64, 1 / 16, 1 / 4, 1.0)
SERIES_BELOW = 1e-2


# ----------------------------------------------------------------------------- Bernoulli

def bern_exact(x):
    """`B(x) = x/expm1(x)`, series below |x| 1e-2, and `B'(x)` (solver.py:95-105)."""
    x = np.asarray(x, dtype=float)
    small = np.abs(x) < SERIES_BELOW
    safe = np.where(small, 1.0, x)
    e = np.expm1(safe)
    with np.errstate(over="ignore", invalid="ignore", divide="ignore"):
        full = safe / e
        dfull = 1.0 / e - safe * (e + 1.0) / (e * e)
    ser = 1.0 - x / 2.0 + x * x / 12.0 - x ** 4 / 720.0
    dser = -0.5 + x / 6.0 - x ** 3 / 180.0
    return np.where(small, ser, full), np.where(small, dser, dfull)


def bern_simss(x):
    """SIMsalabim 5.36's `B` (solver.py:108-121): Taylor of order 1, 2, 4 below |x| 0.05, 0.45,
    1.5, the full expression above; and its derivative."""
    x = np.asarray(x, dtype=float)
    ax = np.abs(x)
    safe = np.where(ax < 1.5, 2.0, x)
    e = np.expm1(safe)
    with np.errstate(over="ignore", invalid="ignore", divide="ignore"):
        full = safe / e
        dfull = 1.0 / e - safe * (e + 1.0) / (e * e)
    o1, d1 = 1.0 - 0.5 * x, np.full_like(x, -0.5)
    o2, d2 = 1.0 - x * (0.5 - x / 12.0), -0.5 + x / 6.0
    o4 = 1.0 + x * (-0.5 + x * (1.0 / 12.0 - x * x / 720.0))
    d4 = -0.5 + x / 6.0 - x ** 3 / 180.0
    val = np.where(ax < 0.05, o1, np.where(ax < 0.45, o2, np.where(ax < 1.5, o4, full)))
    der = np.where(ax < 0.05, d1, np.where(ax < 0.45, d2, np.where(ax < 1.5, d4, dfull)))
    return val, der


BERNOULLI = {"exact": bern_exact, "simss": bern_simss}


# ----------------------------------------------------------------------------- batch tree

def _stencils(dev) -> dict:
    """solver._stencils (solver.py:210-278) for the supported scope, over interior points."""
    NP = len(dev.x) - 2
    i = np.arange(1, NP + 1)
    h, L, eps = dev.h, dev.L, dev.eps
    fac_m = (eps[i] - eps[i - 1]) / (h[i - 1] ** 2 * L ** 2) - 2 * eps[i] * (
        1 / (h[i] * (h[i] + h[i - 1]) * L ** 2) + 1 / (h[i - 1] * (h[i] + h[i - 1]) * L ** 2))
    fac_l = 2 * eps[i] / (h[i - 1] * (h[i] + h[i - 1]) * L ** 2) - (eps[i] - eps[i - 1]) / (
        h[i - 1] ** 2 * L ** 2)
    fac_u = 2 * eps[i] / (h[i] * (h[i] + h[i - 1]) * L ** 2)
    return {
        "fac_l": fac_l, "fac_m": fac_m, "fac_u": fac_u, "hm": h[i - 1], "hp": h[i],
        "fac": 0.5 * L ** 2 * h[i] * h[i - 1] * (h[i] + h[i - 1]),
        "mun_m": dev.mu_n[i - 1], "mun_p": dev.mu_n[i],
        "mup_m": dev.mu_p[i - 1], "mup_p": dev.mu_p[i],
        "offn": np.stack([dev.offset_n[i - 1], dev.offset_n[i], dev.offset_n[i + 1]], -1),
        "offp": np.stack([dev.offset_p[i - 1], dev.offset_p[i], dev.offset_p[i + 1]], -1),
        "dop": dev.N_A[i] - dev.N_D[i], "kd": dev.k_direct[i], "ni2": dev.ni[i] ** 2,
        "Nt": dev.srh_Nt[i], "Cn": dev.srh_Cn[i], "Cp": dev.srh_Cp[i],
        "nt0": dev.srh_nt0[i], "pt0": dev.srh_pt0[i], "G": dev.G[i],
        "a_mask": dev.anion_mask[i].astype(float), "c_mask": dev.cation_mask[i].astype(float),
        "a_fix": dev.anion_fixed[i], "c_fix": dev.cation_fixed[i],
        "n_floor": np.full(NP, DENSITY_FLOOR * np.max(dev.N_c)),
        "sP": 1.0 / (Q * dev.N_c[i]),
        "sC": 1.0 / (np.maximum(dev.mu_n[i], dev.mu_p[i]) * dev.Vt * dev.N_c[i] * h[i]),
    }


_TI_KEYS = ("Nt", "Cn", "Cp", "nt0_lo", "pt0_lo", "nt0_hi", "pt0_hi", "iw", "charge", "cwe")


def bern_complex(x, simss=False):
    """The Bernoulli function (`bern_exact` or `bern_simss`, solver.py:95-121) at complex
    arguments near the real axis, for complex-step derivatives: each branch chosen by the real
    part, every branch analytic."""
    x = np.asarray(x, dtype=complex)
    a = np.abs(x.real)
    if not simss:
        small = a < SERIES_BELOW
        safe = np.where(small, 1.0, x)
        return np.where(small, 1.0 - x / 2.0 + x * x / 12.0 - x ** 4 / 720.0,
                        safe / np.expm1(safe))
    safe = np.where(a < 1.5, 2.0, x)
    full = safe / np.expm1(safe)
    o1 = 1.0 - 0.5 * x
    o2 = 1.0 - x * (0.5 - x / 12.0)
    o4 = 1.0 + x * (-0.5 + x * (1.0 / 12.0 - x * x / 720.0))
    return np.where(a < 0.05, o1, np.where(a < 0.45, o2, np.where(a < 1.5, o4, full)))



def _slots_of(mask, total, masks, totals):
    if masks is None:
        return mask[None].astype(float), np.array([float(total)])
    return masks.astype(float), np.asarray(totals, dtype=float)


def _one(dev) -> dict:
    """One device's tree: batch._device_tree (batch.py:90-126) and solver._ion_setup
    (solver.py:1940-1961) for the supported scope."""
    NP = len(dev.x) - 2
    iface = np.zeros(NP + 1, dtype=bool)
    for k in dev.i1[:-1]:
        iface[k] = True
    generated = Q * dev.L * np.sum(dev.h[:-1] * dev.G[:-1]) / np.sum(dev.h[:-1])
    a_slots, a_totals = _slots_of(dev.anion_mask, dev.anion_total, dev.anion_slots,
                                  dev.anion_totals)
    c_slots, c_totals = _slots_of(dev.cation_mask, dev.cation_total, dev.cation_slots,
                                  dev.cation_totals)
    ti = dev.interface if dev.interface is not None else {k: np.zeros(NP + 1) for k in _TI_KEYS}
    return {
        "s": _stencils(dev), "ti": {k: np.asarray(ti[k], dtype=float) for k in _TI_KEYS},
        "ion": {"hL": dev.h[:-1] * dev.L, "a_slots": a_slots, "a_totals": a_totals,
                "c_slots": c_slots, "c_totals": c_totals},
        "Vt": dev.Vt, "g_frac": dev.G_frac, "L": dev.L, "x": dev.x, "h": dev.h, "eps": dev.eps,
        "N_c": dev.N_c, "ni": dev.ni, "E_c": dev.E_c, "V0": dev.V0, "VL": dev.VL,
        "W_L": dev.W_L, "W_R": dev.W_R,
        "ln_n_left": np.log(dev.n_left), "ln_n_right": np.log(dev.n_right),
        "ln_p_left": np.log(dev.p_left), "ln_p_right": np.log(dev.p_right),
        "offset_n": dev.offset_n, "offset_p": dev.offset_p, "mu_n": dev.mu_n, "mu_p": dev.mu_p,
        "mu_a": np.zeros(NP + 2) if dev.mu_anion is None else np.asarray(dev.mu_anion, float),
        "mu_c": np.zeros(NP + 2) if dev.mu_cation is None else np.asarray(dev.mu_cation, float),
        "G": dev.G,
        "rec": {"kd": dev.k_direct, "ni2": dev.ni ** 2, "Nt": dev.srh_Nt, "Cn": dev.srh_Cn,
                "Cp": dev.srh_Cp, "nt0": dev.srh_nt0, "pt0": dev.srh_pt0},
        "iface": iface, "J_scale": max(generated, 1.0), "R_series": dev.R_series,
        "left_elec": float(dev.left_elec),
        "G_shunt": 1.0 / dev.R_shunt if dev.R_shunt > 0 else 0.0,
        "pre_cond": float(dev.pre_cond), "V_pre": dev.V_pre, "fix_ions": float(dev.fix_ions),
        "curr_diff": float(dev.curr_diff),
    }


def _stack(trees):
    first = trees[0]
    if isinstance(first, dict):
        return {k: _stack([t[k] for t in trees]) for k in first}
    return np.stack([np.asarray(t) for t in trees])


def prepare(devices) -> dict:
    """batch.prepare (batch.py:151-223): one grid size, slots padded with empty ones."""
    sizes = {len(d.x) for d in devices}
    if len(sizes) != 1:
        raise ValueError(f"a batch needs one grid size, got NP + 2 in {sorted(sizes)}")
    trees = [_one(d) for d in devices]
    for sp in ("a", "c"):
        most = max(t["ion"][f"{sp}_slots"].shape[0] for t in trees)
        for t in trees:
            extra = most - t["ion"][f"{sp}_slots"].shape[0]
            if extra:
                sl, tot = t["ion"][f"{sp}_slots"], t["ion"][f"{sp}_totals"]
                t["ion"][f"{sp}_slots"] = np.concatenate([sl, np.zeros((extra, sl.shape[1]))])
                t["ion"][f"{sp}_totals"] = np.concatenate([tot, np.zeros(extra)])
    return _stack(trees)


def take(tree, idx):
    if isinstance(tree, dict):
        return {k: take(v, idx) for k, v in tree.items()}
    return tree[idx]


def put(tree, idx, part):
    for k, v in part.items():
        if isinstance(v, dict):
            put(tree[k], idx, v)
        else:
            tree[k][idx] = v


def _col(v):
    return np.asarray(v)[:, None]


# ----------------------------------------------------------------------------- physics

def _recombination(n, p, r):
    """Direct + SRH through one neutral level (solver.py:734-745); with its derivatives in
    `ln n` and `ln p` (n·∂R/∂n, p·∂R/∂p), which the reference takes by `jax.jvp`."""
    Nt, Cn, Cp, nt0, pt0 = r["Nt"], r["Cn"], r["Cp"], r["nt0"], r["pt0"]
    traps = Nt > 0
    num = Nt * Cn * Cp * (n * p - nt0 * pt0)
    den = np.where(traps, Cn * (n + nt0) + Cp * (p + pt0), 1.0)
    srh = np.where(traps, num / den, 0.0)
    R = r["kd"] * (n * p - r["ni2"]) + srh
    dsrh_n = np.where(traps, (Nt * Cn * Cp * p - srh * Cn) / den, 0.0)
    dsrh_p = np.where(traps, (Nt * Cn * Cp * n - srh * Cp) / den, 0.0)
    dR_n = n * (r["kd"] * p + dsrh_n)
    dR_p = p * (r["kd"] * n + dsrh_p)
    return R, dR_n, dR_p


def _iface_edges(nL, nR, pL, pR, ti):
    """Interface traps per edge (solver.py:814-850, steady state, one level): values
    `(Rn_L, Rn_R, Rp_L, Rp_R, Q)` and their derivatives in `ln nL, ln nR, ln pL, ln pR`."""
    Nt, Cn, Cp, iw = ti["Nt"], ti["Cn"], ti["Cp"], ti["iw"]
    an, bp = Cn * Nt, Cp * Nt
    traps = Nt > 0
    a, b = an * (nL + nR), bp * (pL + pR)
    c, d = an * (ti["nt0_lo"] + ti["nt0_hi"]), bp * (ti["pt0_lo"] + ti["pt0_hi"])
    S = np.where(traps, a + b + c + d, 1.0)
    inv = np.where(traps, 1.0 / S, 0.0)
    full = (a + d) * inv
    empty = (b + c) * inv
    half_q = ti["charge"] * 0.5 * Nt * iw

    val = np.stack([iw * an * (nL * empty - ti["nt0_lo"] * full),
                    iw * an * (nR * empty - ti["nt0_hi"] * full),
                    iw * bp * (pL * full - ti["pt0_lo"] * empty),
                    iw * bp * (pR * full - ti["pt0_hi"] * empty),
                    half_q * (ti["cwe"] - full)])
    derivs = []
    for which in range(4):  # nL, nR, pL, pR
        if which < 2:
            da = an * (nL if which == 0 else nR)
            dfull, dempty = da * empty * inv, -da * empty * inv
        else:
            db = bp * (pL if which == 2 else pR)
            dfull, dempty = -db * full * inv, db * full * inv
        own = [0.0, 0.0, 0.0, 0.0]
        own[which] = 1.0
        derivs.append(np.stack([
            iw * an * (own[0] * nL * empty + nL * dempty - ti["nt0_lo"] * dfull),
            iw * an * (own[1] * nR * empty + nR * dempty - ti["nt0_hi"] * dfull),
            iw * bp * (own[2] * pL * full + pL * dfull - ti["pt0_lo"] * dempty),
            iw * bp * (own[3] * pR * full + pR * dfull - ti["pt0_hi"] * dempty),
            -half_q * dfull]))
    return val, derivs


def _iface_terms(n, p, ti):
    """solver._interface_terms (solver.py:876-914): `(Q, Rn, Rp)` at interior points and their
    derivatives in the point's own, next and previous `(ln n, ln p)`."""
    val, (d_nL, d_nR, d_pL, d_pR) = _iface_edges(n[:, :-1], n[:, 1:], p[:, :-1], p[:, 1:], ti)
    lo, hi = [4, 0, 2], [4, 1, 3]
    X = val[hi][:, :, :-1] + val[lo][:, :, 1:]
    own = np.stack([d_nR[hi][:, :, :-1] + d_nL[lo][:, :, 1:],
                    d_pR[hi][:, :, :-1] + d_pL[lo][:, :, 1:]], -1)
    up = np.stack([d_nR[lo][:, :, 1:], d_pR[lo][:, :, 1:]], -1)
    down = np.stack([d_nL[hi][:, :, :-1], d_pL[hi][:, :, :-1]], -1)
    return X, own, up, down


def _iface_points(n, p, ti):
    """solver._interface_points (solver.py:865-873): `(Rn, Rp)` on all NP + 2 points."""
    val, _ = _iface_edges(n[:, :-1], n[:, 1:], p[:, :-1], p[:, 1:], ti)

    def points(lo, hi):
        return np.concatenate([lo[:, :1], hi[:, :-1] + lo[:, 1:], hi[:, -1:]], 1)

    return points(val[0], val[1]), points(val[2], val[3])


def assemble(full, s, ti, Vt, g_frac, la, lc, bern):
    """solver._assemble (solver.py:1021-1187), supported scope: residual F (B×NP×3), blocks
    A, B, C (B×NP×3×3) and ion columns U (B×NP×3×2) from `full` (B×(NP+2)×3)."""
    Vt = _col(Vt)
    V, n, p = full[..., 0], np.exp(full[..., 1]), np.exp(full[..., 2])
    offn = np.concatenate([s["offn"][:, :, 0], s["offn"][:, -1:, 1:].reshape(-1, 2)], 1)
    offp = np.concatenate([s["offp"][:, :, 0], s["offp"][:, -1:, 1:].reshape(-1, 2)], 1)
    cn = Vt * np.concatenate([s["mun_m"], s["mun_p"][:, -1:]], 1)
    cp = Vt * np.concatenate([s["mup_m"], s["mup_p"][:, -1:]], 1)
    xn = np.diff(V + offn, axis=1) / Vt
    xp = np.diff(V + offp, axis=1) / Vt
    Bnf, dBnf = bern(xn)
    Bnb, dBnb = bern(-xn)
    Bpf, dBpf = bern(xp)
    Bpb, dBpb = bern(-xp)
    n0, n1, p0, p1 = n[:, :-1], n[:, 1:], p[:, :-1], p[:, 1:]
    z = np.zeros_like(xn)
    Fn = cn * (Bnf * n1 - Bnb * n0)
    gn = cn * (dBnf * n1 + dBnb * n0) / Vt
    dFn0 = np.stack([-gn, -cn * Bnb * n0, z], -1)
    dFn1 = np.stack([gn, cn * Bnf * n1, z], -1)
    Fp = cp * (Bpf * p0 - Bpb * p1)
    gp = cp * (dBpf * p0 + dBpb * p1) / Vt
    dFp0 = np.stack([-gp, z, cp * Bpf * p0], -1)
    dFp1 = np.stack([gp, z, -cp * Bpb * p1], -1)

    Vm, nm, pm = V[:, 1:-1], n[:, 1:-1], p[:, 1:-1]
    hm, hp, fac = s["hm"][..., None], s["hp"][..., None], s["fac"]
    zm = np.zeros_like(Vm)
    R, dR_n, dR_p = _recombination(nm, pm, s)
    gen = s["G"] * _col(g_frac)
    dnet = np.stack([zm, -dR_n, -dR_p], -1)
    elec = hm[..., 0] * Fn[:, 1:] - hp[..., 0] * Fn[:, :-1] + fac * (gen - R)
    hole = hp[..., 0] * Fp[:, :-1] - hm[..., 0] * Fp[:, 1:] + fac * (gen - R)
    anion = s["a_mask"] * np.exp(la + Vm / Vt)
    cation = s["c_mask"] * np.exp(lc - Vm / Vt)
    poisson = (s["fac_l"] * V[:, :-2] + s["fac_m"] * Vm + s["fac_u"] * V[:, 2:]
               - Q * (nm - pm + s["dop"] + s["a_fix"] + anion - s["c_fix"] - cation))
    P_A = np.stack([s["fac_l"], zm, zm], -1)
    P_C = np.stack([s["fac_u"], zm, zm], -1)
    P_B = np.stack([s["fac_m"] - Q * (anion + cation) / Vt, -Q * nm, Q * pm], -1)
    sP, sC = s["sP"][..., None], s["sC"][..., None]
    A = np.stack([P_A * sP, -hp * dFn0[:, :-1] * sC, hp * dFp0[:, :-1] * sC], -2)
    Bb = np.stack([P_B * sP,
                   (-hp * dFn1[:, :-1] + hm * dFn0[:, 1:] + fac[..., None] * dnet) * sC,
                   (hp * dFp1[:, :-1] - hm * dFp0[:, 1:] + fac[..., None] * dnet) * sC], -2)
    C = np.stack([P_C * sP, hm * dFn1[:, 1:] * sC, -hm * dFp1[:, 1:] * sC], -2)
    if np.any(ti["Nt"] > 0):
        X, own, up, down = _iface_terms(n, p, ti)
        scale = np.stack([Q * s["sP"], -fac * s["sC"], -fac * s["sC"]], 0)  # 3×B×NP
        poisson = poisson + Q * X[0]
        elec = elec - fac * X[1]
        hole = hole - fac * X[2]

        def block(dd):  # 3×B×NP×2 -> B×NP×3×3, nothing in the potential's column
            dd = np.moveaxis(dd * scale[..., None], 0, 2)
            return np.concatenate([np.zeros_like(dd[..., :1]), dd], -1)

        A, Bb, C = A + block(down), Bb + block(own), C + block(up)
    F = np.stack([poisson * s["sP"], elec * s["sC"], hole * s["sC"]], -1)
    U = np.stack([np.stack([-Q * anion * s["sP"], zm, zm], -1),
                  np.stack([Q * cation * s["sP"], zm, zm], -1)], -1)
    return F, A, Bb, C, U


# ----------------------------------------------------------------------------- ions

def _slot_signs(ion):
    ka, kc = ion["a_slots"].shape[1], ion["c_slots"].shape[1]
    return np.concatenate([np.ones(ka), -np.ones(kc)]), ka


def _masks(ion):
    return np.concatenate([ion["a_slots"], ion["c_slots"]], 1), \
        np.concatenate([ion["a_totals"], ion["c_totals"]], 1)


def point_logs(logs, ion):
    """solver._point_logs (solver.py:1201-1204)."""
    ka = ion["a_slots"].shape[1]
    la = np.einsum("bk,bkn->bn", logs[:, :ka], ion["a_slots"][:, :, 1:-1])
    lc = np.einsum("bk,bkn->bn", logs[:, ka:], ion["c_slots"][:, :, 1:-1])
    return la, lc


def _number(dens, masks, ion):
    """solver._ion_number (solver.py:1241-1252), trapezoidal form."""
    pair = masks[:, :, 1:] * masks[:, :, :-1]
    return np.sum(0.5 * (dens[:, :, 1:] + dens[:, :, :-1]) * pair * ion["hL"][:, None, :], 2)


def ion_constraints(V_full, logs, ion, Vt):
    """solver._ion_constraints (solver.py:1255-1265) and its derivatives in the interior
    potentials `W` (B×K×NP) and in the normalisations `D` (B×K×K, diagonal), which the
    reference takes by `jax.jacrev`."""
    masks, totals = _masks(ion)
    sign, _ = _slot_signs(ion)
    zz = logs[:, :, None] + sign[None, :, None] * V_full[:, None, :] / _col(Vt)[:, :, None]
    dens = masks * np.exp(zz)
    number = _number(dens, masks, ion)
    has = totals > 0
    tot = np.where(has, totals, 1.0)
    g = np.where(has, number / tot - 1.0, 0.0)
    pair = masks[:, :, 1:] * masks[:, :, :-1] * ion["hL"][:, None, :]
    wpt = 0.5 * (pair[:, :, :-1] + pair[:, :, 1:])  # each interior point's two edges
    W = np.where(has[:, :, None], wpt * dens[:, :, 1:-1] * sign[None, :, None]
                 / _col(Vt)[:, :, None] / tot[:, :, None], 0.0)
    Dg = np.where(has, number / tot, 0.0)
    return g, W, Dg


def ion_logs(V_full, ion, Vt):
    """solver._ion_logs (solver.py:1695-1725), Boltzmann ions: closed form."""
    masks, totals = _masks(ion)
    sign, _ = _slot_signs(ion)
    shift = sign[None, :, None] * V_full[:, None, :] / _col(Vt)[:, :, None]
    has = totals > 0
    num = _number(masks * np.exp(shift), masks, ion)
    with np.errstate(divide="ignore"):
        return np.where(has, np.log(np.where(has, totals, 1.0) / np.where(has, num, 1.0)), 0.0)


def _held(ion):
    return np.where(_masks(ion)[1] > 0, 0.0, 1.0)


def slot_columns(U, ion):
    """solver._slot_columns (solver.py:1207-1212): B×NP×3×2 -> B×NP×3×K."""
    a = U[..., :1] * np.swapaxes(ion["a_slots"][:, :, 1:-1], 1, 2)[:, :, None, :]
    c = U[..., 1:] * np.swapaxes(ion["c_slots"][:, :, 1:-1], 1, 2)[:, :, None, :]
    return np.concatenate([a, c], -1)


# ----------------------------------------------------------------------------- linear algebra

def block_thomas(A, Bb, C, d):
    """solver._block_thomas (solver.py:1534-1560): forward elimination and back substitution;
    each node's block solved by LU (NumPy) rather than the reference's adjugate. d: B×NP×3×m."""
    NP = A.shape[1]
    cp = np.empty_like(C)
    dp = np.empty_like(d)
    c_prev = np.zeros_like(C[:, 0])
    d_prev = np.zeros_like(d[:, 0])
    for i in range(NP):
        M = Bb[:, i] - A[:, i] @ c_prev
        rhs = np.concatenate([C[:, i], d[:, i] - A[:, i] @ d_prev], -1)
        sol = np.linalg.solve(M, rhs)
        c_prev, d_prev = sol[..., :3], sol[..., 3:]
        cp[:, i], dp[:, i] = c_prev, d_prev
    x = np.empty_like(d)
    nxt = np.zeros_like(d[:, 0])
    for i in range(NP - 1, -1, -1):
        nxt = dp[:, i] - cp[:, i] @ nxt
        x[:, i] = nxt
    return x


def bordered_solve(A, Bb, C, U, W, D, r, rg):
    """batch._bordered_solve (batch.py:595-603): the sweep on 1 + K right-hand sides, then the
    K×K Schur complement. `W` acts on the potential (row 0) only."""
    X = block_thomas(A, Bb, C, np.concatenate([r[..., None], U], -1))
    XF, XU = X[..., 0], X[..., 1:]
    schur = D - np.einsum("bkn,bnl->bkl", W, XU[:, :, 0, :])
    z = np.linalg.solve(schur, (rg - np.einsum("bkn,bn->bk", W, XF[:, :, 0]))[..., None])[..., 0]
    return XF - np.einsum("bnrk,bk->bnr", XU, z), z


def tridiag(lo, mid, up, rhs):
    """A scalar tridiagonal solve per lane (`lax.linalg.tridiagonal_solve`), rhs B×NP×m."""
    NP = mid.shape[1]
    cp = np.empty_like(mid)
    dp = np.empty_like(rhs)
    c_prev = np.zeros_like(mid[:, 0])
    d_prev = np.zeros_like(rhs[:, 0])
    for i in range(NP):
        m = mid[:, i] - lo[:, i] * c_prev
        c_prev = up[:, i] / m
        d_prev = (rhs[:, i] - lo[:, i, None] * d_prev) / m[:, None]
        cp[:, i], dp[:, i] = c_prev, d_prev
    x = np.empty_like(rhs)
    nxt = np.zeros_like(rhs[:, 0])
    for i in range(NP - 1, -1, -1):
        nxt = dp[:, i] - cp[:, i, None] * nxt
        x[:, i] = nxt
    return x


# ----------------------------------------------------------------------------- Newton

def bounds(d, Vint):
    """batch._bounds (batch.py:255-259): the contacts' `(V, ln n, ln p)`, B×2×3."""
    e = d["left_elec"]
    return np.stack([
        np.stack([d["V0"] + 0.5 * e * Vint, d["ln_n_left"], d["ln_p_left"]], -1),
        np.stack([d["VL"] - 0.5 * e * Vint, d["ln_n_right"], d["ln_p_right"]], -1)], 1)


def full_of(bnd, y):
    return np.concatenate([bnd[:, :1], y, bnd[:, 1:]], 1)


def system(y, logs, bnd, d, s, ion, bern):
    """batch._system (batch.py:518-549) without the time terms."""
    la, lc = point_logs(logs, ion)
    full = full_of(bnd, y)
    F, A, Bb, C, U = assemble(full, s, d["ti"], d["Vt"], d["g_frac"], la, lc, bern)
    U = slot_columns(U, ion)
    g, W, Dg = ion_constraints(full[..., 0], logs, ion, d["Vt"])
    K = logs.shape[1]
    D = np.zeros((y.shape[0], K, K))
    idx = np.arange(K)
    D[:, idx, idx] = Dg + _held(ion)
    return F, g, (A, Bb, C, U, W, D)


def density_steps(y, delta, step, n_floor):
    """solver.density_steps (solver.py:74-88)."""
    dd = delta[..., 1:3]
    below = y[..., 1:3] < np.log(n_floor)[..., None]
    positive = dd > -1
    in_n = np.where(positive, np.log1p(np.where(positive & below, dd, 0.0)), -STEP_CAPS[1])
    in_n = np.clip(in_n, -FLOOR_DROP_CAP, STEP_CAPS[1])
    out = step.copy()
    out[..., 1:3] = np.where(below, in_n, step[..., 1:3])
    return out


def _caps(Vt):
    return np.stack([STEP_CAPS[0] * Vt, np.full_like(Vt, STEP_CAPS[1]),
                     np.full_like(Vt, STEP_CAPS[2])], -1)[:, None, :]


def newton_step(y, logs, bnd, d, s, ion, bern):
    """One damped Newton step (batch.py:759-785; solver._newton_step 1563-1608)."""
    F, g, (A, Bb, C, U, W, D) = system(y, logs, bnd, d, s, ion, bern)
    delta, d_logs = bordered_solve(A, Bb, C, U, W, D, -F, -g)
    caps = _caps(d["Vt"])
    stepv = density_steps(y, delta, np.clip(delta, -caps, caps), s["n_floor"])
    d_logs = np.clip(d_logs, -ION_LOG_CAP, ION_LOG_CAP)
    new = y + stepv
    with np.errstate(over="ignore", invalid="ignore"):
        dens = np.exp(new[..., 1:])
        weight = dens / (dens + s["n_floor"][..., None])
        size = np.maximum(np.maximum(np.max(np.abs(stepv[..., 0]), 1) / d["Vt"],
                                     np.max(np.abs(stepv[..., 1:]) * weight, axis=(1, 2))),
                          np.max(np.abs(d_logs), 1))
    return new, logs + d_logs, size


def current(d, full, bern):
    """batch._current / _current_parts (batch.py:302-403), steady state: SIMsalabim's integral
    form (or the differential one where `curr_diff`), averaged over the intervals; with the
    anode on the left every sign turned. B lanes."""
    g_frac = _col(d["g_frac"])
    V, n, p = full[..., 0], np.exp(full[..., 1]), np.exp(full[..., 2])
    Vt, x, h, L = _col(d["Vt"]), d["x"], d["h"], _col(d["L"])
    NP = x.shape[1] - 2
    R, _, _ = _recombination(n, p, d["rec"])
    if np.any(d["ti"]["Nt"] > 0):
        Rin, Rip = _iface_points(n, p, d["ti"])
    else:
        Rin = Rip = np.zeros_like(R)
    dx = np.diff(x[:, :NP + 1], axis=1)
    width = h[:, :NP + 1]
    G = d["G"]

    def carrier(sn, Vg, dens, mu, R_i):
        Uc = R + R_i - G * g_frac
        Uc[:, 0] = 0.0
        Uc[:, -1] = 0.0
        with np.errstate(over="ignore", invalid="ignore"):
            ev = np.exp(sn * Vg[:, :NP + 1] / Vt)
            int_u = np.concatenate([np.zeros((len(dx), 1)),
                                    np.cumsum(0.5 * dx * (Uc[:, :NP] + Uc[:, 1:NP + 1]), 1)], 1)
            single = np.sum(0.5 * dx * (ev[:, :-1] / mu[:, :NP] + ev[:, 1:] / mu[:, 1:NP + 1]), 1)
            double = np.sum(0.5 * dx * (ev[:, :-1] * int_u[:, :-1] / mu[:, :NP]
                                        + ev[:, 1:] * int_u[:, 1:] / mu[:, 1:NP + 1]), 1)
            K = (Vt[:, 0] * (sn * dens[:, NP + 1] * np.exp(sn * Vg[:, NP + 1] / Vt[:, 0])
                             - sn * dens[:, 0] * np.exp(sn * Vg[:, 0] / Vt[:, 0]))
                 - sn * double) / single
        J = Q * K[:, None] + np.concatenate(
            [np.zeros((len(dx), 1)), np.cumsum(sn * Q * L * width[:, 1:NP + 1] * Uc[:, 1:NP + 1], 1)], 1)
        diff = d["curr_diff"] > 0
        if np.any(diff):
            dV = sn * np.diff(Vg, axis=1) / Vt
            Bm, _ = bern(-dV)
            Bp, _ = bern(dV)
            flux = sn * Q * mu[:, :NP + 1] * Vt * (dens[:, 1:] * Bm - dens[:, :-1] * Bp) / (
                L * h[:, :NP + 1])
            J = np.where(diff[:, None], flux, J)
        through = sn * 0.5 * Q * L * h[:, :NP + 1] * (R_i[:, :NP + 1] + R_i[:, 1:])
        return np.where(d["iface"], np.roll(J, 1, axis=1) + through, J)

    sign = -_col(d["left_elec"])
    Jn = sign * carrier(-1.0, V + d["offset_n"], n, d["mu_n"], Rin)
    Jp = sign * carrier(1.0, V + d["offset_p"], p, d["mu_p"], Rip)
    hh = h[:, :NP + 1]
    return np.sum(hh * (Jn + Jp), 1) / np.sum(hh, 1)


def _lane(d, idx):
    return take(d, idx)


def newton_loop(y, logs, d, Vint, bern, tol, max_iter, strict=False, skip=None):
    """batch._newton_loop (batch.py:740-848) without contacts or an internal-voltage unknown:
    damped Newton per lane until converged, `max_iter`, or a step that is not a number.
    Returns `(y, logs, J, converged, iterations)`; J is the current at the last iterate
    (inf where no step was taken)."""
    nb = y.shape[0]
    y, logs = y.copy(), logs.copy()
    size_h = np.full((nb, STALL_STEPS + 1), np.inf)
    J_h = np.full((nb, STALL_STEPS + 1), np.inf)
    it = np.zeros(nb, dtype=int)
    done = np.zeros(nb, bool) if skip is None else np.asarray(skip, bool).copy()
    Vint = np.broadcast_to(np.asarray(Vint, dtype=float), (nb,))
    while True:
        active = ~done & (it < max_iter) & ~np.isnan(size_h[:, -1])
        if not active.any():
            break
        idx = np.flatnonzero(active)
        dd = _lane(d, idx)
        bnd = bounds(dd, Vint[idx])
        new, logs_new, size = newton_step(y[idx], logs[idx], bnd, dd, dd["s"], dd["ion"], bern)
        J = current(dd, full_of(bnd, new), bern)
        sh = np.concatenate([size_h[idx, 1:], size[:, None]], 1)
        jh = np.concatenate([J_h[idx, 1:], J[:, None]], 1)
        n_it = it[idx] + 1
        size_now, prev = sh[:, -1], sh[:, -2]
        with np.errstate(invalid="ignore"):
            stalled = ((n_it > STALL_STEPS) & (np.max(sh, 1) < ROUND_OFF_FLOOR)
                       & (np.min(sh[:, 1:], 1) >= 0.1 * sh[:, 0]))
            scale = dd["J_scale"] + np.abs(jh[:, -1])
            settled = ((n_it > STALL_STEPS) & (size_now < CURRENT_STEP_CAP)
                       & (np.max(np.abs(jh - jh[:, -1:]), 1) < CURRENT_TOL * scale))
            quadratic = (n_it > 1) & (size_now < QUADRATIC_TOL) & (size_now < QUADRATIC_RATIO * prev)
            if strict:
                conv = (size_now < tol) | stalled
            else:
                conv = (size_now < tol) | stalled | settled | quadratic
        y[idx], logs[idx] = new, logs_new
        size_h[idx], J_h[idx], it[idx], done[idx] = sh, jh, n_it, conv
    return y, logs, J_h[:, -1], done, it


# ----------------------------------------------------------------------------- start

def initial(d, Vint):
    """batch._initial (batch.py:276-299): linear potential and Fermi level."""
    x, L, e = d["x"], _col(d["L"]), _col(d["left_elec"])
    Vint = _col(Vint)
    V = _col(d["V0"]) + 0.5 * e * Vint + x * (_col(d["VL"]) - _col(d["V0"]) - e * Vint) / L
    EF = _col(d["W_L"]) - x * (_col(d["W_L"]) - _col(d["W_R"])) / L
    ln_n = np.log(d["N_c"]) - (EF - d["E_c"]) / _col(d["Vt"])
    ln_p = 2 * np.log(d["ni"]) - ln_n
    return np.stack([V, ln_n, ln_p], -1)


def poisson_delta(full, d, s, ion, coupled=True):
    """solver._poisson_delta (solver.py:1757-1800): Poisson's Newton step with the densities
    following the potential and the ions' normalisations re-fitted; bordered by the slots and
    damped as a whole where there are mobile ions, else clipped per point. The interface traps
    do not enter (`_on_points`)."""
    Vt = _col(d["Vt"])
    V = full[..., 0]
    logs = ion_logs(V, ion, d["Vt"])
    la, lc = point_logs(logs, ion)
    Vm = V[:, 1:-1]
    n, p = np.exp(full[:, 1:-1, 1]), np.exp(full[:, 1:-1, 2])
    ea = s["a_mask"] * np.exp(la + Vm / Vt)
    ec = s["c_mask"] * np.exp(lc - Vm / Vt)
    F = (s["fac_l"] * V[:, :-2] + s["fac_m"] * Vm + s["fac_u"] * V[:, 2:]
         - Q * (n - p + s["dop"] + s["a_fix"] + ea - s["c_fix"] - ec)) * s["sP"]
    mid = (s["fac_m"] - Q * (n + p) / Vt - Q * (ea + ec) / Vt) * s["sP"]
    lo = s["fac_l"] * s["sP"]
    up = s["fac_u"] * s["sP"]
    lo = lo.copy()
    up = up.copy()
    lo[:, 0] = 0.0
    up[:, -1] = 0.0
    dV = tridiag(lo, mid, up, -F[..., None])[..., 0]
    cap = STEP_CAPS[0] * Vt
    clipped = np.clip(dV, -cap, cap)
    if not coupled:
        return clipped
    masks, totals = _masks(ion)
    mobile = np.any(totals > 0, 1)
    if not mobile.any():
        return clipped
    U2 = np.zeros(ea.shape + (3, 2))
    U2[..., 0, 0] = -Q * ea * s["sP"]
    U2[..., 0, 1] = Q * ec * s["sP"]
    Uc = slot_columns(U2, ion)[:, :, 0, :]
    XU = tridiag(lo, mid, up, Uc)
    g, W, Dg = ion_constraints(V, logs, ion, d["Vt"])
    K = logs.shape[1]
    Dm = np.zeros((V.shape[0], K, K))
    Dm[:, np.arange(K), np.arange(K)] = Dg + _held(ion)
    z = np.linalg.solve(Dm - W @ XU, (-g - np.einsum("bkn,bn->bk", W, dV))[..., None])[..., 0]
    step = dV - np.einsum("bnk,bk->bn", XU, z)
    m = np.max(np.abs(step), 1, keepdims=True) / Vt
    safe = np.where(m > 0, m, 1.0)
    step = step * np.where(m > 0, np.minimum(np.log1p(safe), STEP_CAPS[0]) / safe, 1.0)
    return np.where(mobile[:, None], step, clipped)


def poisson_solve(y, d, s, ion, Vint, max_iter):
    """batch._poisson_solve (batch.py:486-503): until max|ΔV/V_T| < 1e-8 or `max_iter`."""
    nb = y.shape[0]
    y = y.copy()
    size = np.full(nb, np.inf)
    it = np.zeros(nb, int)
    Vint = np.broadcast_to(np.asarray(Vint, dtype=float), (nb,))
    while True:
        active = (size > 1e-8) & (it < max_iter)
        if not active.any():
            break
        idx = np.flatnonzero(active)
        dd = _lane(d, idx)
        full = full_of(bounds(dd, Vint[idx]), y[idx])
        dV = poisson_delta(full, dd, take(s, idx), take(ion, idx))
        shift = dV / _col(dd["Vt"])
        y[idx] = y[idx] + np.stack([dV, shift, -shift], -1)
        size[idx] = np.max(np.abs(shift), 1)
        it[idx] += 1
    return y


def _scaled(s, ion, share):
    """solver._scaled_ions (solver.py:2012-2015)."""
    s = dict(s, a_fix=s["a_fix"] * share, c_fix=s["c_fix"] * share)
    return s, dict(ion, a_totals=ion["a_totals"] * share, c_totals=ion["c_totals"] * share)


def _finite(y, logs):
    return np.all(np.isfinite(y), axis=(1, 2)) & np.all(np.isfinite(logs), 1)


def _with(d, s=None, ion=None):
    out = dict(d)
    if s is not None:
        out["s"] = s
    if ion is not None:
        out["ion"] = ion
    return out


def start(d, first, bern, tol, start_iter, strict=False):
    """batch._start (batch.py:875-934), Boltzmann ions, no charged traps: Poisson's start, then
    Newton at `first`, through `ION_DENSITY_STAGES` where that fails on a device with ions."""
    s0, ion0 = d["s"], d["ion"]
    y0 = initial(d, first)[:, 1:-1]
    y = poisson_solve(y0, d, s0, ion0, first, start_iter)
    bnd = bounds(d, first)
    logs = ion_logs(np.concatenate([bnd[:, :1, 0], y[..., 0], bnd[:, 1:, 0]], 1), ion0, d["Vt"])
    y_f, logs_f, _, ok_f, _ = newton_loop(y, logs, d, first, bern, tol, start_iter, strict)
    mobile = np.any(_masks(ion0)[1] > 0, 1)
    done = ok_f | ~mobile
    y_c, logs_c, before = y, logs, 1.0
    ok_c = np.ones_like(done)
    for share in ION_DENSITY_STAGES:
        s_k, ion_k = _scaled(s0, ion0, share)
        logs_c = logs_c + np.log(share / before)
        y_k, logs_k, _, ok_c, _ = newton_loop(y_c, logs_c, _with(d, s_k, ion_k), first, bern,
                                               tol, start_iter, strict, skip=done)
        kept = _finite(y_k, logs_k)
        y_c = np.where(kept[:, None, None], y_k, y_c)
        logs_c = np.where(kept[:, None], logs_k, logs_c)
        before = share
    staged = ~done & ok_c
    kept = _finite(y_f, logs_f)
    y = np.where(staged[:, None, None], y_c, np.where(kept[:, None, None], y_f, y))
    logs = np.where(staged[:, None], logs_c, np.where(kept[:, None], logs_f, logs))
    return y, logs, ok_f | staged


def freeze(s, ion, y, logs, Vt, flag):
    """batch._freeze (batch.py:859-872): the mobile ions of `y` as fixed densities."""
    la, lc = point_logs(logs, ion)
    V = y[..., 0]
    anion = s["a_fix"] + s["a_mask"] * np.exp(la + V / _col(Vt))
    cation = s["c_fix"] + s["c_mask"] * np.exp(lc - V / _col(Vt))
    f = flag[:, None]
    s = dict(s, a_fix=np.where(f, anion, s["a_fix"]), c_fix=np.where(f, cation, s["c_fix"]),
             a_mask=np.where(f, 0.0, s["a_mask"]), c_mask=np.where(f, 0.0, s["c_mask"]))
    ion = dict(ion)
    for k in ("a_slots", "c_slots"):
        ion[k] = np.where(flag[:, None, None], 0.0, ion[k])
    for k in ("a_totals", "c_totals"):
        ion[k] = np.where(flag[:, None], 0.0, ion[k])
    return s, ion


def solve_one(d, voltages, bern, tol, max_iter, start_iter, strict=False, states=False):
    """batch._solve_one (batch.py:937-1006) for every lane at once: start, pre-bias (ions
    frozen after it where `fixIons`), then the scan outwards from the pre-bias — up, then down
    from the pre-bias solution again — each voltage from the last two converged solutions
    extrapolated, the change held to one step's caps. `voltages` ascending."""
    nb = d["Vt"].shape[0]
    nv = len(voltages)
    first = np.where(d["pre_cond"] > 0, d["V_pre"], voltages[0])
    y, logs, solved = start(d, first, bern, tol, start_iter, strict)
    y, logs, _, pre_ok, _ = newton_loop(y, logs, d, first, bern, tol, start_iter, strict,
                                        skip=solved)
    frozen = (d["pre_cond"] > 0) & (d["fix_ions"] > 0)
    s, ion = freeze(d["s"], d["ion"], y, logs, d["Vt"], frozen)
    dz = _with(d, s, ion)
    pre_ok = pre_ok | ~frozen
    caps = _caps(d["Vt"])
    below = np.searchsorted(voltages, first, side="left")
    j = np.arange(nv)
    order = np.where(j[None, :] < (nv - below)[:, None], below[:, None] + j[None, :],
                     nv - 1 - j[None, :])
    turn = j[None, :] == (nv - below)[:, None]
    st = (y, logs, y, logs, first.astype(float), first.astype(float))
    carry = tuple(a.copy() for a in st)
    J_out = np.zeros((nb, nv))
    ok_out = np.zeros((nb, nv), bool)
    it_out = np.zeros((nb, nv), int)
    if states:
        y_out = np.zeros((nb, nv) + y.shape[1:])
        l_out = np.zeros((nb, nv, logs.shape[1]))
    for k in range(nv):
        t = turn[:, k]
        carry = tuple(np.where(t.reshape((-1,) + (1,) * (a.ndim - 1)), a0, a)
                      for a0, a in zip(st, carry))
        yc, lc_, yp, lp, V_last, V_before = carry
        Vint = voltages[order[:, k]]
        with np.errstate(divide="ignore", invalid="ignore"):
            ratio = np.where(V_last != V_before, (Vint - V_last) / (V_last - V_before), 0.0)
        guess = yc + np.clip(ratio[:, None, None] * (yc - yp), -caps, caps)
        lguess = lc_ + np.clip(ratio[:, None] * (lc_ - lp), -ION_LOG_CAP, ION_LOG_CAP)
        y_new, logs_new, J, ok, its = newton_loop(guess, lguess, dz, Vint, bern, tol, max_iter,
                                                  strict)
        keep = ok & _finite(y_new, logs_new)
        new = (y_new, logs_new, yc, lc_, Vint, V_last)
        carry = tuple(np.where(keep.reshape((-1,) + (1,) * (a.ndim - 1)), b, a)
                      for b, a in zip(new, carry))
        rows = np.arange(nb)
        J_out[rows, order[:, k]] = J
        ok_out[rows, order[:, k]] = ok
        it_out[rows, order[:, k]] = its
        if states:
            y_out[rows, order[:, k]] = y_new
            l_out[rows, order[:, k]] = logs_new
    if states:
        return J_out, ok_out & pre_ok[:, None], it_out, (y_out, l_out, dz)
    return J_out, ok_out & pre_ok[:, None], it_out


def solve_batch(batch, voltages, tol=1e-10, max_iter=60, first_max_iter=6,
                bernoulli_name="exact", strict=False):
    """batch.solve_batch / _passes / _solve_batch (batch.py:1033-1047, 1136-1162, 1194-1208):
    `(J, converged, iterations)`, batch × voltages in the caller's order, the shunt's current
    added. Two passes: every device with `first_max_iter` steps per voltage, then the devices
    with a voltage that missed it, with `max_iter`."""
    bern = BERNOULLI[bernoulli_name]
    voltages = np.asarray(voltages, dtype=float)
    order = np.argsort(voltages, kind="stable")
    inv = np.argsort(order, kind="stable")
    vs = voltages[order]

    def run(part, cap):
        J, ok, its = solve_one(part, vs, bern, tol, cap, max_iter, strict)
        return J[:, inv], ok[:, inv], its[:, inv]

    if first_max_iter is None or first_max_iter >= max_iter:
        J, ok, its = run(batch, max_iter)
    else:
        J, ok, its = run(batch, first_max_iter)
        idx = np.flatnonzero(~ok.all(axis=1))
        if idx.size:
            J2, ok2, its2 = run(take(batch, idx), max_iter)
            J[idx], ok[idx], its[idx] = J2, ok2, its2
    return J + batch["G_shunt"][:, None] * voltages[None, :], ok, its


def observed(d, y, logs, Vint):
    """batch._observed (batch.py:1009-1030) in this scope (contacts of infinite surface
    recombination, no free ends, no field-dependent rates): the solution on all NP + 2 points,
    its implied V_oc and PLQY of direct recombination (`solver.solve_state`,
    solver.py:2079-2089) and the ions on the grid (`_ions_on_grid`, solver.py:2096-2102). `d` the
    tree after any freeze; one voltage per lane."""
    s, ion = d["s"], d["ion"]
    full = full_of(bounds(d, Vint), y)
    n, p = np.exp(full[:, 1:-1, 1]), np.exp(full[:, 1:-1, 2])
    vol = s["fac"] / (_col(d["L"]) * s["hm"] * s["hp"])  # solver._volumes (1952-1954)
    k = d["rec"]["kd"][:, 1:-1]
    rad = np.sum(vol * k * n * p, 1)
    rad0 = np.sum(vol * k * d["rec"]["ni2"][:, 1:-1], 1)
    gen = d["g_frac"] * np.sum(vol * d["G"][:, 1:-1], 1)
    with np.errstate(divide="ignore", invalid="ignore"):
        voc = np.where(rad0 > 0, d["Vt"] * np.log(rad / np.where(rad0 > 0, rad0, 1.0)), np.nan)
        plqy = np.where(gen > 0, (rad - rad0) / np.where(gen > 0, gen, 1.0), np.nan)
    la, lc = point_logs(logs, ion)
    V = y[..., 0]
    anion = s["a_fix"] + s["a_mask"] * np.exp(la + V / _col(d["Vt"]))
    cation = s["c_fix"] + s["c_mask"] * np.exp(lc - V / _col(d["Vt"]))
    pad = lambda a: np.concatenate([a[:, :1], a, a[:, -1:]], 1)  # noqa: E731
    return full, voc, plqy, np.stack([pad(anion), pad(cation)], -1)


def solve_states(batch, voltages=0.0, tol=1e-10, max_iter=60, bernoulli_name="exact",
                 strict=False):
    """batch.solve_states (batch.py:1165-1191): the steady states at `voltages` and what
    photoluminescence measures of them; a dict of `V, n, p, qfls, anion, cation`
    (batch × voltages × NP + 2), `implied_voc, plqy, J, converged, iterations`
    (batch × voltages). One pass at `max_iter` (what jaxdd's two passes give)."""
    bern = BERNOULLI[bernoulli_name]
    voltages = np.atleast_1d(np.asarray(voltages, dtype=float))
    order = np.argsort(voltages, kind="stable")
    inv = np.argsort(order, kind="stable")
    vs = voltages[order]
    J, ok, its, (ys, ls, dz) = solve_one(batch, vs, bern, tol, max_iter, max_iter, strict,
                                         states=True)
    nb, nv = J.shape
    full = np.zeros((nb, nv) + (ys.shape[2] + 2, 3))
    voc, plqy = np.zeros((nb, nv)), np.zeros((nb, nv))
    ions = np.zeros((nb, nv, ys.shape[2] + 2, 2))
    for k in range(nv):
        full[:, k], voc[:, k], plqy[:, k], ions[:, k] = observed(
            dz, ys[:, k], ls[:, k], np.full(nb, vs[k]))
    n, p = np.exp(full[..., 1]), np.exp(full[..., 2])
    qfls = batch["Vt"][:, None, None] * np.log(n * p / batch["rec"]["ni2"][:, None, :])
    J = J + batch["G_shunt"][:, None] * vs[None, :]
    out = {"V": full[..., 0], "n": n, "p": p, "qfls": qfls, "implied_voc": voc, "plqy": plqy,
           "J": J, "converged": ok, "iterations": its, "anion": ions[..., 0],
           "cation": ions[..., 1]}
    return {k: v[:, inv] for k, v in out.items()}


# ----------------------------------------------------------------------------- solve_jv

def noise_step(y, logs, bnd, d, bern):
    """solver._noise_step (solver.py:1728-1751): the step the residual's round-off alone
    gives, as `_newton_step` measures its step."""
    la, lc = point_logs(logs, d["ion"])
    full = full_of(bnd, y)
    _, A, Bb, C, _ = assemble(full, d["s"], d["ti"], d["Vt"], d["g_frac"], la, lc, bern)
    a = np.abs(full)
    noise = np.finfo(float).eps * (np.einsum("bnrc,bnc->bnr", np.abs(A), a[:, :-2])
                                   + np.einsum("bnrc,bnc->bnr", np.abs(Bb), a[:, 1:-1])
                                   + np.einsum("bnrc,bnc->bnr", np.abs(C), a[:, 2:]))
    X = block_thomas(A, Bb, C, noise[..., None])[..., 0]
    dens = np.exp(y[..., 1:])
    weight = dens / (dens + d["s"]["n_floor"][..., None])
    return np.maximum(np.max(np.abs(X[..., 0]), 1) / d["Vt"],
                      np.max(np.abs(X[..., 1:]) * weight, axis=(1, 2)))


def _settle(y, logs, d, Vint, bern, tol, max_iter):
    """solver._scan.settle (solver.py:2132-2173), no contacts: Newton to `tol`, the round-off
    floor, or the problem's own noise floor (`noise_step`). One lane."""
    bnd = bounds(d, np.array([Vint]))
    sizes: list[float] = []
    floor = None
    steps = 0
    while steps < max_iter:
        y, logs, size = newton_step(y, logs, bnd, d, d["s"], d["ion"], bern)
        steps += 1
        sizes.append(float(size[0]))
        if np.isnan(sizes[-1]):
            return y, logs, False, steps
        recent = sizes[-STALL_STEPS - 1:]
        done = sizes[-1] < tol or (len(recent) > STALL_STEPS and max(recent) < ROUND_OFF_FLOOR
                                   and min(recent[1:]) >= 0.1 * recent[0])
        if not done and len(recent) > STALL_STEPS and max(recent) < NOISE_FLOOR_CAP:
            if floor is None:
                floor = float(noise_step(y, logs, bnd, d, bern)[0])
            done = max(recent) < floor
        if done:
            return y, logs, True, steps
    return y, logs, False, steps


def _initial_jv(dev, Vint):
    """solver._initial (solver.py:1882-1893)."""
    x, L, e = dev.x, dev.L, dev.left_elec
    V = dev.V0 + 0.5 * e * Vint + x * (dev.VL - dev.V0 - e * Vint) / L
    EF = dev.W_L - x * (dev.W_L - dev.W_R) / L
    n = dev.N_c * np.exp(-(EF - dev.E_c) / dev.Vt)
    p = dev.ni ** 2 / n
    return np.stack([V, np.log(n), np.log(p)], -1)


def _scan_jv(dev, voltages, g_frac, tol, max_iter, bern):
    """solver._scan (solver.py:2105-2245): the start, the pre-bias and its freeze, then each
    voltage in the caller's order from the last converged solution. Yields per voltage
    `(Vint, y, logs, converged, iterations, dz)`: the final iterate (even where Newton did not
    converge) and the tree it was solved in (after any freeze). Raises `RuntimeError` where the
    pre-bias does not converge."""
    d = prepare([dev])
    if g_frac is not None:
        d["g_frac"] = np.array([float(g_frac)])
    voltages = np.asarray(voltages, dtype=float)
    first = dev.V_pre if dev.pre_cond else float(voltages[0])
    yfull = _initial_jv(dev, first)[None]
    y = yfull[:, 1:-1].copy()
    mobile = bool(np.any(_masks(d["ion"])[1] > 0))
    for _ in range(max_iter):
        full = full_of(bounds(d, np.array([first])), y)
        dV = poisson_delta(full, d, d["s"], d["ion"], coupled=mobile)
        shift = dV / d["Vt"][:, None]
        y = y + np.stack([dV, shift, -shift], -1)
        if float(np.max(np.abs(shift))) < 1e-8:
            break
    bnd = bounds(d, np.array([first]))
    logs = ion_logs(full_of(bnd, y)[..., 0], d["ion"], d["Vt"])
    if mobile:
        y_f, logs_f, ok, _ = _settle(y, logs, d, first, bern, tol, max_iter)
        if not ok:
            y_c, logs_c, before = y, logs, 1.0
            for share in ION_DENSITY_STAGES:
                s_k, ion_k = _scaled(d["s"], d["ion"], share)
                logs_c = logs_c + np.log(share / before)
                y_c, logs_c, ok, _ = _settle(y_c, logs_c, _with(d, s_k, ion_k), first, bern,
                                             tol, max_iter)
                before = share
                if not ok:
                    break
            if ok:
                y_f, logs_f = y_c, logs_c
        if ok:
            y, logs = y_f, logs_f
    dz = d
    if dev.pre_cond:
        y, logs, ok, _ = _settle(y, logs, d, dev.V_pre, bern, tol, max_iter)
        if not ok:
            raise RuntimeError(f"no convergence at the pre-bias {dev.V_pre} V")
        if dev.fix_ions:
            s, ion = freeze(d["s"], d["ion"], y, logs, d["Vt"], np.array([True]))
            dz = _with(d, s, ion)
    for Vint in voltages:
        y_new, logs_new, ok, it = _settle(y, logs, dz, float(Vint), bern, tol, max_iter)
        full = full_of(bounds(dz, np.array([float(Vint)])), y_new)
        if ok and np.isfinite(full).all() and np.isfinite(logs_new).all():
            y, logs = y_new, logs_new
        yield float(Vint), y_new, logs_new, ok, it, dz


def solve_jv(dev, voltages, g_frac=None, tol=1e-10, max_iter=200, bernoulli_name="exact"):
    """solver.solve_jv (solver.py:2041-2060) over `_scan_jv`: each voltage in the caller's order
    from the last converged solution. Returns `(J, converged, iterations)`; raises
    `RuntimeError` where the pre-bias does not converge."""
    bern = BERNOULLI[bernoulli_name]
    J, conv, its = [], [], []
    for Vint, y, _, ok, it, dz in _scan_jv(dev, voltages, g_frac, tol, max_iter, bern):
        Jv = float(current(dz, full_of(bounds(dz, np.array([Vint])), y), bern)[0])
        J.append(Jv + (Vint / dev.R_shunt if dev.R_shunt > 0 else 0.0))
        conv.append(ok)
        its.append(it)
    return np.array(J), np.array(conv), np.array(its)


def solve_state(dev, Vint=0.0, g_frac=None, tol=1e-10, max_iter=200, bernoulli_name="exact"):
    """solver.solve_state (solver.py:2063-2093) in this scope (Boltzmann statistics, contacts of
    infinite surface recombination, no field-dependent rates): `_scan_jv` at the one voltage
    `Vint`, its state on all NP + 2 points and what photoluminescence measures of it
    (`observed`). A dict of `x, V, n, p, qfls, anion, cation` (NP + 2), `implied_voc`, `plqy`,
    `J` (`_current`: without the shunt's current, as jaxdd's `solve_state` has it),
    `converged`, `iterations`."""
    bern = BERNOULLI[bernoulli_name]
    (Vint, y, logs, ok, it, dz), = _scan_jv(dev, [Vint], g_frac, tol, max_iter, bern)
    full, voc, plqy, ions = observed(dz, y, logs, np.array([Vint]))
    n, p = np.exp(full[0, :, 1]), np.exp(full[0, :, 2])
    return {"x": np.asarray(dev.x), "V": full[0, :, 0], "n": n, "p": p,
            "qfls": dev.Vt * np.log(n * p / dev.ni ** 2), "implied_voc": float(voc[0]),
            "plqy": float(plqy[0]), "J": float(current(dz, full, bern)[0]),
            "anion": ions[0, :, 0], "cation": ions[0, :, 1], "converged": bool(ok),
            "iterations": int(it)}
